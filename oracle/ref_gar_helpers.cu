// Host driver over three helpers of the reference's GAR vertex filters,
// compiled against the reference's own headers by oracle/build_ref.sh:
//   MinHeap::Insert          core/data_structures/heap.cuh:18-111
//   MiniKernelBitmap::Count  core/data_structures/mini_kernel_bitmap.cuh:53-63
//   HashTable                core/task/gpu_task/kernel/algorithms/hash.cuh:31-65
// It prints one JSON object with their outputs on fixed inputs; the CPU
// restatement in oracle/gar.py is pinned against it.  Test infrastructure.
#include <cstdint>
#include <cstdio>
#include <limits>

#include "core/data_structures/heap.cuh"
#include "core/data_structures/mini_kernel_bitmap.cuh"
#include "core/task/gpu_task/kernel/algorithms/hash.cuh"

namespace K = sics::matrixgraph::core::task::kernel;

static uint32_t lcg(uint64_t* s) {
  *s = *s * 6364136223846793005ull + 1442695040888963407ull;
  return uint32_t(*s >> 33);
}

int main() {
  std::printf("{\"hash\": [");
  for (uint32_t key = 0; key < 40; ++key) std::printf("%s%u", key ? ", " : "", K::HashTable(key));
  std::printf("], \"count\": [");
  uint64_t s = 12345;
  for (int i = 0; i < 96; ++i) {
    uint32_t x = i < 32 ? (1u << i) : (i < 64 ? ((1u << (i - 32)) - 1u) : lcg(&s));
    K::MiniKernelBitmap b(32);
    for (uint32_t bit = 0; bit < 32; ++bit)
      if (x >> bit & 1u) b.SetBit(bit);
    std::printf("%s[%u, %u]", i ? ", " : "", x, b.Count());
  }
  std::printf("], \"heap\": [");
  for (int t = 0; t < 300; ++t) {
    const uint32_t len = lcg(&s) % 24;
    const uint32_t range = t % 3 == 0 ? 16u : 1000u;
    K::MinHeap h;
    std::printf("%s{\"in\": [", t ? ", " : "");
    for (uint32_t j = 0; j < len; ++j) {
      const uint32_t v = lcg(&s) % range;
      h.Insert(v);
      std::printf("%s%u", j ? ", " : "", v);
    }
    std::printf("], \"offset\": %u, \"data\": [", h.get_offset());
    for (uint32_t j = 0; j < h.get_offset(); ++j)
      std::printf("%s%u", j ? ", " : "", h.get_element_by_idx(j));
    std::printf("]}");
  }
  std::printf("]}\n");
  return 0;
}
