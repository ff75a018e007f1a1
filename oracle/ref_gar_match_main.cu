// Host driver of the reference's GARMatch kernels, compiled by
// oracle/build_ref.sh together with the reference's own
// core/task/gpu_task/kernel/kernel_gar_match.cu where it lies (TEST
// INFRASTRUCTURE ONLY: tests/test_gar_ref_gpu.py runs it on the GPU to pin
// the GAR oracle and matrixgraph_gar_match against the reference's real
// output).  It calls GARMatchKernelWrapper::GARMatch
// (kernel_gar_match.cu:365-709) — the function GARMatch::Run
// (core/task/gpu_task/gar_match.cu:193-242) calls for the C-ABI
// matrixgraph_gar_match — without the yaml-based task around it.
//
//   ref_gar_match IN OUT [REPS]
// With REPS > 1 the call is repeated REPS times on the same inputs and the
// median wall time of calls 2..REPS (host arrays in and out, as the
// reference's C-ABI call) is printed to stderr as "ref_gar_match_ms <t>".
// IN (little-endian): int32 n_vertices, n_edges, p_nodes, p_edges,
// row_capacity, match_capacity, has_v_id, has_e_label, has_p_edge_label;
// then uint32 v_id[n_vertices], int32 v_label[n_vertices], uint32
// e_src[n_edges], e_dst[n_edges], e_id[n_edges], int32 e_label[n_edges],
// p_node_label[p_nodes], p_edge_src[p_edges], p_edge_dst[p_edges],
// p_edge_label[p_edges].  An array whose has_ flag is 0 is passed to the
// reference as a null pointer (its contents in the file are ignored), as
// the reference treats absent ids and edge labels.
// OUT: int32 status, num_conditions, row_size, match_size; then row_size
// entries each of uint32 pivot, int32 cond_j, pos, offset, count; then uint32
// matched_v_ids[match_size].  The reference's own log goes to stdout.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "core/task/gpu_task/kernel/kernel_gar_match.cuh"

namespace K = sics::matrixgraph::core::task::kernel;

template <class T>
static bool read_vec(FILE* f, std::vector<T>& v, int n) {
  v.resize(n > 0 ? size_t(n) : 0);
  return n <= 0 || std::fread(v.data(), sizeof(T), size_t(n), f) == size_t(n);
}

int main(int argc, char** argv) {
  if (argc != 3 && argc != 4) {
    std::fprintf(stderr, "usage: ref_gar_match IN OUT [REPS]\n");
    return 2;
  }
  const int reps = argc == 4 ? std::max(1, std::atoi(argv[3])) : 1;
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int32_t h[9];
  if (std::fread(h, 4, 9, in) != 9) return 2;
  const int nv = h[0], ne = h[1], pn = h[2], pe = h[3], row_cap = h[4], match_cap = h[5];
  std::vector<uint32_t> v_id, e_src, e_dst, e_id;
  std::vector<int32_t> v_label, e_label, p_label, p_src, p_dst, p_elabel;
  bool ok = read_vec(in, v_id, nv) && read_vec(in, v_label, nv) && read_vec(in, e_src, ne) &&
            read_vec(in, e_dst, ne) && read_vec(in, e_id, ne) && read_vec(in, e_label, ne) &&
            read_vec(in, p_label, pn) && read_vec(in, p_src, pe) && read_vec(in, p_dst, pe) &&
            read_vec(in, p_elabel, pe);
  std::fclose(in);
  if (!ok) return 2;
  K::GARGraphArrays g{h[6] ? v_id.data() : nullptr, v_label.data(), nv, e_src.data(),
                      e_dst.data(), e_id.data(), h[7] ? e_label.data() : nullptr, ne};
  K::GARPatternArrays p{p_label.data(), pn, p_src.data(), p_dst.data(),
                        h[8] ? p_elabel.data() : nullptr, pe};
  int num_conditions = 0, row_size = 0, match_size = 0;
  std::vector<uint32_t> pivot(size_t(row_cap > 0 ? row_cap : 1)),
      ids(size_t(match_cap > 0 ? match_cap : 1));
  std::vector<int32_t> cond(pivot.size()), pos(pivot.size()), off(pivot.size()),
      cnt(pivot.size());
  K::GARMatchArrays out{&num_conditions, pivot.data(), cond.data(), pos.data(), off.data(),
                        cnt.data(), row_cap, &row_size, ids.data(), match_cap, &match_size};
  int status = 0;
  std::vector<double> ms;
  for (int rep = 0; rep < reps; ++rep) {
    num_conditions = row_size = match_size = 0;
    const auto t0 = std::chrono::steady_clock::now();
    status = K::GARMatchKernelWrapper::GARMatch(g, p, &out);
    const auto t1 = std::chrono::steady_clock::now();
    if (rep > 0) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
  }
  if (!ms.empty()) {
    std::sort(ms.begin(), ms.end());
    std::fprintf(stderr, "ref_gar_match_ms %.6f\n", ms[ms.size() / 2]);
  }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 2;
  const int32_t head[4] = {status, num_conditions, row_size, match_size};
  std::fwrite(head, 4, 4, o);
  for (int r = 0; r < row_size; ++r) {
    std::fwrite(&pivot[r], 4, 1, o);
    std::fwrite(&cond[r], 4, 1, o);
    std::fwrite(&pos[r], 4, 1, o);
    std::fwrite(&off[r], 4, 1, o);
    std::fwrite(&cnt[r], 4, 1, o);
  }
  if (match_size > 0) std::fwrite(ids.data(), 4, size_t(match_size), o);
  std::fclose(o);
  return 0;
}
