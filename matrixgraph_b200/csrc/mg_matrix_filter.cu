// Lossy learned candidate filter, compatible with the reference's
// MatrixFilter (core/task/cpu_task/cpu_subiso.cu:237-277) and its CPU MLP
// helpers (core/task/gpu_task/kernel/kernel_matrix_ops.cu:76-181, 431-509):
//   sim  = (e_u - e_v)^2                      elementwise, float32
//   z1   = relu(W1 . sim + b1)                W1: hidden rows x dim
//   z2   = W2 . z1 + b2                       W2: hidden x 1
//   keep = !(1 / (1 + exp(-z2)) < 0.1)
// Every product and sum is rounded to float32 separately, in the order of the
// reference's scalar loops (no fused multiply-add), so the keep decision
// equals the reference's except where the sigmoid sits within an ulp or two
// of the threshold.  One warp evaluates one candidate: the lanes form the
// squared differences, then each lane accumulates the hidden units it owns
// over the dimensions in order; W1 is stored transposed so those reads are
// coalesced.  The enumerator applies the filter to the level-0 candidates
// (a bitmap over data vertices, built once per call).
#include <algorithm>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "mg_device.cuh"

namespace mg {

constexpr uint32_t kMfMaxHidden = 64;   // the reference's z1[64]
constexpr uint32_t kMfMaxDim = 1024;
constexpr int kMfBlock = 256;

struct MatrixFilter {
  int device = 0;
  uint32_t k_rows = 0, n_rows = 0, dim = 0, hidden = 0;
  std::vector<float> query_emb;  // k_rows x dim
  float* data_emb = nullptr;     // n_rows x dim (device)
  float* w1t = nullptr;          // dim x hidden (W1 transposed, device)
  float* b1 = nullptr;           // hidden (device)
  float* w2 = nullptr;           // hidden (device)
  float* eu = nullptr;           // dim: embedding of the query vertex asked about
  float b2 = 0.f;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  ~MatrixFilter() {
    for (float* p : {data_emb, w1t, b1, w2, eu})
      if (p) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// <dir>meta.yaml (keys x and y) and <dir>embedding.bin (x*y float32,
// row-major): core/data_structures/matrix.cu:12-35.
int read_matrix(const std::string& dir, uint64_t* x, uint64_t* y, std::vector<float>* data) {
  std::ifstream mf(dir + "meta.yaml");
  if (!mf) return set_error(MG_E_IO, "cannot open %smeta.yaml", dir.c_str());
  *x = *y = 0;
  std::string line;
  while (std::getline(mf, line)) {
    std::stringstream ss(line);
    std::string key;
    if (!std::getline(ss, key, ':')) continue;
    uint64_t v = 0;
    if (key == "x" && (ss >> v)) *x = v;
    if (key == "y" && (ss >> v)) *y = v;
  }
  if (*x == 0 || *y == 0 || *x * *y > (1ull << 34))
    return set_error(MG_E_FORMAT, "%smeta.yaml: bad shape %llu x %llu", dir.c_str(),
                     (unsigned long long)*x, (unsigned long long)*y);
  data->resize(*x * *y);
  std::ifstream bf(dir + "embedding.bin", std::ios::binary);
  if (!bf || !bf.read(reinterpret_cast<char*>(data->data()),
                      std::streamsize(data->size() * sizeof(float))))
    return set_error(MG_E_FORMAT, "%sembedding.bin: fewer than %llu float32 values",
                     dir.c_str(), (unsigned long long)data->size());
  return MG_OK;
}

}  // namespace

__global__ void __launch_bounds__(kMfBlock) k_matrix_filter(
    const float* __restrict__ data_emb, const float* __restrict__ eu,
    const float* __restrict__ w1t, const float* __restrict__ b1, const float* __restrict__ w2,
    float b2, uint32_t dim, uint32_t hidden, const uint32_t* __restrict__ cand, uint64_t ncand,
    uint8_t* keep_bytes, uint32_t* keep_bits) {
  extern __shared__ float smem[];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  float* sim = smem + wib * (dim + kMfMaxHidden);
  float* z1 = sim + dim;
  for (uint64_t c = uint64_t(blockIdx.x) * wpb + wib; c < ncand; c += uint64_t(gridDim.x) * wpb) {
    const uint32_t v = __ldg(cand + c);
    const float* ev = data_emb + uint64_t(v) * dim;
    for (uint32_t p = lane; p < dim; p += 32) {
      const float d = __fsub_rn(__ldg(eu + p), __ldg(ev + p));
      sim[p] = __fmul_rn(d, d);
    }
    __syncwarp();
    for (uint32_t j = lane; j < hidden; j += 32) {
      float z = 0.f;
      for (uint32_t p = 0; p < dim; ++p)
        z = __fadd_rn(z, __fmul_rn(sim[p], __ldg(w1t + uint64_t(p) * hidden + j)));
      z = __fadd_rn(z, __ldg(b1 + j));
      z1[j] = z > 0.f ? z : 0.f;
    }
    __syncwarp();
    if (lane == 0) {
      float z2 = 0.f;
      for (uint32_t j = 0; j < hidden; ++j) z2 = __fadd_rn(z2, __fmul_rn(z1[j], __ldg(w2 + j)));
      z2 = __fadd_rn(z2, b2);
      const float s = 1.0f / (1.0f + expf(-z2));
      const bool keep = !(s < 0.1f);
      if (keep_bytes) keep_bytes[c] = keep ? 1 : 0;
      if (keep_bits && keep) atomicOr(keep_bits + (v >> 5), 1u << (v & 31));
    }
    __syncwarp();
  }
}

// Keep bits of every vertex of label bucket `lab` for query vertex u, into
// bits (ceil(n/32) words, cleared here), on stream st.
int matrix_filter_roots(void* filter, const DevGraph* dg, uint32_t u, uint32_t lab,
                        uint32_t* bits, cudaStream_t st) {
  auto* F = static_cast<MatrixFilter*>(filter);
  std::lock_guard<std::mutex> lock(F->mu);
  if (F->device != dg->device)
    return set_error(MG_E_ARG, "matrix filter on device %d, graph on device %d", F->device,
                     dg->device);
  if (u >= F->k_rows)
    return set_error(MG_E_ARG, "matrix filter: query vertex %u, %u query embeddings", u,
                     F->k_rows);
  if (dg->g.n > F->n_rows)
    return set_error(MG_E_ARG, "matrix filter: %u data embeddings for %u vertices", F->n_rows,
                     dg->g.n);
  MG_CK(cudaMemsetAsync(bits, 0, ((uint64_t(dg->g.n) + 31) / 32) * 4, st));
  MG_CK(cudaMemcpyAsync(F->eu, F->query_emb.data() + uint64_t(u) * F->dim, F->dim * 4ull,
                        cudaMemcpyHostToDevice, st));
  const uint64_t b0 = dg->h_bucket_off[lab], nb = dg->h_bucket_off[lab + 1] - b0;
  if (nb == 0) return MG_OK;
  const size_t smem = (kMfBlock / 32) * (F->dim + kMfMaxHidden) * sizeof(float);
  const uint64_t blocks = std::min<uint64_t>((nb + kMfBlock / 32 - 1) / (kMfBlock / 32),
                                             uint64_t(dg->sms) * 16);
  k_matrix_filter<<<unsigned(blocks), kMfBlock, smem, st>>>(
      F->data_emb, F->eu, F->w1t, F->b1, F->w2, F->b2, F->dim, F->hidden,
      dg->g.bucket_vid + b0, nb, nullptr, bits);
  MG_CK(cudaGetLastError());
  // F->eu is rewritten by the next call: finish this one first
  MG_CK(cudaStreamSynchronize(st));
  return MG_OK;
}

}  // namespace mg

extern "C" {

int mg_matrix_filter_load(const char* const dirs[6], int device, void** filter) {
  mg::clear_error();
  if (!dirs || !filter) return mg::set_error(MG_E_ARG, "null argument");
  for (int i = 0; i < 6; ++i)
    if (!dirs[i] || !dirs[i][0]) return mg::set_error(MG_E_ARG, "matrix path %d is empty", i + 1);
  uint64_t x[6], y[6];
  std::vector<float> m[6];
  for (int i = 0; i < 6; ++i) {
    int rc = mg::read_matrix(dirs[i], &x[i], &y[i], &m[i]);
    if (rc) return rc;
  }
  const uint64_t dim = y[0], hidden = x[2];
  if (y[1] != dim || y[2] != dim)
    return mg::set_error(MG_E_FORMAT, "matrix filter: embedding widths %llu, %llu and W1 width "
                         "%llu differ", (unsigned long long)y[0], (unsigned long long)y[1],
                         (unsigned long long)y[2]);
  if (hidden == 0 || hidden > mg::kMfMaxHidden || dim > mg::kMfMaxDim)
    return mg::set_error(MG_E_FORMAT, "matrix filter: hidden %llu (at most %u), dim %llu (at "
                         "most %u)", (unsigned long long)hidden, mg::kMfMaxHidden,
                         (unsigned long long)dim, mg::kMfMaxDim);
  if (x[3] * y[3] != hidden || x[4] != hidden || y[4] != 1 || x[5] * y[5] != 1)
    return mg::set_error(MG_E_FORMAT, "matrix filter: b1 %llux%llu, W2 %llux%llu, b2 %llux%llu "
                         "do not fit %llu hidden units", (unsigned long long)x[3],
                         (unsigned long long)y[3], (unsigned long long)x[4],
                         (unsigned long long)y[4], (unsigned long long)x[5],
                         (unsigned long long)y[5], (unsigned long long)hidden);
  if (x[0] > 0xFFFFFFFFull || x[1] > 0xFFFFFFFFull)
    return mg::set_error(MG_E_FORMAT, "matrix filter: more than 2^32 embedding rows");
  mg::DeviceGuard guard(device);
  auto* F = new mg::MatrixFilter();
  F->device = device;
  F->k_rows = uint32_t(x[0]);
  F->n_rows = uint32_t(x[1]);
  F->dim = uint32_t(dim);
  F->hidden = uint32_t(hidden);
  F->query_emb = std::move(m[0]);
  F->b2 = m[5][0];
  std::vector<float> w1t(dim * hidden);
  for (uint64_t j = 0; j < hidden; ++j)
    for (uint64_t p = 0; p < dim; ++p) w1t[p * hidden + j] = m[2][j * dim + p];
  auto up = [&](float** d, const float* h, uint64_t count) -> int {
    if (cudaMalloc(d, std::max<uint64_t>(count, 1) * 4) != cudaSuccess) {
      cudaGetLastError();
      *d = nullptr;
      return mg::set_error(MG_E_OOM, "matrix filter: cudaMalloc of %llu floats",
                           (unsigned long long)count);
    }
    if (h && cudaMemcpy(*d, h, count * 4, cudaMemcpyHostToDevice) != cudaSuccess)
      return mg::set_error(MG_E_CUDA, "matrix filter: copy to the device failed");
    return MG_OK;
  };
  int rc = up(&F->data_emb, m[1].data(), m[1].size());
  if (!rc) rc = up(&F->w1t, w1t.data(), w1t.size());
  if (!rc) rc = up(&F->b1, m[3].data(), hidden);
  if (!rc) rc = up(&F->w2, m[4].data(), hidden);
  if (!rc) rc = up(&F->eu, nullptr, dim);
  if (!rc && cudaStreamCreateWithFlags(&F->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = mg::set_error(MG_E_CUDA, "matrix filter: cudaStreamCreate failed");
  if (rc) {
    delete F;
    return rc;
  }
  *filter = F;
  return MG_OK;
}

void mg_matrix_filter_free(void* filter) {
  if (!filter) return;
  auto* F = static_cast<mg::MatrixFilter*>(filter);
  mg::DeviceGuard guard(F->device);
  delete F;
}

int mg_matrix_filter_keep(void* filter, uint32_t u, const uint32_t* v, uint64_t nv,
                          uint8_t* keep) {
  mg::clear_error();
  if (!filter || (nv && (!v || !keep))) return mg::set_error(MG_E_ARG, "null argument");
  auto* F = static_cast<mg::MatrixFilter*>(filter);
  std::lock_guard<std::mutex> lock(F->mu);
  if (u >= F->k_rows)
    return mg::set_error(MG_E_ARG, "query vertex %u, %u query embeddings", u, F->k_rows);
  for (uint64_t i = 0; i < nv; ++i)
    if (v[i] >= F->n_rows)
      return mg::set_error(MG_E_ARG, "data vertex %u, %u data embeddings", v[i], F->n_rows);
  if (nv == 0) return MG_OK;
  mg::DeviceGuard guard(F->device);
  cudaStream_t st = F->stream;
  uint32_t* dv = nullptr;
  uint8_t* dk = nullptr;
  MG_CK(cudaMallocAsync((void**)&dv, nv * 4, st));
  MG_CK(cudaMallocAsync((void**)&dk, nv, st));
  MG_CK(cudaMemcpyAsync(dv, v, nv * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(F->eu, F->query_emb.data() + uint64_t(u) * F->dim, F->dim * 4ull,
                        cudaMemcpyHostToDevice, st));
  const size_t smem = (mg::kMfBlock / 32) * (F->dim + mg::kMfMaxHidden) * sizeof(float);
  const uint64_t blocks = std::min<uint64_t>((nv + mg::kMfBlock / 32 - 1) / (mg::kMfBlock / 32),
                                             4096);
  mg::k_matrix_filter<<<unsigned(blocks), mg::kMfBlock, smem, st>>>(
      F->data_emb, F->eu, F->w1t, F->b1, F->w2, F->b2, F->dim, F->hidden, dv, nv, dk, nullptr);
  MG_CK(cudaGetLastError());
  MG_CK(cudaMemcpyAsync(keep, dk, nv, cudaMemcpyDeviceToHost, st));
  cudaFreeAsync(dv, st);
  cudaFreeAsync(dk, st);
  MG_CK(cudaStreamSynchronize(st));
  return MG_OK;
}

}  // extern "C"
