// Learned matching order: a small message-passing network over the query
// graph predicts log(1 + P(S)), the number of partial matches of a connected
// vertex set S of the query (a prefix of a matching order), from data-graph
// label statistics; a dynamic program over connected prefixes then picks the
// order with the least predicted work.  The order only reorders the search:
// counts stay exact.
//
// Network (per sample = query + vertex set S, nodes u in S, F = 8 features,
// H = 64 hidden units):
//   a1(u) = sum_{w in N_S(u)} [x_w ; e_uw]                       (F + 1)
//   h1(u) = relu(W1x x_u + W1m a1(u) + b1)                        (H)
//   a2(u) = sum_{w in N_S(u)} h1(w)                               (H)
//   h2(u) = relu(W2h h1(u) + W2m a2(u) + b2)                      (H)
//   z     = sum_{u in S} h2(u);  r = relu(Wr z + br);  y = wo . r + bo
// Training: FP32 forward/backward kernels, mean squared error on y, Adam
// (Kingma & Ba, 2015).  Inference: BF16 weights, FP32 accumulation.
//
// The reference's learned component is a lossy candidate filter
// (MatrixFilter, core/task/cpu_task/cpu_subiso.cu:237-277); only its weight
// container (embedding.bin + meta.yaml, core/data_structures/matrix.cu:12-35,
// tools/python/train.py:116-139) is reused here for the model file.
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "mg_device.cuh"

namespace mg {

constexpr int MF = 8;    // node features
constexpr int MH = 64;   // hidden units
constexpr int MQ = MAXK; // nodes per query
constexpr int OFF_W1x = 0;
constexpr int OFF_W1m = OFF_W1x + MH * MF;
constexpr int OFF_b1 = OFF_W1m + MH * (MF + 1);
constexpr int OFF_W2h = OFF_b1 + MH;
constexpr int OFF_W2m = OFF_W2h + MH * MH;
constexpr int OFF_b2 = OFF_W2m + MH * MH;
constexpr int OFF_Wr = OFF_b2 + MH;
constexpr int OFF_br = OFF_Wr + MH * MH;
constexpr int OFF_wo = OFF_br + MH;
constexpr int OFF_bo = OFF_wo + MH;
constexpr int NPARAM = OFF_bo + 1;

// Per-query inputs of the network (feature 5, the degree inside S, is filled
// in by the kernels).
struct QFeat {
  float x[MQ][MF];
  float e[MQ][MQ];
  uint32_t adj[MQ];  // undirected adjacency, no self-loops
  uint32_t k;
  uint32_t pad[3];
};

struct Sample {
  uint32_t q;     // query index
  uint32_t mask;  // vertex set S
  float target;   // log(1 + P(S))
  uint32_t pad;
};

struct OrderModel {
  int device = 0;
  unsigned sms = 1;  // multiprocessors of the device
  cudaStream_t stream = nullptr;
  float* params = nullptr;   // NPARAM
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  __nv_bfloat16* params_bf16 = nullptr;
  bool bf16_stale = true;
  uint64_t step = 0;
  ~OrderModel() {
    if (stream) {
      int prev = 0;
      cudaGetDevice(&prev);
      cudaSetDevice(device);
      cudaStreamSynchronize(stream);
      cudaFree(params);
      cudaFree(grad);
      cudaFree(adam_m);
      cudaFree(adam_v);
      cudaFree(params_bf16);
      cudaStreamDestroy(stream);
      cudaSetDevice(prev);
    }
  }
};

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ld(const float* p, int i) { return p[i]; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p, int i) {
  return __bfloat162float(p[i]);
}

struct FwdSmem {
  int nodes[MQ];
  int nn;
  float x[MQ][MF];
  float a1[MQ][MF + 1];
  float h1[MQ][MH];
  float a2[MQ][MH];
  float h2[MQ][MH];
  float z[MH];
  float r[MH];
  float red[MH];
};

// Forward pass of one sample by a block of MH threads; returns y in every
// thread.  Thread j owns hidden unit j.
template <class W>
__device__ float mpnn_forward(const W* P, const QFeat& Q, uint32_t mask, FwdSmem& s) {
  const int j = threadIdx.x;
  if (j == 0) {
    int nn = 0;
    for (int u = 0; u < int(Q.k); ++u)
      if ((mask >> u) & 1u) s.nodes[nn++] = u;
    s.nn = nn;
  }
  __syncthreads();
  const int nn = s.nn;
  for (int t = j; t < nn * MF; t += MH) {
    const int a = t / MF, f = t % MF;
    const int u = s.nodes[a];
    s.x[a][f] = f == 5 ? float(__popc(Q.adj[u] & mask)) * 0.125f : Q.x[u][f];
  }
  __syncthreads();
  for (int t = j; t < nn * (MF + 1); t += MH) {
    const int a = t / (MF + 1), f = t % (MF + 1);
    const int u = s.nodes[a];
    float acc = 0.f;
    for (int b = 0; b < nn; ++b) {
      const int w = s.nodes[b];
      if (!((Q.adj[u] >> w) & 1u)) continue;
      acc += f < MF ? s.x[b][f] : Q.e[u][w];
    }
    s.a1[a][f] = acc;
  }
  __syncthreads();
  for (int a = 0; a < nn; ++a) {
    float v = ld(P, OFF_b1 + j);
    for (int f = 0; f < MF; ++f) v += ld(P, OFF_W1x + j * MF + f) * s.x[a][f];
    for (int f = 0; f < MF + 1; ++f) v += ld(P, OFF_W1m + j * (MF + 1) + f) * s.a1[a][f];
    s.h1[a][j] = fmaxf(v, 0.f);
  }
  __syncthreads();
  for (int a = 0; a < nn; ++a) {
    const int u = s.nodes[a];
    float acc = 0.f;
    for (int b = 0; b < nn; ++b)
      if ((Q.adj[u] >> s.nodes[b]) & 1u) acc += s.h1[b][j];
    s.a2[a][j] = acc;
  }
  __syncthreads();
  float zj = 0.f;
  for (int a = 0; a < nn; ++a) {
    float v = ld(P, OFF_b2 + j);
    for (int l = 0; l < MH; ++l)
      v += ld(P, OFF_W2h + j * MH + l) * s.h1[a][l] + ld(P, OFF_W2m + j * MH + l) * s.a2[a][l];
    v = fmaxf(v, 0.f);
    s.h2[a][j] = v;
    zj += v;
  }
  s.z[j] = zj;
  __syncthreads();
  float rv = ld(P, OFF_br + j);
  for (int l = 0; l < MH; ++l) rv += ld(P, OFF_Wr + j * MH + l) * s.z[l];
  rv = fmaxf(rv, 0.f);
  s.r[j] = rv;
  s.red[j] = ld(P, OFF_wo + j) * rv;
  __syncthreads();
  for (int d = MH / 2; d > 0; d >>= 1) {
    if (j < d) s.red[j] += s.red[j + d];
    __syncthreads();
  }
  const float y = s.red[0] + ld(P, OFF_bo);
  __syncthreads();
  return y;
}

// Forward (+ backward) over samples [0, ns): every block walks a contiguous
// range, accumulates parameter gradients of scale*(y - t)^2 in shared memory
// (thread j owns row j of every matrix) and flushes them with atomics.
// out (optional) receives y per sample.
__global__ void __launch_bounds__(MH) k_mpnn_train(const float* __restrict__ P,
                                                   const QFeat* __restrict__ qf,
                                                   const Sample* __restrict__ smp, uint32_t ns,
                                                   float scale, int backward, float* grad,
                                                   float* loss, float* out) {
  extern __shared__ float g[];  // NPARAM gradient accumulators
  __shared__ FwdSmem s;
  __shared__ float dz[MH], dr[MH];
  __shared__ float dpre2[MQ][MH], gw[MQ][MH], dh1a[MQ][MH], dpre1[MQ][MH];
  const int j = threadIdx.x;
  if (backward)
    for (int t = j; t < NPARAM; t += MH) g[t] = 0.f;
  const uint32_t per = (ns + gridDim.x - 1) / gridDim.x;
  const uint32_t s0 = blockIdx.x * per, s1 = min(ns, s0 + per);
  float lsum = 0.f;
  for (uint32_t si = s0; si < s1; ++si) {
    const Sample sm = smp[si];
    const QFeat& Q = qf[sm.q];
    const float y = mpnn_forward(P, Q, sm.mask, s);
    if (out && j == 0) out[si] = y;
    const float diff = y - sm.target;
    lsum += diff * diff;
    if (!backward) continue;
    const int nn = s.nn;
    const float dy = 2.f * scale * diff;
    // readout
    if (j == 0) g[OFF_bo] += dy;
    g[OFF_wo + j] += dy * s.r[j];
    const float drj = s.r[j] > 0.f ? dy * P[OFF_wo + j] : 0.f;
    dr[j] = drj;
    g[OFF_br + j] += drj;
    for (int l = 0; l < MH; ++l) g[OFF_Wr + j * MH + l] += drj * s.z[l];
    __syncthreads();
    float dzj = 0.f;
    for (int i = 0; i < MH; ++i) dzj += P[OFF_Wr + i * MH + j] * dr[i];
    dz[j] = dzj;
    __syncthreads();
    // layer 2
    for (int a = 0; a < nn; ++a) {
      const float d = s.h2[a][j] > 0.f ? dz[j] : 0.f;
      dpre2[a][j] = d;
      g[OFF_b2 + j] += d;
      for (int l = 0; l < MH; ++l) {
        g[OFF_W2h + j * MH + l] += d * s.h1[a][l];
        g[OFF_W2m + j * MH + l] += d * s.a2[a][l];
      }
    }
    __syncthreads();
    for (int a = 0; a < nn; ++a) {
      float v = 0.f, w2 = 0.f;
      for (int i = 0; i < MH; ++i) {
        v += P[OFF_W2m + i * MH + j] * dpre2[a][i];
        w2 += P[OFF_W2h + i * MH + j] * dpre2[a][i];
      }
      gw[a][j] = v;
      dh1a[a][j] = w2;
    }
    __syncthreads();
    // layer 1
    for (int a = 0; a < nn; ++a) {
      const int u = s.nodes[a];
      float dh = dh1a[a][j];
      for (int b = 0; b < nn; ++b)
        if ((Q.adj[u] >> s.nodes[b]) & 1u) dh += gw[b][j];
      dpre1[a][j] = s.h1[a][j] > 0.f ? dh : 0.f;
    }
    __syncthreads();
    for (int a = 0; a < nn; ++a) {
      const float d = dpre1[a][j];
      g[OFF_b1 + j] += d;
      for (int f = 0; f < MF; ++f) g[OFF_W1x + j * MF + f] += d * s.x[a][f];
      for (int f = 0; f < MF + 1; ++f) g[OFF_W1m + j * (MF + 1) + f] += d * s.a1[a][f];
    }
    __syncthreads();
  }
  if (j == 0 && loss) atomicAdd(loss, lsum * scale);
  if (backward) {
    __syncthreads();
    for (int t = j; t < NPARAM; t += MH)
      if (g[t] != 0.f) atomicAdd(&grad[t], g[t]);
  }
}

// BF16 inference: one sample per block.
__global__ void __launch_bounds__(MH) k_mpnn_infer_bf16(const __nv_bfloat16* __restrict__ P,
                                                        const QFeat* __restrict__ qf,
                                                        const Sample* __restrict__ smp,
                                                        uint32_t ns, float* out) {
  __shared__ FwdSmem s;
  for (uint32_t si = blockIdx.x; si < ns; si += gridDim.x) {
    const Sample sm = smp[si];
    const float y = mpnn_forward(P, qf[sm.q], sm.mask, s);
    if (threadIdx.x == 0) out[si] = y;
  }
}

// Adam (Kingma & Ba, 2015): m, v moment estimates with bias correction.
__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_to_bf16(const float* p, __nv_bfloat16* o, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    o[i] = __float2bfloat16(p[i]);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

const size_t kTrainSmem = size_t(NPARAM) * 4;

int model_init(OrderModel* M, int device) {
  M->device = device;
  MG_CK(cudaSetDevice(device));
  int sms = 0;
  MG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  M->sms = unsigned(std::max(sms, 1));
  MG_CK(cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking));
  MG_CK(cudaMalloc((void**)&M->params, NPARAM * 4));
  MG_CK(cudaMalloc((void**)&M->grad, NPARAM * 4));
  MG_CK(cudaMalloc((void**)&M->adam_m, NPARAM * 4));
  MG_CK(cudaMalloc((void**)&M->adam_v, NPARAM * 4));
  MG_CK(cudaMalloc((void**)&M->params_bf16, NPARAM * 2));
  MG_CK(cudaMemset(M->adam_m, 0, NPARAM * 4));
  MG_CK(cudaMemset(M->adam_v, 0, NPARAM * 4));
  MG_CK(cudaFuncSetAttribute(k_mpnn_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kTrainSmem)));
  return MG_OK;
}

int set_params(OrderModel* M, const float* h) {
  MG_CK(cudaMemcpy(M->params, h, NPARAM * 4, cudaMemcpyHostToDevice));
  M->bf16_stale = true;
  return MG_OK;
}

// Features of a query (see QFeat); returns false when a label is absent from
// the data graph or the statistics are missing.
bool build_qfeat(const QueryGraph& Q, const GraphStats& gs, QFeat* f) {
  std::memset(f, 0, sizeof(*f));
  if (Q.k > MQ || gs.label_deg_mean.empty()) return false;
  f->k = Q.k;
  const double L = std::max<double>(1.0, gs.L);
  int lab[MQ];
  for (uint32_t u = 0; u < Q.k; ++u) {
    lab[u] = gs.compact_label(Q.label_raw[u]);
    if (lab[u] < 0) return false;
  }
  for (uint32_t u = 0; u < Q.k; ++u) {
    const uint32_t nb = (Q.out_mask[u] | Q.in_mask[u]) & ~(1u << u);
    f->adj[u] = nb;
    const int l = lab[u];
    f->x[u][0] = float(std::log1p(double(gs.label_count[l])) / 16.0);
    f->x[u][1] = float(std::log1p(gs.label_deg_mean[l]) / 8.0);
    f->x[u][2] = float(std::log1p(gs.label_deg_max[l]) / 16.0);
    f->x[u][3] = float(std::log1p(gs.label_deg_p99[l]) / 12.0);
    f->x[u][4] = float(double(gs.label_nlb_density[l]) / L);
    f->x[u][5] = 0.f;  // degree inside the sample's set (kernel)
    f->x[u][6] = float(__builtin_popcount(nb)) * 0.125f;
    f->x[u][7] = float(std::log1p(double(gs.n)) / 20.0);
    for (uint32_t w = 0; w < Q.k; ++w)
      if ((nb >> w) & 1u)
        f->e[u][w] = float(std::log1p(double(gs.label_pair_edges[uint64_t(l) * gs.L + lab[w]])) /
                           24.0);
  }
  return true;
}

bool connected(uint32_t mask, const QFeat& f) {
  if (!mask) return false;
  uint32_t seen = mask & (~mask + 1), front = seen;
  while (front) {
    uint32_t nxt = 0;
    for (uint32_t m = front; m; m &= m - 1) nxt |= f.adj[__builtin_ctz(m)];
    nxt &= mask & ~seen;
    seen |= nxt;
    front = nxt;
  }
  return seen == mask;
}

int refresh_bf16(OrderModel* M) {
  if (!M->bf16_stale) return MG_OK;
  k_to_bf16<<<64, 256, 0, M->stream>>>(M->params, M->params_bf16, NPARAM);
  MG_CK(cudaGetLastError());
  M->bf16_stale = false;
  return MG_OK;
}

// Runs BF16 inference for the given samples on the model's device.
int infer(OrderModel* M, const std::vector<QFeat>& qf, const std::vector<Sample>& smp,
          std::vector<float>& out) {
  out.assign(smp.size(), 0.f);
  if (smp.empty()) return MG_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  MG_CK(cudaSetDevice(M->device));
  int rc = refresh_bf16(M);
  if (rc) return rc;
  QFeat* dq;
  Sample* ds;
  float* dout;
  cudaStream_t st = M->stream;
  MG_CK(cudaMallocAsync((void**)&dq, qf.size() * sizeof(QFeat), st));
  MG_CK(cudaMallocAsync((void**)&ds, smp.size() * sizeof(Sample), st));
  MG_CK(cudaMallocAsync((void**)&dout, smp.size() * 4, st));
  MG_CK(cudaMemcpyAsync(dq, qf.data(), qf.size() * sizeof(QFeat), cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(ds, smp.data(), smp.size() * sizeof(Sample), cudaMemcpyHostToDevice, st));
  const unsigned blocks = unsigned(std::min<size_t>(smp.size(), size_t(M->sms) * 32));
  k_mpnn_infer_bf16<<<blocks, MH, 0, st>>>(M->params_bf16, dq, ds, uint32_t(smp.size()), dout);
  MG_CK(cudaMemcpyAsync(out.data(), dout, smp.size() * 4, cudaMemcpyDeviceToHost, st));
  cudaFreeAsync(dq, st);
  cudaFreeAsync(ds, st);
  cudaFreeAsync(dout, st);
  MG_CK(cudaStreamSynchronize(st));
  MG_CK(cudaGetLastError());
  cudaSetDevice(prev);
  return MG_OK;
}

// Whether the last two vertices (a then b) of an order over `all` form the
// closed-form tail the enumerator counts without expanding, and whether the
// last vertex has a single backward neighbour (symmetric adjacency).
void tail_kind(const QueryGraph& Q, const QFeat& f, uint32_t all, uint32_t a, uint32_t b,
               bool* last_o1, bool* tail2) {
  const uint32_t self_b = (Q.out_mask[b] >> b) & 1u, self_a = (Q.out_mask[a] >> a) & 1u;
  const uint32_t bb = f.adj[b] & all & ~(1u << b);
  *last_o1 = __builtin_popcount(bb) == 1 && !self_b;
  *tail2 = false;
  if (!*last_o1 || self_a) return;
  if (bb != (1u << a)) {
    // two leaves of one anchor p (a's only neighbour in `all` is b's): the
    // enumerator counts them in closed form too
    *tail2 = (f.adj[a] & all & ~(1u << a)) == bb;
    return;
  }
  const uint32_t rest = all & ~(1u << a) & ~(1u << b);
  const uint32_t ab = f.adj[a] & rest;
  if (__builtin_popcount(ab) != 1) return;
  const uint32_t p = __builtin_ctz(ab);
  for (uint32_t m = rest; m; m &= m - 1) {
    const uint32_t j = __builtin_ctz(m);
    if (Q.label_raw[j] == Q.label_raw[b] && j != p) return;
  }
  *tail2 = true;
}

// Order with the least predicted work: rows of every prefix length are
// charged their predicted count, except the last prefixes that the
// enumerator closes without expanding.
void choose_order(const QueryGraph& Q, const QFeat& f, const std::vector<float>& pred_of_mask,
                  uint32_t* order) {
  const uint32_t k = Q.k, full = (1u << k) - 1;
  std::vector<double> best(size_t(1) << k, INFINITY);
  std::vector<int8_t> arg(size_t(1) << k, -1);
  auto P = [&](uint32_t m) { return std::expm1(double(pred_of_mask[m])); };
  for (uint32_t u = 0; u < k; ++u) best[1u << u] = P(1u << u);
  for (uint32_t m = 1; m <= full; ++m) {
    if (__builtin_popcount(m) < 2 || !std::isfinite(pred_of_mask[m]) || !connected(m, f)) continue;
    const double pm = P(m);
    for (uint32_t mm = m; mm; mm &= mm - 1) {
      const uint32_t v = __builtin_ctz(mm), rest = m & ~(1u << v);
      if (!(f.adj[v] & rest) || !std::isfinite(best[rest])) continue;
      const double c = best[rest] + pm;
      if (c < best[m]) {
        best[m] = c;
        arg[m] = int8_t(v);
      }
    }
  }
  // Last two vertices: drop the charges the enumerator does not pay.
  double top = INFINITY;
  uint32_t ta = 0, tb = 0;
  if (k >= 3) {
    for (uint32_t b = 0; b < k; ++b) {
      const uint32_t mb = full & ~(1u << b);
      if (!(f.adj[b] & mb)) continue;
      for (uint32_t a = 0; a < k; ++a) {
        if (a == b) continue;
        const uint32_t ma = mb & ~(1u << a);
        if (!(f.adj[a] & ma) || !std::isfinite(best[ma])) continue;
        bool o1, t2;
        tail_kind(Q, f, full, a, b, &o1, &t2);
        const double c = best[ma] + (t2 ? 0.0 : P(mb)) + (o1 ? 0.0 : P(full));
        if (c < top) {
          top = c;
          ta = a;
          tb = b;
        }
      }
    }
  }
  uint32_t m = full;
  int n = int(k);
  if (std::isfinite(top)) {
    order[--n] = tb;
    order[--n] = ta;
    m = full & ~(1u << ta) & ~(1u << tb);
  }
  while (n > 0 && m) {
    if (__builtin_popcount(m) == 1) {
      order[--n] = __builtin_ctz(m);
      break;
    }
    const int v = arg[m];
    if (v < 0) break;
    order[--n] = uint32_t(v);
    m &= ~(1u << v);
  }
  if (n != 0) order_reference(Q, order);  // no connected order found
}

}  // namespace

// Orders of several queries with one inference launch.  Queries the model
// cannot serve (fewer than 3 or more than 12 vertices, labels absent from the
// graph, non-finite predictions) get the reference order.
int order_learned_batch(void* model, const std::vector<const QueryGraph*>& qs,
                        const GraphStats& gs, std::vector<std::array<uint32_t, MAXK>>& orders) {
  auto* M = static_cast<OrderModel*>(model);
  orders.resize(qs.size());
  std::vector<QFeat> feats;
  std::vector<Sample> smp;
  std::vector<int> fidx(qs.size(), -1);
  std::vector<size_t> first(qs.size(), 0);
  for (size_t i = 0; i < qs.size(); ++i) {
    const QueryGraph& Q = *qs[i];
    QFeat f;
    if (Q.k < 3 || Q.k > 12 || !build_qfeat(Q, gs, &f)) {
      order_reference(Q, orders[i].data());
      continue;
    }
    fidx[i] = int(feats.size());
    feats.push_back(f);
    first[i] = smp.size();
    for (uint32_t m = 1; m < (1u << Q.k); ++m)
      smp.push_back(Sample{uint32_t(fidx[i]), m, 0.f, 0});
  }
  std::vector<float> pred;
  int rc = infer(M, feats, smp, pred);
  if (rc) return rc;
  for (size_t i = 0; i < qs.size(); ++i) {
    if (fidx[i] < 0) continue;
    const QueryGraph& Q = *qs[i];
    std::vector<float> pm(size_t(1) << Q.k, NAN);
    bool finite = true;
    for (uint32_t m = 1; m < (1u << Q.k); ++m) {
      pm[m] = pred[first[i] + m - 1];
      finite &= std::isfinite(pm[m]);
    }
    if (!finite) {
      order_reference(Q, orders[i].data());
      continue;
    }
    choose_order(Q, feats[fidx[i]], pm, orders[i].data());
    if (!order_is_permutation(orders[i].data(), Q.k)) order_reference(Q, orders[i].data());
  }
  return MG_OK;
}

int order_learned(void* model, const QueryGraph& q, const GraphStats& gs, uint32_t* order) {
  std::vector<const QueryGraph*> qs{&q};
  std::vector<std::array<uint32_t, MAXK>> out;
  int rc = order_learned_batch(model, qs, gs, out);
  if (rc) return rc;
  std::memcpy(order, out[0].data(), q.k * 4);
  return MG_OK;
}

// ---- training / gradients ----------------------------------------------------
static int gather(DevGraph* dg, const mg_csr_view* const* qs, uint32_t nq,
                  std::vector<QFeat>& feats) {
  int rc = ensure_full_stats(dg);
  if (rc) return rc;
  feats.resize(nq);
  for (uint32_t i = 0; i < nq; ++i) {
    QueryGraph Q;
    if ((rc = normalise_query(qs[i], &Q))) return rc;
    if (!build_qfeat(Q, dg->stats, &feats[i]))
      return set_error(MG_E_ARG, "query %u: a label is absent from the data graph", i);
  }
  return MG_OK;
}

static int train_pass(OrderModel* M, const QFeat* dq, const Sample* ds, uint32_t ns, float scale,
                      bool backward, float* dloss, float* dout) {
  const unsigned blocks = std::max(1u, std::min<unsigned>(ns, M->sms * 2));
  if (backward) MG_CK(cudaMemsetAsync(M->grad, 0, NPARAM * 4, M->stream));
  k_mpnn_train<<<blocks, MH, kTrainSmem, M->stream>>>(M->params, dq, ds, ns, scale,
                                                       backward ? 1 : 0, M->grad, dloss, dout);
  MG_CK(cudaGetLastError());
  return MG_OK;
}

static int samples_of(uint32_t nq, const uint32_t* s_query, const uint32_t* s_mask,
                      const float* s_target, uint32_t ns, std::vector<Sample>& smp) {
  smp.resize(ns);
  for (uint32_t i = 0; i < ns; ++i) {
    if (s_query[i] >= nq) return set_error(MG_E_ARG, "sample %u: query index %u", i, s_query[i]);
    smp[i] = Sample{s_query[i], s_mask[i], s_target ? s_target[i] : 0.f, 0};
  }
  return MG_OK;
}

}  // namespace mg

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
using mg::OrderModel;

extern "C" {

int mg_order_model_create(int device, uint64_t seed, void** model) {
  mg::clear_error();
  if (!model) return mg::set_error(MG_E_ARG, "null argument");
  auto* M = new OrderModel();
  int rc = mg::model_init(M, device);
  if (rc) {
    delete M;
    return rc;
  }
  // He-style initialisation from a seeded normal generator.
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::vector<float> h(mg::NPARAM, 0.f);
  auto fill = [&](int off, int rows, int cols) {
    const float sd = std::sqrt(2.f / float(cols));
    for (int i = 0; i < rows * cols; ++i) h[off + i] = sd * nd(rng);
  };
  fill(mg::OFF_W1x, mg::MH, mg::MF);
  fill(mg::OFF_W1m, mg::MH, mg::MF + 1);
  fill(mg::OFF_W2h, mg::MH, mg::MH);
  fill(mg::OFF_W2m, mg::MH, mg::MH);
  fill(mg::OFF_Wr, mg::MH, mg::MH);
  fill(mg::OFF_wo, 1, mg::MH);
  for (int i = 0; i < mg::MH; ++i) h[mg::OFF_wo + i] *= 0.1f;
  if ((rc = mg::set_params(M, h.data()))) {
    delete M;
    return rc;
  }
  *model = M;
  return MG_OK;
}

void mg_order_model_free(void* model) { delete static_cast<OrderModel*>(model); }

int mg_order_model_num_params(void) { return mg::NPARAM; }

int mg_order_model_get_params(void* model, float* out) {
  mg::clear_error();
  if (!model || !out) return mg::set_error(MG_E_ARG, "null argument");
  auto* M = static_cast<OrderModel*>(model);
  MG_CK(cudaSetDevice(M->device));
  MG_CK(cudaStreamSynchronize(M->stream));
  MG_CK(cudaMemcpy(out, M->params, mg::NPARAM * 4, cudaMemcpyDeviceToHost));
  return MG_OK;
}

int mg_order_model_set_params(void* model, const float* p) {
  mg::clear_error();
  if (!model || !p) return mg::set_error(MG_E_ARG, "null argument");
  auto* M = static_cast<OrderModel*>(model);
  MG_CK(cudaSetDevice(M->device));
  return mg::set_params(M, p);
}

// Weight container of the reference's matrix files: <dir>/meta.yaml with x, y
// (and dtype / order keys) and <dir>/embedding.bin, row-major float32.
int mg_order_model_save(void* model, const char* dir) {
  mg::clear_error();
  if (!model || !dir) return mg::set_error(MG_E_ARG, "null argument");
  std::vector<float> h(mg::NPARAM);
  int rc = mg_order_model_get_params(model, h.data());
  if (rc) return rc;
  std::string d(dir);
  std::ofstream bf(d + "embedding.bin", std::ios::binary | std::ios::trunc);
  if (!bf) return mg::set_error(MG_E_IO, "cannot write %sembedding.bin", dir);
  bf.write(reinterpret_cast<const char*>(h.data()), std::streamsize(h.size() * 4));
  std::ofstream mf(d + "meta.yaml", std::ios::trunc);
  if (!mf) return mg::set_error(MG_E_IO, "cannot write %smeta.yaml", dir);
  mf << "dtype: float32\nendian: little\norder: row_major\nx: 1\ny: " << mg::NPARAM
     << "\nmodel: mg-order-mpnn\nhidden: " << mg::MH << "\nfeatures: " << mg::MF << "\n";
  return (bf && mf) ? MG_OK : mg::set_error(MG_E_IO, "write failed under %s", dir);
}

int mg_order_model_load(const char* dir, int device, void** model) {
  mg::clear_error();
  if (!dir || !model) return mg::set_error(MG_E_ARG, "null argument");
  std::string d(dir);
  std::ifstream mf(d + "meta.yaml");
  if (!mf) return mg::set_error(MG_E_IO, "cannot open %smeta.yaml", dir);
  uint64_t x = 0, y = 0;
  std::string line;
  while (std::getline(mf, line)) {
    std::stringstream ss(line);
    std::string key;
    if (!std::getline(ss, key, ':')) continue;
    uint64_t v = 0;
    if (key == "x" && (ss >> v)) x = v;
    if (key == "y" && (ss >> v)) y = v;
  }
  if (x * y != uint64_t(mg::NPARAM))
    return mg::set_error(MG_E_FORMAT, "%smeta.yaml: %llu x %llu parameters, %d expected", dir,
                         (unsigned long long)x, (unsigned long long)y, mg::NPARAM);
  std::vector<float> h(mg::NPARAM);
  std::ifstream bf(d + "embedding.bin", std::ios::binary);
  if (!bf || !bf.read(reinterpret_cast<char*>(h.data()), std::streamsize(h.size() * 4)))
    return mg::set_error(MG_E_IO, "cannot read %sembedding.bin", dir);
  void* m = nullptr;
  int rc = mg_order_model_create(device, 0, &m);
  if (rc) return rc;
  if ((rc = mg_order_model_set_params(m, h.data()))) {
    mg_order_model_free(m);
    return rc;
  }
  *model = m;
  return MG_OK;
}

// Samples: (query index, vertex-set mask, target log(1 + P)).  Mean squared
// error over the samples; grad_out (NPARAM) receives its gradient, pred_out
// (ns, optional) the FP32 predictions.
int mg_order_model_grad(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                        const uint32_t* s_query, const uint32_t* s_mask, const float* s_target,
                        uint32_t ns, float* grad_out, float* loss_out, float* pred_out) {
  mg::clear_error();
  if (!model || !dgraph || !qs || !s_query || !s_mask || !s_target || ns == 0)
    return mg::set_error(MG_E_ARG, "null argument");
  auto* M = static_cast<OrderModel*>(model);
  auto* dg = static_cast<mg::DevGraph*>(dgraph);
  std::lock_guard<std::mutex> lock(dg->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  MG_CK(cudaSetDevice(M->device));
  std::vector<mg::QFeat> feats;
  int rc = mg::gather(dg, qs, nq, feats);
  if (rc) return rc;
  std::vector<mg::Sample> smp;
  if ((rc = mg::samples_of(nq, s_query, s_mask, s_target, ns, smp))) return rc;
  cudaStream_t st = M->stream;
  mg::QFeat* dq;
  mg::Sample* ds;
  float *dl, *dout = nullptr;
  MG_CK(cudaMallocAsync((void**)&dq, feats.size() * sizeof(mg::QFeat), st));
  MG_CK(cudaMallocAsync((void**)&ds, smp.size() * sizeof(mg::Sample), st));
  MG_CK(cudaMallocAsync((void**)&dl, 4, st));
  if (pred_out) MG_CK(cudaMallocAsync((void**)&dout, ns * 4ull, st));
  MG_CK(cudaMemcpyAsync(dq, feats.data(), feats.size() * sizeof(mg::QFeat),
                        cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(ds, smp.data(), smp.size() * sizeof(mg::Sample), cudaMemcpyHostToDevice,
                        st));
  MG_CK(cudaMemsetAsync(dl, 0, 4, st));
  rc = mg::train_pass(M, dq, ds, ns, 1.f / float(ns), grad_out != nullptr, dl, dout);
  if (rc == MG_OK) {
    if (grad_out)
      MG_CK(cudaMemcpyAsync(grad_out, M->grad, mg::NPARAM * 4, cudaMemcpyDeviceToHost, st));
    if (loss_out) MG_CK(cudaMemcpyAsync(loss_out, dl, 4, cudaMemcpyDeviceToHost, st));
    if (pred_out) MG_CK(cudaMemcpyAsync(pred_out, dout, ns * 4ull, cudaMemcpyDeviceToHost, st));
  }
  cudaFreeAsync(dq, st);
  cudaFreeAsync(ds, st);
  cudaFreeAsync(dl, st);
  if (dout) cudaFreeAsync(dout, st);
  MG_CK(cudaStreamSynchronize(st));
  cudaSetDevice(prev);
  return rc;
}

// Adam over shuffled mini-batches for `epochs` passes; *final_loss receives
// the mean squared error of the last epoch (FP32 forward).
int mg_order_model_train(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                         const uint32_t* s_query, const uint32_t* s_mask, const float* s_target,
                         uint32_t ns, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                         float* final_loss) {
  mg::clear_error();
  if (!model || !dgraph || !qs || !s_query || !s_mask || !s_target || ns == 0 || batch == 0)
    return mg::set_error(MG_E_ARG, "null argument");
  auto* M = static_cast<OrderModel*>(model);
  auto* dg = static_cast<mg::DevGraph*>(dgraph);
  std::lock_guard<std::mutex> lock(dg->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  MG_CK(cudaSetDevice(M->device));
  std::vector<mg::QFeat> feats;
  int rc = mg::gather(dg, qs, nq, feats);
  if (rc) return rc;
  std::vector<mg::Sample> smp;
  if ((rc = mg::samples_of(nq, s_query, s_mask, s_target, ns, smp))) return rc;
  cudaStream_t st = M->stream;
  mg::QFeat* dq;
  mg::Sample* ds;
  float* dl;
  MG_CK(cudaMalloc((void**)&dq, feats.size() * sizeof(mg::QFeat)));
  MG_CK(cudaMalloc((void**)&ds, smp.size() * sizeof(mg::Sample)));
  MG_CK(cudaMalloc((void**)&dl, 4));
  MG_CK(cudaMemcpy(dq, feats.data(), feats.size() * sizeof(mg::QFeat), cudaMemcpyHostToDevice));
  std::mt19937_64 rng(seed);
  float last = 0.f;
  const float b1 = 0.9f, b2 = 0.999f;
  for (uint32_t ep = 0; ep < epochs && rc == MG_OK; ++ep) {
    std::shuffle(smp.begin(), smp.end(), rng);
    MG_CK(cudaMemcpyAsync(ds, smp.data(), smp.size() * sizeof(mg::Sample),
                          cudaMemcpyHostToDevice, st));
    MG_CK(cudaMemsetAsync(dl, 0, 4, st));
    uint32_t nbatches = 0;
    for (uint32_t b0 = 0; b0 < ns && rc == MG_OK; b0 += batch) {
      const uint32_t nb = std::min(batch, ns - b0);
      rc = mg::train_pass(M, dq, ds + b0, nb, 1.f / float(nb), true, dl, nullptr);
      ++M->step;
      ++nbatches;
      const float c1 = 1.f - std::pow(b1, float(M->step));
      const float c2 = 1.f - std::pow(b2, float(M->step));
      mg::k_adam<<<64, 256, 0, st>>>(M->params, M->grad, M->adam_m, M->adam_v, mg::NPARAM, lr,
                                     b1, b2, 1e-8f, c1, c2);
    }
    float l = 0.f;
    MG_CK(cudaMemcpyAsync(&l, dl, 4, cudaMemcpyDeviceToHost, st));
    MG_CK(cudaStreamSynchronize(st));
    last = nbatches ? l / float(nbatches) : 0.f;  // mean of the batch means
  }
  M->bf16_stale = true;
  cudaFree(dq);
  cudaFree(ds);
  cudaFree(dl);
  if (final_loss) *final_loss = last;
  cudaSetDevice(prev);
  return rc;
}

// BF16 predictions y = log(1 + P(S)) for samples (query index, mask).
int mg_order_model_predict(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                           const uint32_t* s_query, const uint32_t* s_mask, uint32_t ns,
                           float* out) {
  mg::clear_error();
  if (!model || !dgraph || !qs || !s_query || !s_mask || !out)
    return mg::set_error(MG_E_ARG, "null argument");
  auto* M = static_cast<OrderModel*>(model);
  auto* dg = static_cast<mg::DevGraph*>(dgraph);
  std::lock_guard<std::mutex> lock(dg->mu);
  std::vector<mg::QFeat> feats;
  int rc = mg::gather(dg, qs, nq, feats);
  if (rc) return rc;
  std::vector<mg::Sample> smp;
  if ((rc = mg::samples_of(nq, s_query, s_mask, nullptr, ns, smp))) return rc;
  std::vector<float> pred;
  if ((rc = mg::infer(M, feats, smp, pred))) return rc;
  std::memcpy(out, pred.data(), ns * 4ull);
  return MG_OK;
}

// The network inputs of one query (for an independent re-implementation):
// x[16][8] (feature 5 left 0), e[16][16], adj[16].
int mg_order_model_features(void* dgraph, const mg_csr_view* q, float* x, float* e,
                            uint32_t* adj) {
  mg::clear_error();
  if (!dgraph || !q || !x || !e || !adj) return mg::set_error(MG_E_ARG, "null argument");
  auto* dg = static_cast<mg::DevGraph*>(dgraph);
  std::lock_guard<std::mutex> lock(dg->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  MG_CK(cudaSetDevice(dg->device));
  std::vector<mg::QFeat> f;
  const mg_csr_view* qs[1] = {q};
  int rc = mg::gather(dg, qs, 1, f);
  cudaSetDevice(prev);
  if (rc) return rc;
  std::memcpy(x, f[0].x, sizeof(f[0].x));
  std::memcpy(e, f[0].e, sizeof(f[0].e));
  std::memcpy(adj, f[0].adj, sizeof(f[0].adj));
  return MG_OK;
}

}  // extern "C"
