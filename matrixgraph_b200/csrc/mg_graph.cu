// Data-graph upload and the derived device indices.
//
// The reference keeps the raw CSR byte buffer in managed memory and
// re-derives labels and degrees inside every filter call
// (core/task/gpu_task/kernel/kernel_woj_subsio.cu:545-561, :753-815).  Here
// the graph is uploaded once into plain device memory and turned into
// label-sliced adjacency (each list reordered by (label, id)), neighbour-label
// bit words (the sound subset form of NeighborLabelCounterFilter,
// kernel_woj_subsio.cu:385-446) and label buckets (the level-0 candidate
// ranges).
#include <algorithm>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <thread>

#include <cub/cub.cuh>

#include "mg_device.cuh"

namespace mg {

int dev_alloc(DevGraph* dg, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_error(MG_E_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  dg->allocs.push_back(*p);
  dg->info.device_bytes += bytes;
  return MG_OK;
}

void free_workspace(Workspace* ws);
void free_lanes(LaneSet* ls);

DevGraph::~DevGraph() {
  if (stream) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    free_workspace(ws);
    free_lanes(lanes);
    for (void* p : allocs) cudaFree(p);
    cudaStreamDestroy(stream);
    cudaSetDevice(prev);
  }
}

namespace {

// Global -> local id through a dense table over [0, max_vid].
__global__ void k_build_g2l(const uint32_t* globalid, uint32_t n, uint32_t* g2l,
                            uint32_t max_vid, uint32_t* err) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t gid = globalid[i];
    if (gid > max_vid) {
      atomicOr(err, ERR_RANGE);
      continue;
    }
    g2l[gid] = uint32_t(i);
  }
}

__global__ void k_map_edges(uint32_t* adj, uint64_t m, const uint32_t* g2l,
                            uint32_t max_vid, uint32_t* err) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < m;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t gid = adj[i];
    uint32_t l = gid <= max_vid ? g2l[gid] : FULL;
    if (l == FULL) atomicOr(err, ERR_RANGE);
    adj[i] = l == FULL ? 0 : l;
  }
}

// Warp per vertex: flags unsorted or repeated entries and ids >= n.
__global__ void k_check_lists(const uint32_t* off, const uint32_t* adj, uint32_t n,
                              uint32_t* flags) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  uint32_t bad = 0;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t s = off[v], e = off[v + 1];
    for (uint32_t j = s + lane; j < e; j += 32) {
      uint32_t a = adj[j];
      if (a >= n) bad |= 2;
      if (j + 1 < e && a >= adj[j + 1]) bad |= 1;
    }
  }
  bad = __reduce_or_sync(FULL, bad);
  if (lane == 0 && bad) atomicOr(flags, bad);
}

// Distinct entries per (sorted) list.
__global__ void k_count_unique(const uint32_t* off, const uint32_t* adj, uint32_t n,
                               uint32_t* newdeg) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t s = off[v], e = off[v + 1];
    uint32_t c = 0;
    for (uint32_t j = s + lane; j < e; j += 32) c += (j == s || adj[j] != adj[j - 1]);
    c = __reduce_add_sync(FULL, c);
    if (lane == 0) newdeg[v] = c;
  }
}

__global__ void k_compact_unique(const uint32_t* off, const uint32_t* adj, uint32_t n,
                                 const uint32_t* newoff, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t s = off[v], e = off[v + 1];
    uint32_t base = newoff[v];
    for (uint32_t j0 = s; j0 < e; j0 += 32) {
      uint32_t j = j0 + lane;
      bool keep = j < e && (j == s || adj[j] != adj[j - 1]);
      uint32_t bal = __ballot_sync(FULL, keep);
      if (keep) out[base + __popc(bal & ((1u << lane) - 1))] = adj[j];
      base += __popc(bal);
    }
  }
}

// Warp per vertex: label histogram -> slice offsets, neighbour-label bits,
// then a stable scatter of the (id-sorted) list into (label, id) order.
// Shared memory: one L-word histogram per warp.
__global__ void k_partition_labels(const uint32_t* off, const uint32_t* adj, uint32_t n,
                                   const uint32_t* label, uint32_t L, uint32_t W,
                                   uint32_t* loff, uint32_t* adjL, uint32_t* nlb,
                                   uint32_t* deg, uint32_t* selfbits) {
  extern __shared__ uint32_t sh[];
  const uint32_t lane = threadIdx.x & 31;
  uint32_t* hist = sh + (threadIdx.x >> 5) * L;
  const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  const uint32_t per = (L + 31) / 32;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t s = off[v], e = off[v + 1];
    for (uint32_t b = lane; b < L; b += 32) hist[b] = 0;
    __syncwarp();
    bool self = false;
    for (uint32_t j = s + lane; j < e; j += 32) {
      uint32_t a = adj[j];
      self |= (a == v);
      atomicAdd(&hist[label[a]], 1u);
    }
    __syncwarp();
    for (uint32_t w = 0; w < W; ++w) {
      uint32_t b = w * 32 + lane;
      uint32_t bits = __ballot_sync(FULL, b < L && hist[b] > 0);
      if (lane == 0) nlb[v * uint64_t(W) + w] = bits;
    }
    // Lane-owned runs of `per` bins, warp exclusive scan of the run sums.
    uint32_t run = 0;
    for (uint32_t b = lane * per; b < min(L, lane * per + per); ++b) run += hist[b];
    uint32_t incl = run;
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(FULL, incl, d);
      if (lane >= d) incl += t;
    }
    uint32_t acc = s + incl - run;
    for (uint32_t b = lane * per; b < min(L, lane * per + per); ++b) {
      uint32_t c = hist[b];
      loff[v * uint64_t(L) + b] = acc;
      hist[b] = acc;  // becomes the scatter cursor
      acc += c;
    }
    __syncwarp();
    for (uint32_t j0 = s; j0 < e; j0 += 32) {
      uint32_t j = j0 + lane;
      bool valid = j < e;
      uint32_t a = valid ? adj[j] : 0;
      uint32_t lab = valid ? label[a] : FULL;
      uint32_t peers = __match_any_sync(FULL, lab);
      uint32_t rank = __popc(peers & ((1u << lane) - 1));
      uint32_t leader = __ffs(peers) - 1;
      uint32_t basepos = valid ? hist[lab] : 0;
      __syncwarp();
      if (valid) adjL[basepos + rank] = a;
      if (valid && lane == leader) hist[lab] = basepos + __popc(peers);
      __syncwarp();
    }
    self = __any_sync(FULL, self);
    if (lane == 0) {
      deg[v] = e - s;
      if (self) atomicOr(&selfbits[v >> 5], 1u << (v & 31));
    }
    __syncwarp();
  }
}

__global__ void k_set_u32(uint32_t* p, uint64_t i, uint32_t v) { p[i] = v; }

// Per-label degree sums / maxima / log2 histograms and label-pair edge counts
// (features of the order model).
__global__ void k_label_stats(const uint32_t* loff, const uint32_t* label, uint32_t n,
                              uint32_t L, unsigned long long* deg_sum,
                              unsigned int* deg_max, unsigned long long* deg_hist,
                              unsigned long long* pair) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < n;
       v += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t lv = label[v];
    uint32_t s = loff[v * uint64_t(L)], e = loff[(v + 1) * uint64_t(L)];
    uint32_t d = e - s;
    atomicAdd(&deg_sum[lv], (unsigned long long)d);
    atomicMax(&deg_max[lv], d);
    uint32_t bin = d == 0 ? 0 : 32 - __clz(d);
    atomicAdd(&deg_hist[lv * 33 + bin], 1ull);
    for (uint32_t l = 0; l < L; ++l) {
      uint32_t a = loff[v * uint64_t(L) + l], b = loff[v * uint64_t(L) + l + 1];
      if (b > a) atomicAdd(&pair[lv * uint64_t(L) + l], (unsigned long long)(b - a));
    }
  }
}

unsigned host_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t == 0 ? 1 : std::min(t, 32u);
}

bool arrays_equal(const uint32_t* a, const uint32_t* b, uint64_t words) {
  if (a == b) return true;
  unsigned T = host_threads();
  if (words < (1u << 20)) T = 1;
  std::vector<std::thread> ts;
  std::vector<char> eq(T, 1);
  uint64_t chunk = (words + T - 1) / T;
  for (unsigned t = 0; t < T; ++t)
    ts.emplace_back([&, t]() {
      uint64_t lo = t * chunk, hi = std::min(words, lo + chunk);
      if (lo < hi) eq[t] = std::memcmp(a + lo, b + lo, (hi - lo) * 4) == 0;
    });
  for (auto& th : ts) th.join();
  for (char c : eq)
    if (!c) return false;
  return true;
}

inline unsigned grid_for(uint64_t items, unsigned block, unsigned cap) {
  uint64_t g = (items + block - 1) / block;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(g, cap)));
}

}  // namespace

// Hub bitmaps: block h sets the bits of hub h's whole d-adjacency (the
// label-ordered list of vertex y spans [loff[y*L], loff[(y+1)*L])).
__global__ void __launch_bounds__(256) k_hub_bits(const uint32_t* __restrict__ adj,
                                                  const uint32_t* __restrict__ loff, uint32_t L,
                                                  const uint32_t* __restrict__ hub_vid,
                                                  uint32_t words, uint32_t* bits) {
  const uint32_t y = hub_vid[blockIdx.x];
  const uint32_t s = loff[uint64_t(y) * L], e = loff[uint64_t(y + 1) * L];
  uint32_t* row = bits + uint64_t(blockIdx.x) * words;
  for (uint32_t j = s + threadIdx.x; j < e; j += blockDim.x) {
    const uint32_t x = adj[j];
    atomicOr(row + (x >> 5), 1u << (x & 31));
  }
}

// Selects the hubs of direction d (decreasing degree within the byte budget,
// ties at the cut all in or all out) and builds their bitmaps.
static int build_hubs(DevGraph* dg, int d, const std::vector<uint32_t>& deg, uint64_t budget,
                      uint32_t min_degree) {
  const uint32_t n = dg->g.n;
  const uint32_t words = ((n + 31) / 32 + 3) & ~3u;  // rows start on 16-byte boundaries
  const uint64_t row_bytes = uint64_t(words) * 4;
  uint64_t cap = std::min<uint64_t>(budget / row_bytes, NO_HUB);
  if (cap == 0) return MG_OK;
  std::vector<uint32_t> cand;
  for (uint32_t v = 0; v < n; ++v)
    if (deg[v] >= min_degree) cand.push_back(v);
  if (cand.empty()) return MG_OK;
  uint32_t cut = min_degree;
  if (cand.size() > cap) {
    std::vector<uint32_t> dv(cand.size());
    for (size_t i = 0; i < cand.size(); ++i) dv[i] = deg[cand[i]];
    std::nth_element(dv.begin(), dv.begin() + (cap - 1), dv.end(), std::greater<uint32_t>());
    cut = dv[cap - 1];  // the cap-th largest degree
    uint64_t at_or_above = 0;
    for (uint32_t x : dv) at_or_above += x >= cut;
    if (at_or_above > cap) ++cut;  // ties at the cut would overflow: leave them out
  }
  std::vector<uint32_t> hub_vid;
  std::vector<uint16_t> slot(n, NO_HUB);
  for (uint32_t v : cand)
    if (deg[v] >= cut) {
      slot[v] = uint16_t(hub_vid.size());
      hub_vid.push_back(v);
    }
  if (hub_vid.empty()) return MG_OK;
  cudaStream_t st = dg->stream;
  uint16_t* d_slot;
  uint32_t *d_bits, *d_vid;
  int rc;
  if ((rc = dev_alloc(dg, (void**)&d_slot, uint64_t(n) * 2))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_bits, hub_vid.size() * row_bytes))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_vid, hub_vid.size() * 4))) return rc;
  MG_CK(cudaMemcpyAsync(d_slot, slot.data(), uint64_t(n) * 2, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(d_vid, hub_vid.data(), hub_vid.size() * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemsetAsync(d_bits, 0, hub_vid.size() * row_bytes, st));
  k_hub_bits<<<unsigned(hub_vid.size()), 256, 0, st>>>(dg->g.adj[d], dg->g.loff[d], dg->g.L,
                                                      d_vid, words, d_bits);
  MG_CK(cudaGetLastError());
  MG_CK(cudaStreamSynchronize(st));
  dg->g.hub_slot[d] = d_slot;
  dg->g.hub_bits[d] = d_bits;
  dg->g.hub_vid[d] = d_vid;
  dg->g.n_hubs[d] = uint32_t(hub_vid.size());
  dg->g.hub_words = words;
  dg->info.hubs += uint32_t(hub_vid.size());
  dg->info.hub_min_degree = cut;
  dg->info.hub_bytes += hub_vid.size() * row_bytes;
  return MG_OK;
}

// Builds adjacency + slices for one direction from raw host arrays.
static int build_direction(DevGraph* dg, int d, const uint32_t* h_off, const uint32_t* h_adj,
                           uint32_t m, const uint32_t* d_g2l, uint32_t max_vid,
                           const uint32_t* d_label, uint32_t* d_err) {
  cudaStream_t st = dg->stream;
  const uint32_t n = dg->g.n, L = dg->g.L, W = dg->g.W;
  uint32_t *off = nullptr, *adj = nullptr;
  MG_CK(cudaMallocAsync((void**)&off, (uint64_t(n) + 1) * 4, st));
  MG_CK(cudaMallocAsync((void**)&adj, std::max<uint64_t>(1, m) * 4ull, st));
  MG_CK(cudaMemcpyAsync(off, h_off, (uint64_t(n) + 1) * 4, cudaMemcpyHostToDevice, st));
  if (m) MG_CK(cudaMemcpyAsync(adj, h_adj, uint64_t(m) * 4, cudaMemcpyHostToDevice, st));
  if (d_g2l && m) k_map_edges<<<grid_for(m, 256, dg->sms * 32), 256, 0, st>>>(adj, m, d_g2l, max_vid, d_err);
  uint32_t* d_flags = d_err + 1;
  MG_CK(cudaMemsetAsync(d_flags, 0, 4, st));
  k_check_lists<<<grid_for(uint64_t(n) * 32, 256, dg->sms * 32), 256, 0, st>>>(off, adj, n, d_flags);
  uint32_t flags = 0;
  MG_CK(cudaMemcpyAsync(&flags, d_flags, 4, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  if (flags & 2) {
    cudaFreeAsync(off, st);
    cudaFreeAsync(adj, st);
    return set_error(MG_E_FORMAT, "adjacency entry outside the vertex range");
  }
  uint32_t mm = m;
  if (flags & 1) {
    // Unsorted or repeated entries: segmented sort, then drop repeats.
    uint32_t* sorted = nullptr;
    MG_CK(cudaMallocAsync((void**)&sorted, std::max<uint64_t>(1, m) * 4ull, st));
    size_t tmp_bytes = 0;
    MG_CK(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp_bytes, adj, sorted, m, n, off,
                                             off + 1, st));
    void* tmp = nullptr;
    MG_CK(cudaMallocAsync(&tmp, std::max<size_t>(16, tmp_bytes), st));
    MG_CK(cub::DeviceSegmentedSort::SortKeys(tmp, tmp_bytes, adj, sorted, m, n, off,
                                             off + 1, st));
    cudaFreeAsync(tmp, st);
    uint32_t *newdeg = nullptr, *newoff = nullptr;
    MG_CK(cudaMallocAsync((void**)&newdeg, (uint64_t(n) + 1) * 4, st));
    MG_CK(cudaMallocAsync((void**)&newoff, (uint64_t(n) + 1) * 4, st));
    k_count_unique<<<grid_for(uint64_t(n) * 32, 256, dg->sms * 32), 256, 0, st>>>(off, sorted, n, newdeg);
    tmp_bytes = 0;
    MG_CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, newdeg, newoff, n + 1, st));
    MG_CK(cudaMallocAsync(&tmp, std::max<size_t>(16, tmp_bytes), st));
    k_set_u32<<<1, 1, 0, st>>>(newdeg, n, 0);
    MG_CK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, newdeg, newoff, n + 1, st));
    cudaFreeAsync(tmp, st);
    k_compact_unique<<<grid_for(uint64_t(n) * 32, 256, dg->sms * 32), 256, 0, st>>>(off, sorted, n, newoff, adj);
    MG_CK(cudaMemcpyAsync(&mm, newoff + n, 4, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(sorted, st);
    cudaFreeAsync(newdeg, st);
    cudaFreeAsync(off, st);
    off = newoff;
    MG_CK(cudaStreamSynchronize(st));
  }
  uint32_t *adjL, *loff, *nlb, *deg;
  int rc;
  if ((rc = dev_alloc(dg, (void**)&adjL, uint64_t(std::max(mm, 1u)) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&loff, (uint64_t(n) * L + 1) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&nlb, uint64_t(n) * W * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&deg, uint64_t(n) * 4))) return rc;
  const unsigned block = 256;
  const size_t smem = size_t(block / 32) * L * 4;
  k_partition_labels<<<grid_for(uint64_t(n) * 32, block, dg->sms * 16), block, smem, st>>>(
      off, adj, n, d_label, L, W, loff, adjL, nlb, deg, const_cast<uint32_t*>(dg->g.selfbits));
  k_set_u32<<<1, 1, 0, st>>>(loff, uint64_t(n) * L, mm);
  MG_CK(cudaGetLastError());
  cudaFreeAsync(off, st);
  cudaFreeAsync(adj, st);
  dg->g.adj[d] = adjL;
  dg->g.loff[d] = loff;
  dg->g.nlb[d] = nlb;
  dg->g.deg[d] = deg;
  if (d == 0) dg->info.m_out = mm;
  else dg->info.m_in = mm;
  return MG_OK;
}

static int upload(const mg_csr_view* v, int device, const mg_upload_opts& uo, DevGraph* dg) {
  int rc = validate_csr_view(v);
  if (rc) return rc;
  if (v->n == 0) return set_error(MG_E_ARG, "empty data graph");
  int ndev = 0;
  MG_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev)
    return set_error(MG_E_ARG, "device %d not present (%d devices)", device, ndev);
  MG_CK(cudaSetDevice(device));
  dg->device = device;
  int sms = 0;
  MG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  dg->sms = unsigned(std::max(sms, 1));
  MG_CK(cudaStreamCreateWithFlags(&dg->stream, cudaStreamNonBlocking));
  cudaStream_t st = dg->stream;
  const uint32_t n = v->n;
  dg->g.n = n;
  dg->info.n = n;
  dg->info.device = device;

  // Label compaction (host): distinct raw labels, ascending.  Small label
  // values (the usual case) are collected with a presence table in one pass;
  // other values by sorting a copy.
  std::vector<uint32_t> vals;
  {
    uint32_t lmax = 0;
    for (uint32_t i = 0; i < n; ++i) lmax = std::max(lmax, v->labels[i]);
    if (lmax < (1u << 22)) {
      std::vector<uint8_t> seen(uint64_t(lmax) + 1, 0);
      for (uint32_t i = 0; i < n; ++i) seen[v->labels[i]] = 1;
      for (uint32_t x = 0; x <= lmax; ++x)
        if (seen[x]) vals.push_back(x);
    } else {
      vals.assign(v->labels, v->labels + n);
      std::sort(vals.begin(), vals.end());
      vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    }
  }
  if (vals.size() > MG_MAX_LABELS)
    return set_error(MG_E_LIMIT, "%zu distinct labels; at most %d supported", vals.size(),
                     MG_MAX_LABELS);
  const uint32_t L = uint32_t(vals.size());
  const uint32_t W = (L + 31) / 32;
  dg->g.L = L;
  dg->g.W = W;
  dg->info.n_labels = L;
  dg->info.nlb_words = W;
  dg->stats.n = n;
  dg->stats.L = L;
  dg->stats.label_values = vals;
  std::vector<uint32_t> lab(n);
  std::vector<uint64_t> cnt(L, 0);
  if (vals.back() < (1u << 22)) {
    std::vector<uint32_t> to_compact(uint64_t(vals.back()) + 1, 0);
    for (uint32_t c = 0; c < L; ++c) to_compact[vals[c]] = c;
    for (uint32_t i = 0; i < n; ++i) {
      lab[i] = to_compact[v->labels[i]];
      cnt[lab[i]]++;
    }
  } else {
    for (uint32_t i = 0; i < n; ++i) {
      lab[i] = uint32_t(std::lower_bound(vals.begin(), vals.end(), v->labels[i]) - vals.begin());
      cnt[lab[i]]++;
    }
  }
  dg->stats.label_count = cnt;
  dg->h_bucket_off.assign(L + 1, 0);
  for (uint32_t l = 0; l < L; ++l) dg->h_bucket_off[l + 1] = dg->h_bucket_off[l] + uint32_t(cnt[l]);
  std::vector<uint32_t> bvid(n), bpos(n);
  {
    std::vector<uint32_t> cur(dg->h_bucket_off.begin(), dg->h_bucket_off.end() - 1);
    for (uint32_t i = 0; i < n; ++i) {
      bpos[i] = cur[lab[i]] - dg->h_bucket_off[lab[i]];
      bvid[cur[lab[i]]++] = i;
    }
  }
  uint32_t *d_label, *d_boff, *d_bvid, *d_bpos, *d_self, *d_gid, *d_err;
  if ((rc = dev_alloc(dg, (void**)&d_label, uint64_t(n) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_boff, uint64_t(L + 1) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_bvid, uint64_t(n) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_bpos, uint64_t(n) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_self, uint64_t((n + 31) / 32) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_gid, uint64_t(n) * 4))) return rc;
  if ((rc = dev_alloc(dg, (void**)&d_err, 16))) return rc;
  MG_CK(cudaMemcpyAsync(d_label, lab.data(), uint64_t(n) * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(d_boff, dg->h_bucket_off.data(), uint64_t(L + 1) * 4,
                        cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(d_bvid, bvid.data(), uint64_t(n) * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(d_bpos, bpos.data(), uint64_t(n) * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(d_gid, v->globalid, uint64_t(n) * 4, cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemsetAsync(d_self, 0, uint64_t((n + 31) / 32) * 4, st));
  MG_CK(cudaMemsetAsync(d_err, 0, 16, st));
  dg->g.label = d_label;
  dg->g.bucket_off = d_boff;
  dg->g.bucket_vid = d_bvid;
  dg->g.bucket_pos = d_bpos;
  dg->g.selfbits = d_self;
  dg->g.globalid = d_gid;

  // Global ids -> local ids when the stored ids are not the identity.
  bool ident = true;
  for (uint32_t i = 0; i < n && ident; ++i) ident = v->globalid[i] == i;
  uint32_t* d_g2l = nullptr;
  if (!ident) {
    MG_CK(cudaMallocAsync((void**)&d_g2l, (uint64_t(v->max_vid) + 1) * 4, st));
    MG_CK(cudaMemsetAsync(d_g2l, 0xFF, (uint64_t(v->max_vid) + 1) * 4, st));
    k_build_g2l<<<grid_for(n, 256, dg->sms * 32), 256, 0, st>>>(d_gid, n, d_g2l, v->max_vid, d_err);
  }
  const bool sym = v->m_in == v->m_out && arrays_equal(v->in_off, v->out_off, uint64_t(n) + 1) &&
                   arrays_equal(v->in_edges, v->out_edges, v->m_out);
  dg->g.symmetric = sym;
  dg->info.symmetric = sym;
  dg->stats.symmetric = sym;
  rc = build_direction(dg, 0, v->out_off, v->out_edges, v->m_out, d_g2l, v->max_vid, d_label, d_err);
  if (rc == MG_OK) {
    if (sym) {
      dg->g.adj[1] = dg->g.adj[0];
      dg->g.loff[1] = dg->g.loff[0];
      dg->g.nlb[1] = dg->g.nlb[0];
      dg->g.deg[1] = dg->g.deg[0];
      dg->info.m_in = dg->info.m_out;
    } else {
      rc = build_direction(dg, 1, v->in_off, v->in_edges, v->m_in, d_g2l, v->max_vid, d_label, d_err);
    }
  }
  if (d_g2l) cudaFreeAsync(d_g2l, st);
  if (rc) return rc;
  uint32_t err = 0;
  MG_CK(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  if (err & ERR_RANGE) return set_error(MG_E_FORMAT, "vertex id outside [0, max_vid] or unknown");
  // Maximum degree (host reduction over the reference outdeg is not trusted:
  // read the distinct-neighbour degrees back), then the hub bitmaps.
  uint64_t budget = uo.hub_bytes;
  if (budget == MG_HUB_AUTO) {
    size_t free_b = 0, total_b = 0;
    MG_CK(cudaMemGetInfo(&free_b, &total_b));
    budget = std::min<uint64_t>(4ull << 30, free_b / 8);
  }
  const uint32_t min_degree = uo.hub_min_degree ? uo.hub_min_degree : 128u;
  for (int d = 0; d < (sym ? 1 : 2); ++d) {
    std::vector<uint32_t> h(n);
    MG_CK(cudaMemcpy(h.data(), dg->g.deg[d], uint64_t(n) * 4, cudaMemcpyDeviceToHost));
    if (d == 0) dg->info.max_degree = *std::max_element(h.begin(), h.end());
    if (budget && (rc = build_hubs(dg, d, h, sym ? budget : budget / 2, min_degree))) return rc;
  }
  if (sym) {
    dg->g.hub_slot[1] = dg->g.hub_slot[0];
    dg->g.hub_bits[1] = dg->g.hub_bits[0];
    dg->g.hub_vid[1] = dg->g.hub_vid[0];
    dg->g.n_hubs[1] = dg->g.n_hubs[0];
  }
  return MG_OK;
}

int ensure_full_stats(DevGraph* dg) {
  if (dg->stats_full) return MG_OK;
  const uint32_t L = dg->g.L, n = dg->g.n;
  cudaStream_t st = dg->stream;
  unsigned long long *dsum, *dhist, *dpair;
  unsigned int* dmax;
  MG_CK(cudaMallocAsync((void**)&dsum, L * 8ull, st));
  MG_CK(cudaMallocAsync((void**)&dhist, L * 33 * 8ull, st));
  MG_CK(cudaMallocAsync((void**)&dpair, uint64_t(L) * L * 8, st));
  MG_CK(cudaMallocAsync((void**)&dmax, L * 4ull, st));
  MG_CK(cudaMemsetAsync(dsum, 0, L * 8ull, st));
  MG_CK(cudaMemsetAsync(dhist, 0, L * 33 * 8ull, st));
  MG_CK(cudaMemsetAsync(dpair, 0, uint64_t(L) * L * 8, st));
  MG_CK(cudaMemsetAsync(dmax, 0, L * 4ull, st));
  k_label_stats<<<grid_for(n, 256, dg->sms * 32), 256, 0, st>>>(dg->g.loff[0], dg->g.label, n, L, dsum, dmax,
                                                  dhist, dpair);
  std::vector<unsigned long long> hsum(L), hhist(L * 33), hpair(uint64_t(L) * L);
  std::vector<unsigned int> hmax(L);
  MG_CK(cudaMemcpyAsync(hsum.data(), dsum, L * 8ull, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(hhist.data(), dhist, L * 33 * 8ull, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(hpair.data(), dpair, uint64_t(L) * L * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(hmax.data(), dmax, L * 4ull, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  cudaFreeAsync(dsum, st);
  cudaFreeAsync(dhist, st);
  cudaFreeAsync(dpair, st);
  cudaFreeAsync(dmax, st);
  auto& S = dg->stats;
  S.label_deg_mean.assign(L, 0);
  S.label_deg_max.assign(L, 0);
  S.label_deg_p99.assign(L, 0);
  S.label_pair_edges.assign(hpair.begin(), hpair.end());
  S.label_nlb_density.assign(L, 0);
  for (uint32_t l = 0; l < L; ++l) {
    uint64_t c = S.label_count[l];
    S.label_deg_mean[l] = c ? double(hsum[l]) / double(c) : 0.0;
    S.label_deg_max[l] = double(hmax[l]);
    uint64_t target = c - c / 100, acc = 0;
    for (uint32_t b = 0; b < 33; ++b) {
      acc += hhist[l * 33 + b];
      if (acc >= target && c) {
        S.label_deg_p99[l] = b == 0 ? 0.0 : double((1ull << b) - 1);
        break;
      }
    }
    uint64_t nl = 0;
    for (uint32_t l2 = 0; l2 < L; ++l2) nl += hpair[uint64_t(l) * L + l2] > 0;
    S.label_nlb_density[l] = nl;
  }
  dg->stats_full = true;
  return MG_OK;
}

// Device of an entry point that takes no device argument: the one named by
// MATRIXGRAPH_CUDA_DEVICE when it is a valid index (the reference's
// set_device_from_env, core/go_api/matrixgraph_go_api.cu:22-34), else the
// calling thread's current device.  The current device is not changed.
int env_or_current_device(int* dev) {
  int count = 0;
  MG_CK(cudaGetDeviceCount(&count));
  const char* s = std::getenv("MATRIXGRAPH_CUDA_DEVICE");
  if (s && s[0]) {
    const int d = std::atoi(s);
    if (d >= 0 && d < count) {
      *dev = d;
      return MG_OK;
    }
  }
  MG_CK(cudaGetDevice(dev));
  return MG_OK;
}

}  // namespace mg

extern "C" {

int mg_graph_upload(const mg_csr_view* g, int device, void** dgraph) {
  return mg_graph_upload_ex(g, device, nullptr, dgraph);
}

int mg_graph_upload_ex(const mg_csr_view* g, int device, const mg_upload_opts* opts,
                       void** dgraph) {
  mg::clear_error();
  if (!g || !dgraph) return mg::set_error(MG_E_ARG, "null argument");
  mg_upload_opts uo{MG_HUB_AUTO, 0, 0};
  if (opts) uo = *opts;
  if (uo._reserved) return mg::set_error(MG_E_ARG, "reserved upload option must be 0");
  auto* dg = new (std::nothrow) mg::DevGraph();
  if (!dg) return mg::set_error(MG_E_OOM, "host allocation failed");
  int prev = 0;
  cudaGetDevice(&prev);
  int rc;
  try {
    rc = mg::upload(g, device, uo, dg);
  } catch (const std::bad_alloc&) {
    rc = mg::set_error(MG_E_OOM, "host allocation failed");
  }
  cudaSetDevice(prev);
  if (rc) {
    delete dg;
    return rc;
  }
  *dgraph = dg;
  return MG_OK;
}

void mg_graph_free(void* dgraph) { delete static_cast<mg::DevGraph*>(dgraph); }

int mg_graph_get_info(void* dgraph, mg_graph_info* info) {
  mg::clear_error();
  if (!dgraph || !info) return mg::set_error(MG_E_ARG, "null argument");
  *info = static_cast<mg::DevGraph*>(dgraph)->info;
  return MG_OK;
}

}  // extern "C"
