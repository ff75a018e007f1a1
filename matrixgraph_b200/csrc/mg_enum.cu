// Exact subgraph enumeration: candidate filtering + worst-case-optimal-join
// extension by sorted-list intersection, as a memory-bounded hybrid
// BFS/DFS over level tables.
//
// Replaces the reference GPU WOJ path (WOJFilterVCKernel
// core/task/gpu_task/kernel/kernel_woj_subsio.cu:532-604, the per-table
// MergeSort core/task/gpu_task/kernel/algorithms/sort.cuh:59-105 and
// WOJJoinKernel kernel_woj_subsio.cu:623-721), which joins one key column at
// a time, never checks cycle closure or injectivity and caps its output at
// kMaxNumWeft rows.  Here:
//   * a level table holds partial matches of prefix length i (SoA columns);
//   * the work kernel picks, per row, the shortest label slice among the
//     backward neighbours' adjacency (the driving list) and the scan turns
//     the driving lengths into an element index space;
//   * the expand kernel assigns one element (row, driving entry) per thread,
//     so hub rows spread over many warps; the other backward slices are
//     probed in the hub bitmap when their vertex is a hub, else by binary
//     search, injectivity is checked against the row, the
//     label/degree/neighbour-label filter prunes, and survivors are appended
//     with warp-aggregated atomics (__ballot_sync / __popc);
//   * a table chunk never holds more than `cap` rows: the host walks the
//     levels depth-first, expanding at most `cap` elements of a level before
//     descending, so intermediate results never exceed the scratch budget;
//   * in count mode the last position is never materialised: when it has a
//     single backward neighbour its count is the slice length minus the
//     injectivity collisions, added while expanding the position before it;
//     a two-position pendant tail is counted from two-hop aggregates while
//     expanding the position three before the end.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "mg_device.cuh"

namespace mg {

const char* last_error_cstr();

// ---------------------------------------------------------------------------
// Workspace (per graph handle)
// ---------------------------------------------------------------------------
// Pendant-tail keys of a call and the two-hop aggregates of their hubs.
struct TailStore {
  unsigned long long* A = nullptr;
  unsigned long long* AD = nullptr;
  uint64_t cap = 0;
  unsigned long long* lazy = nullptr;  // packed (AD << 32 | A), ~0 = not yet filled
  uint64_t lazy_cap = 0;
  TailKey* keys = nullptr;
  uint32_t keys_cap = 0;
};

struct Workspace {
  int device = 0;
  uint64_t cap = 0;       // rows per level table (and elements per chunk)
  uint32_t rows0 = 0;     // capacity of the level-0 table (one row per query)
  int levels = 0;         // level tables allocated: 0..levels-1
  uint32_t* col[MAXK][MAXK] = {};
  uint32_t* qid[MAXK] = {};
  uint32_t* work[MAXK] = {};
  uint64_t* woff[MAXK] = {};
  uint32_t* dstart[MAXK] = {};
  uint8_t* dci[MAXK] = {};
  uint64_t* bsum = nullptr;
  uint32_t bsum_cap = 0;
  uint32_t* tile_row = nullptr;  // first row of every expand tile of a segment
  uint32_t* root_keep = nullptr; // matrix-filter keep bits of the level-0 candidates
  uint64_t root_keep_words = 0;
  TailStore tails;
  unsigned long long* ctr = nullptr;     // device counters
  unsigned long long* h_ctr = nullptr;   // pinned mirror
  unsigned long long* counts = nullptr;  // per query
  unsigned long long* lvl_rows = nullptr;  // per query, MAXK + 1 prefix lengths
  unsigned long long* q_elems = nullptr;   // per query, elements scheduled
  uint32_t counts_cap = 0;
  PlanDev* plans = nullptr;
  uint32_t plans_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  std::vector<void*> allocs;
  uint64_t bytes = 0;
};

// Counter slots.
enum : int {
  C_OUT = 0, C_BALG = 1, C_BALGC = 2, C_ERR = 3, C_EMIT = 4, C_TILE = 6,
  // Lane pipeline (sizes live on the device), one slot per level l:
  C_LOUT = 8,                // rows the expand of level l wrote (= rows of level l+1)
  C_LTILE = C_LOUT + MAXK,   // work-queue position of the expand of level l
  C_LT = C_LTILE + MAXK,     // candidate elements of level l
  C_LSCAN = C_LT + MAXK,     // tile counter of the work/scan kernel of level l
  C_NUM = C_LSCAN + MAXK
};

void free_workspace(Workspace* ws) {
  if (!ws) return;
  for (void* p : ws->allocs) cudaFree(p);
  if (ws->h_ctr) cudaFreeHost(ws->h_ctr);
  if (ws->ev0) cudaEventDestroy(ws->ev0);
  if (ws->ev1) cudaEventDestroy(ws->ev1);
  if (ws->ev2) cudaEventDestroy(ws->ev2);
  if (ws->ev3) cudaEventDestroy(ws->ev3);
  delete ws;
}

static int ws_alloc(Workspace* ws, void** p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_error(MG_E_OOM, "enumeration scratch: cudaMalloc(%zu) failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  ws->allocs.push_back(*p);
  ws->bytes += bytes;
  return MG_OK;
}

constexpr uint64_t kDefaultCap = 1ull << 24;
constexpr uint32_t kProbeMin = 1;  // default: every hub slice is probed in the bitmap
constexpr int SCAN_TILE = 4096;
constexpr int EXPAND_BLOCK = 256;                 // elements per expand tile
constexpr uint64_t kSegment = 1ull << 26;         // elements per expand launch

static uint64_t level_row_bytes(int l) { return uint64_t(l) * 4 + 4 + 4 + 8 + 4 + 1; }

static int ensure_ws(DevGraph* dg, uint64_t cap, int levels, uint32_t nq) {
  Workspace*& ws = dg->ws;
  if (ws && (ws->cap != cap || ws->rows0 < nq)) {
    cudaStreamSynchronize(dg->stream);
    free_workspace(ws);
    ws = nullptr;
  }
  if (!ws) {
    ws = new Workspace();
    ws->device = dg->device;
    ws->cap = cap;
    ws->rows0 = std::max<uint32_t>(nq, 1024);
    int rc;
    if ((rc = ws_alloc(ws, (void**)&ws->ctr, C_NUM * 8))) return rc;
    MG_CK(cudaMallocHost((void**)&ws->h_ctr, C_NUM * 8));
    MG_CK(cudaEventCreate(&ws->ev0));
    MG_CK(cudaEventCreate(&ws->ev1));
    MG_CK(cudaEventCreate(&ws->ev2));
    MG_CK(cudaEventCreate(&ws->ev3));
    ws->bsum_cap = uint32_t((std::max<uint64_t>(cap, ws->rows0) + SCAN_TILE - 1) / SCAN_TILE + 1);
    if ((rc = ws_alloc(ws, (void**)&ws->bsum, uint64_t(ws->bsum_cap) * 8))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->tile_row, (kSegment / EXPAND_BLOCK + 2) * 4))) return rc;
  }
  if (ws->counts_cap < nq) {
    int rc;
    if ((rc = ws_alloc(ws, (void**)&ws->counts, uint64_t(nq) * 8))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->lvl_rows, uint64_t(nq) * (MAXK + 1) * 8))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->q_elems, uint64_t(nq) * 8))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->plans, uint64_t(nq) * sizeof(PlanDev)))) return rc;
    ws->counts_cap = ws->plans_cap = nq;
  }
  for (int l = ws->levels; l < levels; ++l) {
    const uint64_t rows = l == 0 ? ws->rows0 : cap;
    int rc;
    for (int j = 0; j < l; ++j)
      if ((rc = ws_alloc(ws, (void**)&ws->col[l][j], rows * 4))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->qid[l], rows * 4))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->work[l], rows * 4))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->woff[l], (rows + 1) * 8))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->dstart[l], rows * 4))) return rc;
    if ((rc = ws_alloc(ws, (void**)&ws->dci[l], rows))) return rc;
    ws->levels = l + 1;
  }
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
struct TabPtrs {
  uint32_t* col[MAXK];
  uint32_t* qid;  // nullptr: single query, q = 0
};

struct StepArgs {
  GraphDev g;
  const PlanDev* plans;
  uint32_t level;   // rows hold positions 0..level-1; position `level` is extended
  uint32_t R;       // rows of the input table
  TabPtrs in;
  uint32_t* work;
  uint64_t* woff;
  uint32_t* dstart;
  uint8_t* dci;
  uint64_t t0, t1;  // element range of this expand launch
  TabPtrs out;
  uint64_t out_cap;
  unsigned long long* ctr;
  unsigned long long* counts;
  unsigned long long* lvl_rows;  // per query: surviving prefixes of length 0..MAXK
  unsigned long long* q_elems;   // per query: candidate elements scheduled so far
  unsigned long long q_budget;   // per-query element budget (0: none)
  uint32_t count_mode;
  uint32_t filters;
  uint32_t stats;
  uint32_t nq;
  uint32_t* emit_col[MAXK];
  uint64_t emit_cap;
  uint64_t root_begin, root_end;  // level-0 candidate range (root_end 0: all)
  uint32_t root_step;             // level-0 stride inside the range (>= 1)
  uint32_t probe_min;             // shortest hub slice probed in the hub bitmap
  const uint32_t* tile_row;        // first row of each tile of [t0, t1)
  uint32_t grab;   // expand tiles taken per work-queue grab
  const TailKey* tkeys;
  // Two-position pendant tails (tail_dense): counted while expanding
  // position k-3; the two-hop aggregates of a hub m_p are read at
  // tkeys[kid].base + hub slot, those of other vertices summed in place.
  uint32_t tail_dense;
  uint32_t star;  // two-leaf star endings are counted in closed form (PlanDev::star2)
  const unsigned long long* tdA;
  const unsigned long long* tdAD;
  unsigned long long* tdL;  // lazily filled aggregates of non-hub vertices
  // Lane pipeline: row and element counts come from the counters (C_LOUT,
  // C_LT), the expand's queue and output use the per-level slots, and no
  // host value of R, t0 or t1 is read.
  uint32_t lane;
  uint32_t out_slot, tile_slot;  // counter slots of the output rows / work queue
  uint64_t cap_rows;             // rows of a lane's level table
  uint64_t seg_cap;              // elements one lane expand launch can tile
  unsigned long long* scan_status;  // look-back words of the work/scan kernel
  uint32_t spin_limit;           // bounded device waits (iterations)
  const uint32_t* root_keep;     // level-0 candidates kept by the matrix filter
                                 // (bit per vertex; nullptr: no filter)
};

// Rows of the input table of a lane launch at level a.level.
__device__ __forceinline__ uint64_t lane_rows(const StepArgs& a) {
  if (a.level == 0) return 1;
  const uint64_t r = a.ctr[C_LOUT + a.level - 1];
  return r < a.cap_rows ? r : a.cap_rows;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t l = threadIdx.x & 31;
  return (1u << l) - 1u;
}

// Binary search for x in the sorted range a[s, e).
__device__ __forceinline__ bool contains(const uint32_t* __restrict__ a, uint32_t s, uint32_t e,
                                         uint32_t x) {
  uint32_t lo = s, hi = e;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    uint32_t v = __ldg(a + mid);
    if (v < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < e && __ldg(a + lo) == x;
}

__device__ __forceinline__ void slice_of(const GraphDev& g, uint32_t dir, uint32_t y,
                                         uint32_t lab, uint32_t& s, uint32_t& e) {
  const uint32_t* p = g.loff[dir] + uint64_t(y) * g.L + lab;
  s = __ldg(p);
  e = __ldg(p + 1);
}

// Probe strategy: a slice of a hub with at least `pmin` entries is probed in
// the hub's bitmap (one load, but a random sector of a row that may not sit
// in L2); shorter slices and non-hubs by binary search (a few loads that
// usually hit L1, since the elements of one row probe the same slice).
__device__ __forceinline__ bool hub_bit(const GraphDev& g, uint32_t d, uint16_t h, uint32_t x) {
  return (__ldg(g.hub_bits[d] + uint64_t(h) * g.hub_words + (x >> 5)) >> (x & 31)) & 1u;
}

// x in the d-adjacency of y, where x is known to carry the label of the slice
// [s, e) of y being asked about.
__device__ __forceinline__ bool in_slice_se(const GraphDev& g, uint32_t d, uint32_t y, uint32_t s,
                                            uint32_t e, uint32_t x, uint32_t pmin) {
  if (g.hub_slot[d] && e - s >= pmin) {
    const uint16_t h = __ldg(g.hub_slot[d] + y);
    if (h != NO_HUB) return hub_bit(g, d, h, x);
  }
  return contains(g.adj[d], s, e, x);
}

// x (labelled lab) in the label-lab slice of y's d-adjacency; with pmin <= 1
// a hub needs no slice offsets at all.
__device__ __forceinline__ bool in_slice(const GraphDev& g, uint32_t d, uint32_t y, uint32_t lab,
                                         uint32_t x, uint32_t pmin) {
  uint32_t s, e;
  if (g.hub_slot[d] && pmin <= 1) {
    const uint16_t h = __ldg(g.hub_slot[d] + y);
    if (h != NO_HUB) return hub_bit(g, d, h, x);
    slice_of(g, d, y, lab, s, e);  // not a hub: search the slice
    return contains(g.adj[d], s, e, x);
  }
  slice_of(g, d, y, lab, s, e);
  return in_slice_se(g, d, y, s, e, x, pmin);
}

__device__ __forceinline__ bool pass_filters(const GraphDev& g, const PlanDev& P, uint32_t i,
                                             uint32_t x, uint32_t filters) {
  if (filters & MG_FILTER_DEGREE) {
    if (__ldg(g.deg[0] + x) < P.req[0][i]) return false;
    if (!g.symmetric && __ldg(g.deg[1] + x) < P.req[1][i]) return false;
  }
  if (filters & MG_FILTER_NLB) {
    for (uint32_t w = 0; w < g.W; ++w) {
      if (P.nlbq[0][i][w] & ~__ldg(g.nlb[0] + uint64_t(x) * g.W + w)) return false;
      if (!g.symmetric && (P.nlbq[1][i][w] & ~__ldg(g.nlb[1] + uint64_t(x) * g.W + w)))
        return false;
    }
  }
  return true;
}

__device__ __forceinline__ bool has_self(const GraphDev& g, uint32_t x) {
  return (__ldg(g.selfbits + (x >> 5)) >> (x & 31)) & 1u;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(FULL, v, d);
  return v;
}

// Largest r in [lo, hi] with woff[r] <= t (woff non-decreasing, woff[lo] <= t).
__device__ __forceinline__ uint32_t find_row(const uint64_t* __restrict__ woff, uint32_t lo,
                                             uint32_t hi, uint64_t t) {
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (woff[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Adds a thread's accumulated match count and prefix survivors of query q:
// s1 prefixes of length i+1, s2 of length i+2 and sk of length k (the last
// two from closed-form counts).
__device__ __forceinline__ void acc_flush(const StepArgs& a, uint32_t q, uint32_t i,
                                          unsigned long long cnt, unsigned long long s1,
                                          unsigned long long sk, unsigned long long s2 = 0) {
  if (cnt) atomicAdd(&a.counts[q], cnt);
  unsigned long long* L = a.lvl_rows + uint64_t(q) * (MAXK + 1);
  if (s1) atomicAdd(&L[i + 1], s1);
  if (s2) atomicAdd(&L[i + 2], s2);
  if (sk) atomicAdd(&L[a.plans[q].k], sk);
}

// Flush of a warp's accumulators: one atomic per value when every lane holds
// the same query, else one per lane.
__device__ __forceinline__ void acc_flush_warp(const StepArgs& a, uint32_t q, uint32_t i,
                                               unsigned long long& cnt,
                                               unsigned long long& s1,
                                               unsigned long long& sk,
                                               unsigned long long& s2, bool force) {
  const bool uniform = __all_sync(FULL, q == __shfl_sync(FULL, q, 0));
  if (uniform) {
    const unsigned long long c = warp_sum(cnt), x = warp_sum(s1), y = warp_sum(sk),
                             z = warp_sum(s2);
    if ((threadIdx.x & 31) == 0) acc_flush(a, q, i, c, x, y, z);
    cnt = s1 = sk = s2 = 0;
  } else if (force) {
    acc_flush(a, q, i, cnt, s1, sk, s2);
    cnt = s1 = sk = s2 = 0;
  }
}

// Two-hop aggregates of one tail key for the hubs of direction da, warp per
// hub: for y labelled lp,
//   A(y)  = sum_{x in N^{da}_{la}(y)} (|N^{db}_{lb}(x)| - [x self-loop, la == lb]),
//   AD(y) = sum_{x in N^{da}_{la}(y)} |N^{db}_{lb}(x)|
// at tdA / tdAD[tk.base + hub slot] (hubs of other labels are skipped: no
// prefix can match them at position p).
__global__ void __launch_bounds__(256) k_tail_dense(GraphDev g, TailKey tk,
                                                    unsigned long long* tdA,
                                                    unsigned long long* tdAD) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  const uint32_t nh = g.n_hubs[tk.da];
  for (uint64_t h = warp; h < nh; h += nwarps) {
    const uint32_t y = __ldg(g.hub_vid[tk.da] + h);
    if (__ldg(g.label + y) != tk.lp) continue;
    uint32_t s, e;
    slice_of(g, tk.da, y, tk.la, s, e);
    unsigned long long sa = 0, sd = 0;
    for (uint32_t q = s + lane; q < e; q += 32) {
      const uint32_t x = __ldg(g.adj[tk.da] + q);
      uint32_t xs, xe;
      slice_of(g, tk.db, x, tk.lb, xs, xe);
      sd += xe - xs;
      sa += xe - xs - ((tk.la == tk.lb && has_self(g, x)) ? 1u : 0u);
    }
    sa = warp_sum(sa);
    sd = warp_sum(sd);
    if (lane == 0) {
      tdA[tk.base + h] = sa;
      tdAD[tk.base + h] = sd;
    }
  }
}

// Two-hop aggregates A(m_p), AD(m_p) of a tail (see k_tail_dense): from the
// hub table when m_p is a hub; otherwise from the key's lazy table over the
// bucket of label l_p, filled on first use by whichever thread needs the
// entry (A and AD packed in one 64-bit word, so a reader sees an entry whole
// or not at all; concurrent fillers store the same value), or summed over the
// label-l_a slice [s, e) when the entry cannot be tabled.  Entries whose AD
// does not fit 32 bits are never tabled.
__device__ __forceinline__ void tail_agg(const StepArgs& a, const PlanDev& P, uint32_t mp,
                                         uint32_t s, uint32_t e, long long& c, long long& d) {
  const GraphDev& g = a.g;
  const uint32_t da = P.tail_da, db = P.tail_db;
  const TailKey& tk = a.tkeys[P.tail_kid];
  if (tk.base != ~0ull && g.hub_slot[da]) {
    const uint16_t h = __ldg(g.hub_slot[da] + mp);
    if (h != NO_HUB) {
      c = (long long)a.tdA[tk.base + h];
      d = (long long)a.tdAD[tk.base + h];
      return;
    }
  }
  unsigned long long* slot = nullptr;
  if (tk.lazy != ~0ull) {
    slot = a.tdL + tk.lazy + __ldg(g.bucket_pos + mp);
    const unsigned long long w = *reinterpret_cast<volatile unsigned long long*>(slot);
    if (w != ~0ull) {
      c = (long long)(w & 0xFFFFFFFFull);
      d = (long long)(w >> 32);
      return;
    }
  }
  const uint32_t la = tk.la, lb = tk.lb;
  c = d = 0;
  for (uint32_t j = s; j < e; ++j) {
    const uint32_t x = __ldg(g.adj[da] + j);
    uint32_t xs, xe;
    slice_of(g, db, x, lb, xs, xe);
    d += xe - xs;
    c += (long long)(xe - xs) - ((la == lb && has_self(g, x)) ? 1 : 0);
  }
  if (slot && d < 0xFFFFFFFFll)
    atomicExch(slot, (unsigned long long)(d) << 32 | (unsigned long long)(c));
}

// Closed-form count of one prefix of length a = k-2 under a two-position
// pendant tail (PlanDev::tail2).  With I the matched prefix, S = the
// label-l_a slice [s, e) of m_p, D(x) = |N_{l_b}(x)| and c(x) = D(x) - [x has
// a self-loop and l_a == l_b], and A(y) = sum_{x in S(y)} c(x),
// AD(y) = sum_{x in S(y)} D(x):
//   count = A(m_p) - sum_{i in Ia, m_i in S} (c(m_i) - #{j in J : m_j in N_{l_b}(m_i)})
//           - sum_{j in J} |S|                   (every j in J is p itself)
// Also returns the number of length-(k-1) prefixes |S \ I| and their
// algorithmic bytes sum_{x in S \ I} D(x).  col(j) is the vertex matched at
// position j < a.
template <class Col>
__device__ __forceinline__ void tail_close(const StepArgs& a, const PlanDev& P, Col col,
                                           uint32_t mp, uint32_t s, uint32_t e, long long c,
                                           long long d, unsigned long long& cnt,
                                           unsigned long long& pre, unsigned long long& dsum) {
  const GraphDev& g = a.g;
  const uint32_t ia = P.k - 2;
  const uint32_t la = P.label[ia], lb = P.label[ia + 1];
  const uint32_t da = P.tail_da, db = P.tail_db;
  unsigned long long inS = 0;
  for (uint32_t mi = P.tail_Ia; mi; mi &= mi - 1) {
    const uint32_t i2 = __ffs(mi) - 1;
    const uint32_t x = col(i2);
    if (!in_slice_se(g, da, mp, s, e, x, a.probe_min)) continue;
    inS += 1;
    uint32_t xs, xe;
    slice_of(g, db, x, lb, xs, xe);
    long long cx = (long long)(xe - xs);
    d -= cx;
    if (la == lb && has_self(g, x)) cx -= 1;
    for (uint32_t mj = P.tail_J; mj; mj &= mj - 1) {
      const uint32_t j = __ffs(mj) - 1;
      if (in_slice_se(g, db, x, xs, xe, col(j), a.probe_min)) cx -= 1;
    }
    c -= cx;
  }
  c -= (long long)__popc(P.tail_J) * (long long)(e - s);
  cnt = (unsigned long long)c;
  pre = (unsigned long long)(e - s) - inS;
  dsum = (unsigned long long)d;
}

// Closed-form count of one prefix of length k-2 whose plan ends in two leaves
// a = k-2, b = k-1 of one anchor p (PlanDev::star2).  S_a and S_b are the
// label-l_a and label-l_b slices of m_p in direction d; A_x is |S_x| minus the
// earlier matches labelled l_x that lie in S_x (injectivity).  Then
//   count = A_a * (A_a - 1)   when l_a == l_b (S_b == S_a, b differs from a),
//   count = A_a * A_b         otherwise (a and b cannot collide),
// the prefixes of length k-1 number A_a, and the algorithmic bytes of the two
// positions are (8 + 4|S_a|) per prefix of length k-2 plus (8 + 4|S_b|) per
// prefix of length k-1 (count-mode definition: 8 for the last position).
// col(j) is the vertex matched at position j < k-2.
template <class Col>
__device__ __forceinline__ void star_close(const StepArgs& a, const PlanDev& P, Col col,
                                           unsigned long long& cnt, unsigned long long& pre,
                                           unsigned long long& bal,
                                           unsigned long long& balc) {
  const GraphDev& g = a.g;
  const uint32_t ia = P.k - 2, ib = P.k - 1, d = P.star_d;
  const uint32_t mp = col(P.star_p);
  uint32_t sa, ea;
  slice_of(g, d, mp, P.label[ia], sa, ea);
  unsigned long long A = ea - sa;
  for (uint32_t m = P.samelab[ia]; m; m &= m - 1)
    if (in_slice_se(g, d, mp, sa, ea, col(__ffs(m) - 1), a.probe_min)) A -= 1;
  unsigned long long lb_len;
  if (P.label[ib] == P.label[ia]) {
    cnt = A ? A * (A - 1) : 0ull;
    lb_len = ea - sa;
  } else {
    uint32_t sb, eb;
    slice_of(g, d, mp, P.label[ib], sb, eb);
    unsigned long long B = eb - sb;
    for (uint32_t m = P.samelab[ib]; m; m &= m - 1)
      if (in_slice_se(g, d, mp, sb, eb, col(__ffs(m) - 1), a.probe_min)) B -= 1;
    cnt = A * B;
    lb_len = eb - sb;
  }
  pre = A;
  bal = 8ull + 4ull * (ea - sa) + A * (8ull + 4ull * lb_len);
  balc = 8ull + 4ull * (ea - sa) + A * 8ull;
}

// Work kernel: per row, the driving slice (shortest backward slice, or the
// label bucket for a position without backward neighbours) and the
// algorithmic-byte charge of extending the row.
// Driving slice of table row r at position a.level: its length (the row's
// candidate elements, 0 when nothing is to be expanded), start and constraint
// index (DCI_BUCKET: the label bucket), and the row's algorithmic-byte
// charges (full-slice and count-mode definitions).
__device__ __forceinline__ uint32_t row_work(const StepArgs& a, const PlanDev& P, uint64_t r,
                                             uint32_t q, uint32_t& bs, uint8_t& bci,
                                             unsigned long long& ch, unsigned long long& chc) {
  const GraphDev& g = a.g;
  const uint32_t i = a.level;
  const uint32_t lab = P.label[i];
  const uint32_t nc = P.ncons[i];
  uint32_t best;
  bs = 0;
  bci = DCI_BUCKET;
  ch = chc = 0;
  if (P.zero) {
    best = 0;
  } else if (nc == 0) {
    bs = __ldg(g.bucket_off + lab);
    best = __ldg(g.bucket_off + lab + 1) - bs;
    if (i == 0 && a.root_end) {
      const uint64_t rb = a.root_begin < best ? a.root_begin : uint64_t(best);
      const uint64_t re = a.root_end < best ? a.root_end : uint64_t(best);
      bs += uint32_t(rb);
      best = re > rb ? uint32_t((re - rb + a.root_step - 1) / a.root_step) : 0u;
    }
    ch = chc = (unsigned long long)best * (12ull + 4ull * g.W);
  } else {
    best = FULL;
    for (uint32_t c = 0; c < nc; ++c) {
      const uint32_t cs = P.cons[i][c];
      const uint32_t y = a.in.col[cs & 0xFF][r];
      uint32_t s, e;
      slice_of(g, cs >> 8, y, lab, s, e);
      ch += 8ull + 4ull * (e - s);
      if (e - s < best) {
        best = e - s;
        bs = s;
        bci = uint8_t(c);
      }
    }
    chc = (i + 1 == P.k && P.last_o1) ? 8ull : ch;
  }
  if (a.q_budget && best) {
    // Per-query budget: a query whose scheduled elements pass the budget
    // stops expanding (its count is reported as unknown).
    const unsigned long long before = atomicAdd(&a.q_elems[q], (unsigned long long)best);
    if (before + best > a.q_budget) best = 0;
  }
  return best;
}

__global__ void __launch_bounds__(256) k_work(StepArgs a) {
  unsigned long long bal = 0, balc = 0;
  // Contiguous rows per block: rows of one query stay together.
  const uint64_t per = ((a.R + gridDim.x - 1) / gridDim.x + blockDim.x - 1) / blockDim.x *
                       blockDim.x;
  const uint64_t r_end = min(uint64_t(a.R), (uint64_t(blockIdx.x) + 1) * per);
  for (uint64_t r = blockIdx.x * per + threadIdx.x; r < r_end; r += blockDim.x) {
    const uint32_t q = a.in.qid ? a.in.qid[r] : 0u;
    const PlanDev& P = a.plans[q];
    uint32_t bs;
    uint8_t bci;
    unsigned long long ch, chc;
    a.work[r] = row_work(a, P, r, q, bs, bci, ch, chc);
    a.dstart[r] = bs;
    a.dci[r] = bci;
    bal += ch;
    balc += chc;
  }
  bal = warp_sum(bal);
  balc = warp_sum(balc);
  if ((threadIdx.x & 31) == 0 && (bal | balc)) {
    atomicAdd(&a.ctr[C_BALG], bal);
    atomicAdd(&a.ctr[C_BALGC], balc);
  }
}

// Scan of the per-row driving lengths into 64-bit element offsets.
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v,
                                                                   unsigned long long* total) {
  __shared__ unsigned long long wsum[33];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long incl = v;
  for (int d = 1; d < 32; d <<= 1) {
    unsigned long long t = __shfl_up_sync(FULL, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t nw = blockDim.x >> 5;
    unsigned long long s = lane < nw ? wsum[lane] : 0ull;
    unsigned long long si = s;
    for (int d = 1; d < 32; d <<= 1) {
      unsigned long long t = __shfl_up_sync(FULL, si, d);
      if (lane >= d) si += t;
    }
    if (lane < nw) wsum[lane] = si - s;
    if (lane == nw - 1) wsum[32] = si;
  }
  __syncthreads();
  unsigned long long res = wsum[wid] + incl - v;
  *total = wsum[32];
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(256) k_scan_reduce(const uint32_t* __restrict__ in, uint32_t R,
                                                     uint64_t* bsum) {
  const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
  unsigned long long s = 0;
  for (uint32_t j = threadIdx.x; j < SCAN_TILE; j += blockDim.x) {
    uint64_t idx = base + j;
    if (idx < R) s += in[idx];
  }
  s = warp_sum(s);
  __shared__ unsigned long long ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) t += ws[w];
    bsum[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_scan_bsum(uint64_t* bsum, uint32_t nb, uint64_t* total_out) {
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += blockDim.x) {
    uint32_t i = base + threadIdx.x;
    unsigned long long v = i < nb ? bsum[i] : 0ull;
    unsigned long long tot;
    unsigned long long ex = block_exclusive_scan(v, &tot);
    if (i < nb) bsum[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(256) k_scan_apply(const uint32_t* __restrict__ in, uint32_t R,
                                                    const uint64_t* __restrict__ bsum,
                                                    uint64_t* out) {
  __shared__ uint32_t tile[SCAN_TILE + SCAN_TILE / 32];
  const uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
  for (uint32_t j = threadIdx.x; j < SCAN_TILE; j += blockDim.x) {
    uint64_t idx = base + j;
    tile[j + (j >> 5)] = idx < R ? in[idx] : 0u;
  }
  __syncthreads();
  constexpr uint32_t PER = SCAN_TILE / 256;
  const uint32_t t0 = threadIdx.x * PER;
  unsigned long long s = 0;
  for (uint32_t j = 0; j < PER; ++j) s += tile[(t0 + j) + ((t0 + j) >> 5)];
  unsigned long long tot;
  unsigned long long ex = block_exclusive_scan(s, &tot) + bsum[blockIdx.x];
  for (uint32_t j = 0; j < PER; ++j) {
    uint64_t idx = base + t0 + j;
    if (idx < R) out[idx] = ex;
    ex += tile[(t0 + j) + ((t0 + j) >> 5)];
  }
}

// First row of every tile of the element range [t0, t1): tile_row[j] is the
// row holding element t0 + j*EXPAND_BLOCK (clamped to t1 - 1), j = 0..ntiles.
__global__ void __launch_bounds__(256) k_tile_rows(const uint64_t* __restrict__ woff, uint32_t R,
                                                   uint64_t t0, uint64_t t1, uint32_t ntiles,
                                                   uint32_t* tile_row) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j <= ntiles;
       j += gridDim.x * blockDim.x) {
    uint64_t t = t0 + uint64_t(j) * EXPAND_BLOCK;
    if (t > t1 - 1) t = t1 - 1;
    tile_row[j] = find_row(woff, 0, R - 1, t);
  }
}

// Launch shapes of the expand kernel, fixed at compile time so a launch
// carries only the code (and registers) of the paths its rows can take.
enum : int {
  X_WRITE = 1,  // survivors are appended to the next level table
  X_EMIT = 2,   // complete matches are written as rows (emit mode)
  X_FUSED = 4,  // the last position (one backward slice) is closed in place
  X_TAIL = 8,   // a two-position pendant tail is closed from dense aggregates
  X_ONE = 16,   // one query, no row query ids: its plan is staged in shared memory
};

// Expand kernel: one element (row, driving entry) per thread.
template <int MODE>
__global__ void __launch_bounds__(EXPAND_BLOCK) k_expand(StepArgs a) {
  const uint32_t i = a.level;
  const GraphDev& g = a.g;
  const uint32_t lane = threadIdx.x & 31;
  uint64_t t0 = a.t0, t1 = a.t1;
  if (a.lane) {  // lane pipeline: this level's elements, capped (k_tile_rows_lane flags it)
    t0 = 0;
    t1 = a.ctr[C_LT + i];
    if (t1 > a.seg_cap) t1 = a.seg_cap;
  }
  const uint64_t span = t1 - t0;
  const uint64_t ntiles = (span + EXPAND_BLOCK - 1) / EXPAND_BLOCK;
  unsigned long long cnt = 0, bal = 0, balc = 0, s1 = 0, sk = 0, s2 = 0;
  uint32_t cnt_q = 0;
  // Device work queue: each block takes `grab` consecutive tiles at a time,
  // so a block walks contiguous element ranges (same rows, same query) and a
  // hub row's elements still spread over many blocks.
  __shared__ unsigned long long s_base, s_wbase;
  __shared__ uint32_t s_wcnt[EXPAND_BLOCK / 32];
  // A single query's plan is read by every element: staged once per block,
  // its fields are shared-memory loads with 32-bit addressing.
  __shared__ PlanDev s_plan;
  if constexpr ((MODE & X_ONE) != 0) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.plans);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s_plan);
    for (uint32_t w = threadIdx.x; w < sizeof(PlanDev) / 4; w += EXPAND_BLOCK) dst[w] = src[w];
    __syncthreads();
  }
  // Tiles per grab: about 16 grabs per block over the launch (fewer queue
  // atomics and barriers), at least 4, at most 32.
  uint64_t grab = a.grab;
  if (!grab) {
    grab = ntiles / (uint64_t(gridDim.x) * 16);
    grab = grab < 4 ? 4 : (grab > 32 ? 32 : grab);
  }
  for (;;) {
    if (threadIdx.x == 0) s_base = atomicAdd(&a.ctr[a.tile_slot], (unsigned long long)grab);
    __syncthreads();
    const uint64_t gbase = s_base;
    __syncthreads();
    if (gbase >= ntiles) break;
    const uint64_t gend = min(gbase + grab, ntiles);
    for (uint64_t tile = gbase; tile < gend; ++tile) {
      const uint64_t tb = t0 + tile * EXPAND_BLOCK;
      const uint64_t te = min(tb + EXPAND_BLOCK, t1);
      const uint32_t rlo = __ldg(a.tile_row + tile), rhi = __ldg(a.tile_row + tile + 1);
      const uint64_t t = tb + threadIdx.x;
      const bool valid = t < te;
      bool ok = false, fin = false, fused = false, ftail = false;
      uint32_t r = 0, x = 0, q = 0;
      if (valid) {
        r = find_row(a.woff, rlo, rhi, t);
        const uint32_t e = uint32_t(t - a.woff[r]);
        const uint8_t ci = a.dci[r];
        const uint32_t ds = a.dstart[r];
        const PlanDev* Pp;
        if constexpr ((MODE & X_ONE) != 0) {
          Pp = &s_plan;
        } else {
          q = a.in.qid ? a.in.qid[r] : 0u;
          Pp = a.plans + q;
        }
        const PlanDev& P = *Pp;
        const uint32_t lab = P.label[i];
        uint32_t ddir = 0;
        if (ci == DCI_BUCKET) {
          x = __ldg(g.bucket_vid + ds + (i == 0 ? uint64_t(e) * a.root_step : uint64_t(e)));
        } else {
          ddir = P.cons[i][ci] >> 8;
          x = __ldg(g.adj[ddir] + ds + e);
        }
        ok = true;
        // the lossy matrix filter drops level-0 candidates it rejects
        if (i == 0 && a.root_keep && !((__ldg(a.root_keep + (x >> 5)) >> (x & 31)) & 1u))
          ok = false;
        // injectivity: only earlier positions with the same label can collide
        for (uint32_t m = P.samelab[i]; m && ok; m &= m - 1) {
          const uint32_t j = __ffs(m) - 1;
          if (a.in.col[j][r] == x) ok = false;
        }
        // remaining backward neighbours: binary search in their label slices
        const uint32_t nc = P.ncons[i];
        for (uint32_t c = 0; c < nc && ok; ++c) {
          if (c == ci) continue;
          const uint32_t cs = P.cons[i][c];
          const uint32_t y = a.in.col[cs & 0xFF][r];
          ok = in_slice(g, cs >> 8, y, lab, x, a.probe_min);
        }
        if (ok && ((P.selfloop_mask >> i) & 1u)) ok = has_self(g, x);
        fin = (i + 1 == P.k);
        if constexpr ((MODE & X_FUSED) != 0)
          fused = !fin && a.count_mode && (i + 2 == P.k) && P.last_o1;
        if constexpr ((MODE & X_TAIL) != 0)
          ftail = ((a.tail_dense && P.tail2) || (a.star && P.star2)) && i + 3 == P.k;
        // Filters prune positions whose survivors are extended further; the
        // position before a last position counted in closed form is not
        // filtered (the closed form already yields 0 for hopeless candidates).
        if (ok && !fin && a.filters && !(i + 2 == P.k && P.last_o1))
          ok = pass_filters(g, P, i, x, a.filters);
        if (ok) {
          if (q != cnt_q) {
            acc_flush(a, cnt_q, i, cnt, s1, sk, s2);
            cnt = s1 = sk = s2 = 0;
            cnt_q = q;
          }
          s1 += 1;
          if (fin) {
            if (a.count_mode) cnt += 1;
          } else if ((MODE & X_TAIL) && ftail && P.star2) {
            // The prefix ending in x has length k-2 and the plan ends in two
            // leaves of one anchor: counted here, not stored.
            unsigned long long tc, tp, tb, tbc;
            star_close(a, P, [&](uint32_t j) { return j == i ? x : a.in.col[j][r]; }, tc, tp,
                       tb, tbc);
            cnt += tc;
            sk += tc;
            s2 += tp;
            bal += tb;
            balc += tbc;
          } else if ((MODE & X_TAIL) && ftail) {
            // The prefix ending in x has length k-2: its two-position pendant
            // tail is counted here from the dense aggregates, not stored.
            const uint32_t mp = P.tail_p == i ? x : a.in.col[P.tail_p][r];
            uint32_t ts, te;
            slice_of(g, P.tail_da, mp, P.label[P.k - 2], ts, te);
            long long ac, ad;
            tail_agg(a, P, mp, ts, te, ac, ad);
            unsigned long long tc, tp, td;
            tail_close(a, P, [&](uint32_t j) { return j == i ? x : a.in.col[j][r]; }, mp, ts, te,
                       ac, ad, tc, tp, td);
            cnt += tc;
            sk += tc;
            s2 += tp;
            bal += 8ull + 4ull * (te - ts) + 8ull * tp + 4ull * td;
            balc += 8ull + 4ull * (te - ts) + 8ull * tp;
          } else if ((MODE & X_FUSED) && fused) {
            const uint32_t kl = P.k - 1;
            const uint32_t cs = P.cons[kl][0];
            const uint32_t pos = cs & 0xFF, dir = cs >> 8;
            const uint32_t y = pos == i ? x : a.in.col[pos][r];
            uint32_t s, en;
            slice_of(g, dir, y, P.label[kl], s, en);
            unsigned long long c1 = en - s;
            bal += 8ull + 4ull * c1;
            balc += 8ull;
            for (uint32_t m = P.samelab[kl]; m; m &= m - 1) {
              const uint32_t j = __ffs(m) - 1;
              if ((P.guar[kl] >> j) & 1u) {
                c1 -= 1;
              } else {
                const uint32_t mj = j == i ? x : a.in.col[j][r];
                c1 -= in_slice_se(g, dir, y, s, en, mj, a.probe_min) ? 1ull : 0ull;
              }
            }
            sk += c1;
            cnt += c1;
          }
        }
      }
      // Survivors that extend the prefix: append to the next level table.  One
      // reservation per tile keeps a tile's survivors (one row run, usually one
      // query) contiguous in the next table.
      // Launches without an output table (last or closed-form positions) skip
      // the reservation and its barriers.
      const bool wr = ok && !fin && !fused && !ftail;
      if constexpr ((MODE & X_WRITE) != 0) {
        const uint32_t wm = __ballot_sync(FULL, wr);
        if (lane == 0) s_wcnt[threadIdx.x >> 5] = __popc(wm);
        __syncthreads();
        if (threadIdx.x == 0) {
          uint32_t tot = 0;
          for (uint32_t w = 0; w < EXPAND_BLOCK / 32; ++w) {
            const uint32_t c = s_wcnt[w];
            s_wcnt[w] = tot;
            tot += c;
          }
          s_wbase = tot ? atomicAdd(&a.ctr[a.out_slot], (unsigned long long)tot) : 0ull;
        }
        __syncthreads();
        if (wm) {
          if (wr) {
            const unsigned long long idx = s_wbase + s_wcnt[threadIdx.x >> 5] + __popc(wm & lanemask_lt());
            if (idx < a.out_cap) {
              for (uint32_t j = 0; j < i; ++j) a.out.col[j][idx] = a.in.col[j][r];
              a.out.col[i][idx] = x;
              if (a.out.qid) a.out.qid[idx] = q;
            } else {
              atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_OVERFLOW);
            }
          }
        }
      } else if (wr) {
        atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_OVERFLOW);  // no table to append to
      }
      // Emit mode: complete matches as rows in query-vertex order.
      if constexpr ((MODE & X_EMIT) != 0) {
      const bool em = ok && fin && !a.count_mode;
      const uint32_t emm = __ballot_sync(FULL, em);
      if (emm) {
        const uint32_t leader = __ffs(emm) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(&a.ctr[C_EMIT], (unsigned long long)__popc(emm));
        base = __shfl_sync(FULL, base, leader);
        if (em) {
          const unsigned long long idx = base + __popc(emm & lanemask_lt());
          if (idx < a.emit_cap) {
            const PlanDev& P = (MODE & X_ONE) ? s_plan : a.plans[q];
            for (uint32_t j = 0; j < i; ++j)
              a.emit_col[P.perm[j]][idx] = __ldg(g.globalid + a.in.col[j][r]);
            a.emit_col[P.perm[i]][idx] = __ldg(g.globalid + x);
          } else {
            atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_OVERFLOW);
          }
        }
      }
      }  // X_EMIT
      if constexpr ((MODE & X_WRITE) != 0) __syncthreads();  // s_wcnt / s_wbase reused next tile
    }
    // Once per grab in a batch: fold the per-thread counts of a warp that holds
    // one query (a single query's counts are folded once, at the end).
    if (a.in.qid) acc_flush_warp(a, cnt_q, i, cnt, s1, sk, s2, false);
  }  // grab loop
  acc_flush_warp(a, cnt_q, i, cnt, s1, sk, s2, true);
  bal = warp_sum(bal);
  balc = warp_sum(balc);
  if (lane == 0 && (bal | balc)) {
    atomicAdd(&a.ctr[C_BALG], bal);
    atomicAdd(&a.ctr[C_BALGC], balc);
  }
}

// ---- lane pipeline kernels --------------------------------------------------
// Look-back words of the single-pass work/scan: [epoch:20 | status:2 | value:42].
constexpr int LB_VALUE_BITS = 42;
constexpr unsigned long long LB_AGG = 1, LB_INC = 2;
constexpr int WS_ROWS = 1024;  // rows per work/scan tile (4 per thread)

__device__ __forceinline__ unsigned long long lb_word(uint32_t epoch, unsigned long long st,
                                                      unsigned long long v) {
  return (uint64_t(epoch) << (LB_VALUE_BITS + 2)) | (st << LB_VALUE_BITS) |
         (v & ((1ull << LB_VALUE_BITS) - 1));
}

// Work + scan of one lane level in one pass: tiles of WS_ROWS rows are taken
// in launch order from a counter; each computes its rows' driving slices,
// publishes its sum, and adds the sums of the tiles before it (decoupled
// look-back: a predecessor's inclusive prefix, or its sum and keep looking).
// A tile only ever waits for tiles claimed before it, whose blocks are
// running, and every wait gives up after spin_limit polls (ERR_TIMEOUT).
// The last tile writes the level's element total to woff[R] and C_LT.
__global__ void __launch_bounds__(256) k_work_scan(StepArgs a, uint32_t epoch) {
  const uint32_t i = a.level;
  const uint64_t R = lane_rows(a);
  const uint64_t ntiles = (R + WS_ROWS - 1) / WS_ROWS;
  unsigned long long bal = 0, balc = 0;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_prefix;
  for (;;) {
    if (threadIdx.x == 0) s_tile = uint32_t(atomicAdd(&a.ctr[C_LSCAN + i], 1ull));
    __syncthreads();
    const uint64_t tile = s_tile;
    __syncthreads();
    if (tile >= ntiles) break;
    const uint64_t base = tile * WS_ROWS + uint64_t(threadIdx.x) * 4;
    unsigned long long v[4], sum = 0;
    for (int j = 0; j < 4; ++j) {
      const uint64_t r = base + j;
      v[j] = 0;
      if (r < R) {
        const PlanDev& P = a.plans[0];
        uint32_t bs;
        uint8_t bci;
        unsigned long long ch, chc;
        const uint32_t w = row_work(a, P, r, 0, bs, bci, ch, chc);
        a.work[r] = w;
        a.dstart[r] = bs;
        a.dci[r] = bci;
        bal += ch;
        balc += chc;
        v[j] = w;
        sum += w;
      }
    }
    unsigned long long tot;
    const unsigned long long ex = block_exclusive_scan(sum, &tot);
    if (threadIdx.x == 0) {
      unsigned long long* st = a.scan_status;
      atomicExch(st + tile, lb_word(epoch, tile == 0 ? LB_INC : LB_AGG, tot));
      unsigned long long prefix = 0;
      for (int64_t t = int64_t(tile) - 1; t >= 0; --t) {
        unsigned long long w = 0;
        uint32_t spins = 0;
        for (;;) {
          w = atomicAdd(st + t, 0ull);
          if ((w >> (LB_VALUE_BITS + 2)) == epoch && ((w >> LB_VALUE_BITS) & 3ull)) break;
          if (++spins > a.spin_limit) {
            atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_TIMEOUT);
            w = lb_word(epoch, LB_INC, 0);
            break;
          }
          __nanosleep(64);
        }
        prefix += w & ((1ull << LB_VALUE_BITS) - 1);
        if (((w >> LB_VALUE_BITS) & 3ull) == LB_INC) break;
      }
      if (tile > 0) atomicExch(st + tile, lb_word(epoch, LB_INC, prefix + tot));
      if (prefix + tot >= (1ull << LB_VALUE_BITS))
        atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_OVERFLOW);
      s_prefix = prefix;
      if (tile + 1 == ntiles) {
        a.woff[R] = prefix + tot;
        a.ctr[C_LT + i] = prefix + tot;
      }
    }
    __syncthreads();
    unsigned long long o = s_prefix + ex;
    for (int j = 0; j < 4; ++j) {
      const uint64_t r = base + j;
      if (r < R) a.woff[r] = o;
      o += v[j];
    }
  }
  bal = warp_sum(bal);
  balc = warp_sum(balc);
  if ((threadIdx.x & 31) == 0 && (bal | balc)) {
    atomicAdd(&a.ctr[C_BALG], bal);
    atomicAdd(&a.ctr[C_BALGC], balc);
  }
}

// First row of every expand tile of a lane level (the element total is read
// from the device; a total beyond the lane's tile buffer is flagged and the
// query is re-run on the chunked path).
__global__ void __launch_bounds__(256) k_tile_rows_lane(StepArgs a) {
  const uint64_t R = lane_rows(a);
  uint64_t T = a.ctr[C_LT + a.level];
  if (T > a.seg_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      atomicOr(&a.ctr[C_ERR], (unsigned long long)ERR_OVERFLOW);
    T = a.seg_cap;
  }
  if (T == 0 || R == 0) return;
  const uint64_t ntiles = (T + EXPAND_BLOCK - 1) / EXPAND_BLOCK;
  for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j <= ntiles;
       j += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t t = j * EXPAND_BLOCK;
    if (t > T - 1) t = T - 1;
    const_cast<uint32_t*>(a.tile_row)[j] = find_row(a.woff, 0, uint32_t(R - 1), t);
  }
}

// End of one query on a lane: its count, survivors per prefix length and
// error bits go to the batch arrays (entry q), and the lane's per-query state
// is cleared for the next query.  A query past its element budget reports
// UINT64_MAX.
__global__ void k_lane_done(unsigned long long* ctr, unsigned long long* counts,
                            unsigned long long* lvl, unsigned long long* qel,
                            unsigned long long budget, uint32_t q,
                            unsigned long long* out_counts, unsigned long long* out_lvl,
                            unsigned long long* out_err, unsigned long long* out_balg) {
  const uint32_t t = threadIdx.x;
  if (t <= MAXK) {
    out_lvl[uint64_t(q) * (MAXK + 1) + t] = lvl[t];
    lvl[t] = 0;
  }
  __syncwarp();
  if (t == 0) {
    out_counts[q] = (budget && qel[0] > budget) ? ~0ull : counts[0];
    out_err[q] = ctr[C_ERR];
    out_balg[2ull * q] = ctr[C_BALG];
    out_balg[2ull * q + 1] = ctr[C_BALGC];
    counts[0] = 0;
    qel[0] = 0;
    ctr[C_ERR] = 0;
    ctr[C_BALG] = 0;
    ctr[C_BALGC] = 0;
  }
  for (int c = C_LOUT + int(t); c < C_NUM; c += 32) ctr[c] = 0;
}

__global__ void k_iota(uint32_t* p, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = i;
}

// ---------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------
int build_plan(const DevGraph* dg, const QueryGraph& Q, const uint32_t* order, PlanDev* P) {
  std::memset(P, 0, sizeof(*P));
  const uint32_t k = Q.k;
  P->k = k;
  const bool sym = dg->g.symmetric != 0;
  int clab[MAXK];
  for (uint32_t u = 0; u < k; ++u) clab[u] = dg->stats.compact_label(Q.label_raw[u]);
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t u = order[i];
    P->perm[i] = u;
    if (clab[u] < 0) P->zero = 1;
    P->label[i] = clab[u] < 0 ? 0 : uint32_t(clab[u]);
  }
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t u = order[i];
    uint32_t nc = 0;
    for (uint32_t j = 0; j < i; ++j) {
      const uint32_t w = order[j];
      const bool w_to_u = (Q.out_mask[w] >> u) & 1u;  // u in N_out(w)
      const bool u_to_w = (Q.out_mask[u] >> w) & 1u;  // u in N_in(w)
      if (sym) {
        if (w_to_u || u_to_w) P->cons[i][nc++] = j;
      } else {
        if (w_to_u) P->cons[i][nc++] = j;
        if (u_to_w) P->cons[i][nc++] = j | (1u << 8);
      }
      if (Q.label_raw[w] == Q.label_raw[u]) P->samelab[i] |= 1u << j;
    }
    P->ncons[i] = nc;
    if ((Q.out_mask[u] >> u) & 1u) P->selfloop_mask |= 1u << i;
    uint32_t nb0 = sym ? (Q.out_mask[u] | Q.in_mask[u]) : Q.out_mask[u];
    uint32_t nb1 = Q.in_mask[u];
    P->req[0][i] = __builtin_popcount(nb0);
    P->req[1][i] = sym ? 0 : __builtin_popcount(nb1);
    for (uint32_t w = 0; w < k; ++w) {
      if (clab[w] < 0) continue;
      if ((nb0 >> w) & 1u) P->nlbq[0][i][clab[w] >> 5] |= 1u << (clab[w] & 31);
      if (!sym && ((nb1 >> w) & 1u)) P->nlbq[1][i][clab[w] >> 5] |= 1u << (clab[w] & 31);
    }
  }
  const uint32_t kl = k - 1;
  P->last_o1 = (k >= 2 && P->ncons[kl] == 1 && !((P->selfloop_mask >> kl) & 1u)) ? 1u : 0u;
  if (P->last_o1 && k >= 3 && !P->zero) {
    const uint32_t ia = k - 2;
    const uint32_t cb = P->cons[kl][0], ca = P->cons[ia][0];
    if ((cb & 0xFF) == ia && P->ncons[ia] == 1 && !((P->selfloop_mask >> ia) & 1u)) {
      const uint32_t p = ca & 0xFF, da = ca >> 8, db = cb >> 8;
      uint32_t Ia = 0, J = 0;
      for (uint32_t j = 0; j < ia; ++j) {
        if (P->label[j] == P->label[ia]) Ia |= 1u << j;
        if (P->label[j] == P->label[kl]) J |= 1u << j;
      }
      // every j in J must be p with x in N^{rev db}(m_p) <=> x in N^{da}(m_p)
      const bool ok = J == 0 || (J == (1u << p) && (sym || da != db));
      if (ok) {
        P->tail2 = 1;
        P->tail_p = p;
        P->tail_da = da;
        P->tail_db = db;
        P->tail_Ia = Ia;
        P->tail_J = J;
      }
    }
  }
  if (!P->tail2 && P->last_o1 && k >= 3 && !P->zero) {
    // Two final leaves of one anchor: k-2 and k-1 have the same single
    // backward constraint (position and direction), so they are not adjacent.
    const uint32_t ia = k - 2, cb = P->cons[kl][0];
    if (P->ncons[ia] == 1 && P->cons[ia][0] == cb && (cb & 0xFF) < ia &&
        !((P->selfloop_mask >> ia) & 1u)) {
      P->star2 = 1;
      P->star_p = cb & 0xFF;
      P->star_d = cb >> 8;
    }
  }
  if (P->last_o1) {
    const uint32_t cs = P->cons[kl][0];
    const uint32_t ws = order[cs & 0xFF], dir = cs >> 8;
    for (uint32_t m = P->samelab[kl]; m; m &= m - 1) {
      const uint32_t j = __builtin_ctz(m);
      const uint32_t wj = order[j];
      bool g;
      if (sym) g = ((Q.out_mask[ws] >> wj) & 1u) || ((Q.out_mask[wj] >> ws) & 1u);
      else if (dir == 0) g = (Q.out_mask[ws] >> wj) & 1u;  // m(j) in N_out(m(ws))
      else g = (Q.out_mask[wj] >> ws) & 1u;                // m(j) in N_in(m(ws))
      if (g) P->guar[kl] |= 1u << j;
    }
  }
  return MG_OK;
}

static int choose_order(DevGraph* dg, const QueryGraph& Q, const mg_opts& o, uint32_t* order) {
  switch (o.order) {
    case MG_ORDER_REFERENCE:
      order_reference(Q, order);
      return MG_OK;
    case MG_ORDER_STRONG:
      order_strong(Q, dg->stats, order);
      return MG_OK;
    case MG_ORDER_LEARNED: {
      if (!o.model) {
        order_reference(Q, order);
        return MG_OK;
      }
      int rc = ensure_full_stats(dg);
      if (rc) return rc;
      return order_learned(o.model, Q, dg->stats, order);
    }
    case MG_ORDER_GIVEN:
      if (!o.given_order) return set_error(MG_E_ARG, "MG_ORDER_GIVEN without given_order");
      std::memcpy(order, o.given_order, Q.k * 4);
      if (!order_is_permutation(order, Q.k))
        return set_error(MG_E_ARG, "given_order is not a permutation of 0..%u", Q.k - 1);
      return MG_OK;
    default:
      return set_error(MG_E_ARG, "unknown order %d", o.order);
  }
}

// ---------------------------------------------------------------------------
// Host driver: depth-first walk over level chunks
// ---------------------------------------------------------------------------
struct EmitBuf {
  uint32_t* col[MAXK] = {};
  uint64_t cap = 0;
};

struct RunResult {
  uint64_t balg = 0, balgc = 0, launches = 0, chunks = 0, elements = 0, expand_launches = 0;
  uint64_t reruns = 0;  // batch queries counted again on the chunked path
  double expand_ms = 0;
  uint64_t surv[MAXK + 2] = {};
  uint64_t emitted = 0;
  double ms = 0;
};

static inline unsigned grid_for(uint64_t items, unsigned block, unsigned cap) {
  uint64_t g = (items + block - 1) / block;
  return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(g, cap)));
}

// Launches the expand kernel specialised for what the rows of level `lvl`
// can need: a write when the level writes a table, emit rows in emit mode,
// in-place closing of a last position or of a pendant tail when a plan has
// one right after this position.
static void launch_expand(const StepArgs& a, const PlanDev* plans, uint32_t nplans,
                          bool count_mode, bool writes, unsigned grid, cudaStream_t st) {
  const uint32_t i = a.level;
  bool fused = false, tail = false, emit = false;
  for (uint32_t pi = 0; pi < nplans; ++pi) {
    const PlanDev& p = plans[pi];
    if (count_mode && p.k == i + 2 && p.last_o1) fused = true;
    if (((a.tail_dense && p.tail2) || (a.star && p.star2)) && p.k == i + 3) tail = true;
    if (!count_mode && p.k == i + 1) emit = true;
  }
  const bool one = nplans == 1 && a.in.qid == nullptr;
  const int mode = (writes ? X_WRITE : 0) | (emit ? X_EMIT : 0) | (fused ? X_FUSED : 0) |
                   (tail ? X_TAIL : 0) | (one ? X_ONE : 0);
  switch (mode) {
#define MG_X(m) \
  case m:       \
    k_expand<m><<<grid, EXPAND_BLOCK, 0, st>>>(a); \
    break;
    MG_X(0) MG_X(1) MG_X(2) MG_X(3) MG_X(4) MG_X(5) MG_X(6) MG_X(7)
    MG_X(8) MG_X(9) MG_X(10) MG_X(11) MG_X(12) MG_X(13) MG_X(14) MG_X(15)
    MG_X(16) MG_X(17) MG_X(18) MG_X(19) MG_X(20) MG_X(21) MG_X(22) MG_X(23)
    MG_X(24) MG_X(25) MG_X(26) MG_X(27) MG_X(28) MG_X(29) MG_X(30) MG_X(31)
#undef MG_X
  }
}

// Tail keys (da, la, db, lb, lp) of the plans that end in a two-position
// pendant tail, their hub aggregate tables (one entry per hub of direction
// da; all keys of a call share one array of at most 2^27 entries), their lazy
// tables over the bucket of l_p (cleared here; at most 2^30 entries in all)
// and the tail fields of `a`.  A key past either limit sums in place.
template <class Alloc>
static int setup_tails(DevGraph* dg, std::vector<PlanDev>& plans, TailStore& ts, Alloc alloc,
                       cudaStream_t st, StepArgs* a, uint64_t* launches) {
  std::vector<TailKey> keys;
  uint64_t entries = 0, lazy = 0;
  for (PlanDev& p : plans) {
    if (!p.tail2) continue;
    TailKey tk{p.tail_da, p.label[p.k - 2], p.tail_db, p.label[p.k - 1], p.label[p.tail_p], 0, 0,
               0};
    uint32_t kid = 0;
    while (kid < keys.size() && std::memcmp(&keys[kid], &tk, 20) != 0) ++kid;
    if (kid == keys.size()) {
      const uint64_t nh = dg->g.n_hubs[tk.da];
      tk.base = (nh && entries + nh <= (1ull << 27)) ? entries : ~0ull;
      if (tk.base != ~0ull) entries += nh;
      const uint64_t nb = dg->h_bucket_off[tk.lp + 1] - dg->h_bucket_off[tk.lp];
      tk.lazy = (lazy + nb <= (1ull << 30)) ? lazy : ~0ull;
      if (tk.lazy != ~0ull) lazy += nb;
      keys.push_back(tk);
    }
    p.tail_kid = kid;
  }
  if (keys.empty()) return MG_OK;
  int rc;
  if (ts.cap < entries) {
    if ((rc = alloc((void**)&ts.A, entries * 8))) return rc;
    if ((rc = alloc((void**)&ts.AD, entries * 8))) return rc;
    ts.cap = entries;
  }
  if (ts.lazy_cap < lazy) {
    if ((rc = alloc((void**)&ts.lazy, lazy * 8))) return rc;
    ts.lazy_cap = lazy;
  }
  if (lazy) MG_CK(cudaMemsetAsync(ts.lazy, 0xFF, lazy * 8, st));
  if (ts.keys_cap < keys.size()) {
    if ((rc = alloc((void**)&ts.keys, keys.size() * sizeof(TailKey)))) return rc;
    ts.keys_cap = uint32_t(keys.size());
  }
  MG_CK(cudaMemcpyAsync(ts.keys, keys.data(), keys.size() * sizeof(TailKey),
                        cudaMemcpyHostToDevice, st));
  for (const TailKey& tk : keys) {
    if (tk.base == ~0ull) continue;
    k_tail_dense<<<grid_for(uint64_t(dg->g.n_hubs[tk.da]) * 32, 256, dg->sms * 16), 256, 0, st>>>(
        dg->g, tk, ts.A, ts.AD);
    ++*launches;
  }
  MG_CK(cudaGetLastError());
  a->tail_dense = 1;
  a->tdA = ts.A;
  a->tdAD = ts.AD;
  a->tdL = ts.lazy;
  a->tkeys = ts.keys;
  return MG_OK;
}

static int run_levels(DevGraph* dg, std::vector<PlanDev> plans, bool count_mode,
                      const EmitBuf* emit, const mg_opts& o, uint64_t* counts_out,
                      RunResult* res, uint64_t* lvl_rows_out = nullptr) {
  const uint32_t nq = uint32_t(plans.size());
  uint32_t kmax = 1;
  for (auto& p : plans) kmax = std::max(kmax, p.k);
  // Default rows per level chunk: scaled with the graph so small graphs do
  // not reserve gigabytes of scratch; chunking keeps larger results exact.
  uint64_t auto_cap = 1ull << 16;
  while (auto_cap < kDefaultCap && auto_cap < 4 * (uint64_t(dg->g.n) + dg->info.m_out))
    auto_cap <<= 1;
  uint64_t cap = o.chunk_rows ? o.chunk_rows : auto_cap;
  cap = std::max<uint64_t>(cap, 1);
  if (cap > (1ull << 31)) return set_error(MG_E_ARG, "chunk_rows above 2^31");
  if (o.mem_budget_bytes) {
    uint64_t per_row = 0;
    for (uint32_t l = 1; l < kmax; ++l) per_row += level_row_bytes(int(l));
    if (per_row && cap * per_row > o.mem_budget_bytes) {
      cap = o.mem_budget_bytes / per_row;
      if (cap == 0) return set_error(MG_E_OOM, "memory budget below one row per level");
    }
  }
  int rc = ensure_ws(dg, cap, int(kmax), nq);
  if (rc) return rc;
  Workspace* ws = dg->ws;
  cudaStream_t st = dg->stream;
  MG_CK(cudaMemcpyAsync(ws->plans, plans.data(), nq * sizeof(PlanDev), cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemsetAsync(ws->counts, 0, nq * 8ull, st));
  MG_CK(cudaMemsetAsync(ws->lvl_rows, 0, uint64_t(nq) * (MAXK + 1) * 8, st));
  MG_CK(cudaMemsetAsync(ws->q_elems, 0, uint64_t(nq) * 8, st));
  MG_CK(cudaMemsetAsync(ws->ctr, 0, C_NUM * 8, st));
  MG_CK(cudaEventRecord(ws->ev0, st));


  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = dg->g;
  a.plans = ws->plans;
  a.ctr = ws->ctr;
  a.counts = ws->counts;
  a.lvl_rows = ws->lvl_rows;
  a.q_elems = ws->q_elems;
  a.q_budget = nq > 1 ? o.max_elements : 0;  // batch: per-query budget
  a.count_mode = count_mode ? 1u : 0u;
  a.filters = o.filters & MG_FILTER_ALL;
  a.grab = o.grab;
  a.stats = nq == 1 ? 1u : 0u;
  a.nq = nq;
  if (emit) {
    for (int j = 0; j < MAXK; ++j) a.emit_col[j] = emit->col[j];
    a.emit_cap = emit->cap;
  }
  a.root_step = o.root_step > 1 ? o.root_step : 1u;
  a.probe_min = o.probe_min ? o.probe_min : kProbeMin;
  a.out_slot = C_OUT;
  a.tile_slot = C_TILE;
  if (o.root_end || a.root_step > 1) {
    a.root_begin = o.root_begin;
    a.root_end = o.root_end ? o.root_end : ~0ull;
  }
  const bool batch = nq > 1;
  if (batch) {
    k_iota<<<grid_for(nq, 256, 1024), 256, 0, st>>>(ws->qid[0], nq);
    res->launches++;
  }
  if (o.matrix_filter && !batch && !plans[0].zero) {
    const uint64_t words = (uint64_t(dg->g.n) + 31) / 32;
    if (ws->root_keep_words < words) {
      if ((rc = ws_alloc(ws, (void**)&ws->root_keep, words * 4))) return rc;
      ws->root_keep_words = words;
    }
    if ((rc = matrix_filter_roots(o.matrix_filter, dg, plans[0].perm[0], plans[0].label[0],
                                  ws->root_keep, st)))
      return rc;
    a.root_keep = ws->root_keep;
    res->launches++;
  }
  uint64_t T[MAXK] = {}, cur[MAXK] = {};
  uint32_t R[MAXK] = {};
  R[0] = nq;
  int lvl = 0;
  bool need_work = true;
  const unsigned sms = dg->sms;
  uint64_t elements = 0;

  // Pendant tails counted in closed form (count mode): tail-key table and
  // memo table of two-hop aggregates, shared by every query of the call.
  bool dense = false;
  if (count_mode && o.no_tail != 1) {
    rc = setup_tails(dg, plans, ws->tails,
                     [&](void** p, size_t bytes) { return ws_alloc(ws, p, bytes); }, st, &a,
                     &res->launches);
    if (rc) return rc;
    dense = a.tail_dense != 0;
    if (dense)
      MG_CK(cudaMemcpyAsync(ws->plans, plans.data(), nq * sizeof(PlanDev),
                            cudaMemcpyHostToDevice, st));
  }
  a.star = count_mode && o.no_tail != 1;
  // writes[l]: some query can append rows to the level-(l+1) table.
  bool writes[MAXK] = {};
  for (uint32_t l = 0; l < kmax; ++l)
    for (auto& p : plans)
      if (p.k > l + 1 && !(count_mode && p.k == l + 2 && p.last_o1) &&
          !(dense && p.tail2 && p.k == l + 3) && !(a.star && p.star2 && p.k == l + 3))
        writes[l] = true;

  auto launch_work_scan = [&](int l) -> int {
    k_work<<<grid_for(R[l], 256, sms * 16), 256, 0, st>>>(a);
    const uint32_t nb = (R[l] + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_reduce<<<nb, 256, 0, st>>>(ws->work[l], R[l], ws->bsum);
    k_scan_bsum<<<1, 1024, 0, st>>>(ws->bsum, nb, ws->woff[l] + R[l]);
    k_scan_apply<<<nb, 256, 0, st>>>(ws->work[l], R[l], ws->bsum, ws->woff[l]);
    res->launches += 4;
    MG_CK(cudaMemcpyAsync(&ws->h_ctr[0], ws->woff[l] + R[l], 8, cudaMemcpyDeviceToHost, st));
    MG_CK(cudaStreamSynchronize(st));
    return MG_OK;
  };
  auto tab = [&](int l) {
    TabPtrs t{};
    for (int j = 0; j < l; ++j) t.col[j] = ws->col[l][j];
    t.qid = batch ? ws->qid[l] : nullptr;
    return t;
  };
  while (true) {
    if (need_work) {
      a.level = uint32_t(lvl);
      a.R = R[lvl];
      a.in = tab(lvl);
      a.work = ws->work[lvl];
      a.woff = ws->woff[lvl];
      a.dstart = ws->dstart[lvl];
      a.dci = ws->dci[lvl];
      if ((rc = launch_work_scan(lvl))) return rc;
      T[lvl] = ws->h_ctr[0];
      cur[lvl] = 0;
      need_work = false;
    }
    if (cur[lvl] < T[lvl]) {
      const uint64_t t0 = cur[lvl];
      const uint64_t t1 = writes[lvl] ? std::min(T[lvl], t0 + cap) : T[lvl];
      elements += t1 - t0;
      if (nq == 1 && o.max_elements && elements > o.max_elements) {
        cudaStreamSynchronize(st);
        return set_error(MG_E_LIMIT, "work budget of %llu candidate elements exceeded",
                         (unsigned long long)o.max_elements);
      }
      a.tile_row = ws->tile_row;
      a.level = uint32_t(lvl);
      a.R = R[lvl];
      a.in = tab(lvl);
      a.work = ws->work[lvl];
      a.woff = ws->woff[lvl];
      a.dstart = ws->dstart[lvl];
      a.dci = ws->dci[lvl];
      a.t0 = t0;
      a.t1 = t1;
      if (writes[lvl]) {
        a.out = tab(lvl + 1);
        a.out_cap = cap;
      } else {
        a.out = TabPtrs{};
        a.out_cap = 0;
      }
      MG_CK(cudaMemsetAsync(ws->ctr + C_OUT, 0, 8, st));
      for (uint64_t s0 = t0; s0 < t1; s0 += kSegment) {
        const uint64_t s1 = std::min(t1, s0 + kSegment);
        const uint32_t ntiles = uint32_t((s1 - s0 + EXPAND_BLOCK - 1) / EXPAND_BLOCK);
        a.t0 = s0;
        a.t1 = s1;
        k_tile_rows<<<grid_for(uint64_t(ntiles) + 1, 256, sms * 16), 256, 0, st>>>(
            ws->woff[lvl], R[lvl], s0, s1, ntiles, ws->tile_row);
        MG_CK(cudaMemsetAsync(ws->ctr + C_TILE, 0, 8, st));
        if (o.kernel_events) MG_CK(cudaEventRecord(ws->ev2, st));
        launch_expand(a, plans.data(), nq, count_mode, writes[lvl],
                      grid_for(s1 - s0, EXPAND_BLOCK, sms * 8), st);
        if (o.kernel_events) {
          MG_CK(cudaEventRecord(ws->ev3, st));
          MG_CK(cudaEventSynchronize(ws->ev3));
          float kms = 0;
          MG_CK(cudaEventElapsedTime(&kms, ws->ev2, ws->ev3));
          res->expand_ms += kms;
        }
        res->expand_launches++;
        res->launches += 2;
      }
      res->chunks++;
      MG_CK(cudaGetLastError());
      cur[lvl] = t1;
      if (writes[lvl]) {
        MG_CK(cudaMemcpyAsync(&ws->h_ctr[0], ws->ctr + C_OUT, 8, cudaMemcpyDeviceToHost, st));
        MG_CK(cudaStreamSynchronize(st));
        const uint64_t rows = ws->h_ctr[0];
        if (rows > cap) return set_error(MG_E_CUDA, "level table overflow (%llu > %llu)",
                                         (unsigned long long)rows, (unsigned long long)cap);
        if (rows > 0) {
          R[lvl + 1] = uint32_t(rows);
          ++lvl;
          need_work = true;
        }
      }
    } else {
      if (lvl == 0) break;
      --lvl;
    }
  }
  MG_CK(cudaEventRecord(ws->ev1, st));
  MG_CK(cudaMemcpyAsync(ws->h_ctr, ws->ctr, C_NUM * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(counts_out, ws->counts, nq * 8ull, cudaMemcpyDeviceToHost, st));
  if (lvl_rows_out)
    MG_CK(cudaMemcpyAsync(lvl_rows_out, ws->lvl_rows, uint64_t(nq) * (MAXK + 1) * 8,
                          cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(res->surv, ws->lvl_rows, (MAXK + 1) * 8, cudaMemcpyDeviceToHost, st));
  std::vector<unsigned long long> qel;
  if (a.q_budget) {
    qel.resize(nq);
    MG_CK(cudaMemcpyAsync(qel.data(), ws->q_elems, uint64_t(nq) * 8, cudaMemcpyDeviceToHost, st));
  }
  MG_CK(cudaStreamSynchronize(st));
  MG_CK(cudaGetLastError());
  float ms = 0;
  MG_CK(cudaEventElapsedTime(&ms, ws->ev0, ws->ev1));
  res->ms = ms;
  res->elements = elements;
  for (uint32_t q = 0; q < qel.size(); ++q)
    if (qel[q] > a.q_budget) counts_out[q] = ~0ull;  // over budget: unknown
  res->balg = ws->h_ctr[C_BALG];
  res->balgc = ws->h_ctr[C_BALGC];
  res->emitted = ws->h_ctr[C_EMIT];
  if (ws->h_ctr[C_ERR] & ERR_OVERFLOW) return set_error(MG_E_CUDA, "device table overflow");
  return MG_OK;
}

// ---- emit: lexicographic sort of rows (LSD over columns) ------------------
__global__ void k_gather(const uint32_t* __restrict__ src, const uint32_t* __restrict__ perm,
                         uint32_t* dst, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = src[perm[i]];
}

__global__ void k_rows_out(uint32_t* const* cols, const uint32_t* __restrict__ perm, uint32_t k,
                           uint32_t* rows, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n * k;
       i += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t r = i / k;
    uint32_t c = uint32_t(i - r * k);
    rows[i] = cols[c][perm[r]];
  }
}

// ---- emit: stable LSD radix sort of (key, index) pairs ----------------------
// One pass sorts by one 8-bit digit of the 32-bit keys:
//   k_rs_hist    per-tile digit counts, stored digit-major (count[d * nt + t]);
//   scan         exclusive offsets over that digit-major order (k_scan_*);
//   k_rs_scatter each tile re-reads its keys in order and writes key and index
//                to offset[d * nt + t] + (earlier keys of the tile with digit d).
// Four passes order the keys; rows are sorted column by column from the last
// one, and stability keeps earlier passes' order among equal keys.
constexpr int RS_TILE = 2048;        // keys per tile (8 rounds of 256)
constexpr int RS_BLOCK = 256;

__global__ void __launch_bounds__(RS_BLOCK) k_rs_hist(const uint32_t* __restrict__ keys,
                                                     uint64_t n, uint32_t shift, uint32_t nt,
                                                     uint32_t* counts) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = uint64_t(blockIdx.x) * RS_TILE;
  for (uint32_t j = threadIdx.x; j < RS_TILE; j += RS_BLOCK) {
    const uint64_t i = base + j;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[uint64_t(threadIdx.x) * nt + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_BLOCK) k_rs_scatter(const uint32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vals,
                                                        uint64_t n, uint32_t shift, uint32_t nt,
                                                        const uint64_t* __restrict__ offs,
                                                        uint32_t* keys_out, uint32_t* vals_out) {
  __shared__ uint32_t run[256];               // keys of each digit placed so far
  __shared__ uint32_t wc[RS_BLOCK / 32][256];  // this round: keys of each digit per warp
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = 0;
  for (int w = 0; w < RS_BLOCK / 32; ++w) wc[w][threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = uint64_t(blockIdx.x) * RS_TILE;
  for (uint32_t r0 = 0; r0 < RS_TILE; r0 += RS_BLOCK) {
    const uint64_t i = base + r0 + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0u;
    const uint32_t d = (key >> shift) & 255u;
    // lanes of this warp holding the same digit, in lane (= input) order
    const uint32_t peers = __match_any_sync(FULL, valid ? d : 256u + lane);
    const uint32_t below = __popc(peers & lanemask_lt());
    if (valid && below == 0) wc[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pos = run[d] + below;
      for (uint32_t w = 0; w < warp; ++w) pos += wc[w][d];
      const uint64_t o = offs[uint64_t(d) * nt + blockIdx.x] + pos;
      keys_out[o] = key;
      vals_out[o] = vals[i];
    }
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < RS_BLOCK / 32; ++w) {
      add += wc[w][threadIdx.x];
      wc[w][threadIdx.x] = 0;
    }
    run[threadIdx.x] += add;
    __syncthreads();
  }
}

static int sort_and_copy(DevGraph* dg, const EmitBuf& eb, uint32_t k, uint64_t n, uint32_t* h_rows,
                         uint64_t n_copy) {
  cudaStream_t st = dg->stream;
  if (n == 0 || n_copy == 0) return MG_OK;
  const uint32_t nt = uint32_t((n + RS_TILE - 1) / RS_TILE);
  const uint64_t nc = uint64_t(nt) * 256;  // digit-major counts of one pass
  if (nc >= (1ull << 32)) return set_error(MG_E_LIMIT, "emit sort of %llu rows", (unsigned long long)n);
  uint32_t *perm_a, *perm_b, *keys_a, *keys_b, *cnt;
  uint64_t *offs, *bsum;
  MG_CK(cudaMallocAsync((void**)&perm_a, n * 4, st));
  MG_CK(cudaMallocAsync((void**)&perm_b, n * 4, st));
  MG_CK(cudaMallocAsync((void**)&keys_a, n * 4, st));
  MG_CK(cudaMallocAsync((void**)&keys_b, n * 4, st));
  MG_CK(cudaMallocAsync((void**)&cnt, nc * 4, st));
  MG_CK(cudaMallocAsync((void**)&offs, (nc + 1) * 8, st));
  const uint32_t nb = uint32_t((nc + SCAN_TILE - 1) / SCAN_TILE);
  MG_CK(cudaMallocAsync((void**)&bsum, (uint64_t(nb) + 1) * 8, st));
  k_iota<<<grid_for(n, 256, 4096), 256, 0, st>>>(perm_a, uint32_t(n));
  for (int c = int(k) - 1; c >= 0; --c) {
    k_gather<<<grid_for(n, 256, 4096), 256, 0, st>>>(eb.col[c], perm_a, keys_a, n);
    for (uint32_t shift = 0; shift < 32; shift += 8) {
      k_rs_hist<<<nt, RS_BLOCK, 0, st>>>(keys_a, n, shift, nt, cnt);
      k_scan_reduce<<<nb, 256, 0, st>>>(cnt, uint32_t(nc), bsum);
      k_scan_bsum<<<1, 1024, 0, st>>>(bsum, nb, offs + nc);
      k_scan_apply<<<nb, 256, 0, st>>>(cnt, uint32_t(nc), bsum, offs);
      k_rs_scatter<<<nt, RS_BLOCK, 0, st>>>(keys_a, perm_a, n, shift, nt, offs, keys_b, perm_b);
      std::swap(keys_a, keys_b);
      std::swap(perm_a, perm_b);
    }
  }
  MG_CK(cudaGetLastError());
  uint32_t** d_cols;
  MG_CK(cudaMallocAsync((void**)&d_cols, sizeof(uint32_t*) * MAXK, st));
  MG_CK(cudaMemcpyAsync(d_cols, eb.col, sizeof(uint32_t*) * MAXK, cudaMemcpyHostToDevice, st));
  uint32_t* d_rows;
  MG_CK(cudaMallocAsync((void**)&d_rows, n_copy * k * 4, st));
  k_rows_out<<<grid_for(n_copy * k, 256, 4096), 256, 0, st>>>(d_cols, perm_a, k, d_rows, n_copy);
  MG_CK(cudaMemcpyAsync(h_rows, d_rows, n_copy * k * 4, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  for (void* p : {(void*)perm_a, (void*)perm_b, (void*)keys_a, (void*)keys_b, (void*)cnt,
                  (void*)offs, (void*)bsum, (void*)d_cols, (void*)d_rows})
    cudaFreeAsync(p, st);
  MG_CK(cudaStreamSynchronize(st));
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Entry-point bodies
// ---------------------------------------------------------------------------
static mg_opts resolve_opts(const mg_opts* o) {
  mg_opts r;
  mg_opts_default(&r);
  if (o) r = *o;
  return r;
}

// Checks that do not depend on the query or the graph.
static int check_opts(const mg_opts& o) {
  if (o.root_end && o.root_begin > o.root_end)
    return set_error(MG_E_ARG, "root_begin > root_end");
  return MG_OK;
}

static void fill_stats(mg_stats* st, const PlanDev& P, const RunResult& res, uint64_t count) {
  if (!st) return;
  std::memset(st, 0, sizeof(*st));
  st->k = P.k;
  for (uint32_t i = 0; i < P.k; ++i) st->order[i] = P.perm[i];
  for (uint32_t i = 1; i <= P.k && i <= MAXK; ++i) st->level_rows[i] = res.surv[i];
  st->level_rows[P.k] = count;
  st->balg_bytes = res.balg;
  st->balg_count_bytes = res.balgc;
  st->device_ms = res.ms;
  st->launches = res.launches;
  st->chunks = res.chunks;
  st->elements = res.elements;
  st->expand_ms = res.expand_ms;
  st->expand_launches = res.expand_launches;
}

static int prepare(DevGraph* dg, const mg_csr_view* q, const mg_opts& o, PlanDev* P) {
  int rc = check_opts(o);
  if (rc) return rc;
  QueryGraph Q;
  rc = normalise_query(q, &Q);
  if (rc) return rc;
  uint32_t order[MAXK];
  if ((rc = choose_order(dg, Q, o, order))) return rc;
  return build_plan(dg, Q, order, P);
}

int subiso_count(DevGraph* dg, const mg_csr_view* q, const mg_opts* opts, uint64_t* count,
                 mg_stats* st) {
  const mg_opts o = resolve_opts(opts);
  PlanDev P;
  int rc = prepare(dg, q, o, &P);
  if (rc) return rc;
  std::vector<PlanDev> plans(1, P);
  RunResult res;
  uint64_t c = 0;
  if ((rc = run_levels(dg, plans, true, nullptr, o, &c, &res))) return rc;
  *count = c;
  fill_stats(st, P, res, c);
  return MG_OK;
}

int subiso_emit(DevGraph* dg, const mg_csr_view* q, const mg_opts* opts, uint32_t* rows,
                uint64_t cap_rows, uint64_t* n_rows, mg_stats* st) {
  const mg_opts o = resolve_opts(opts);
  PlanDev P;
  int rc = prepare(dg, q, o, &P);
  if (rc) return rc;
  std::vector<PlanDev> plans(1, P);
  RunResult res;
  uint64_t c = 0;
  if ((rc = run_levels(dg, plans, true, nullptr, o, &c, &res))) return rc;
  *n_rows = c;
  if (c >= (1ull << 31))
    return set_error(MG_E_LIMIT, "%llu matches: emit supports fewer than 2^31 rows",
                     (unsigned long long)c);
  EmitBuf eb;
  eb.cap = c;
  cudaStream_t s = dg->stream;
  for (uint32_t j = 0; j < P.k; ++j)
    MG_CK(cudaMallocAsync((void**)&eb.col[j], std::max<uint64_t>(c, 1) * 4, s));
  RunResult res2;
  uint64_t c2 = 0;
  rc = run_levels(dg, plans, false, &eb, o, &c2, &res2);
  if (rc == MG_OK && res2.emitted != c)
    rc = set_error(MG_E_CUDA, "emit pass produced %llu rows, count pass %llu",
                   (unsigned long long)res2.emitted, (unsigned long long)c);
  if (rc == MG_OK) rc = sort_and_copy(dg, eb, P.k, c, rows, std::min(c, cap_rows));
  for (uint32_t j = 0; j < P.k; ++j) cudaFreeAsync(eb.col[j], s);
  cudaStreamSynchronize(s);
  if (rc) return rc;
  res2.balg = res.balg;
  res2.balgc = res.balgc;
  fill_stats(st, P, res2, c);
  if (st) st->device_ms = res.ms + res2.ms;
  if (c > cap_rows)
    return set_error(MG_E_CAPACITY, "%llu matches, %llu rows written",
                     (unsigned long long)c, (unsigned long long)cap_rows);
  return MG_OK;
}

// ---------------------------------------------------------------------------
// Batch lane pipeline
//
// Each query of a batch runs as a fixed sequence of launches (per level: the
// single-pass work/scan, the tile-row lookup, the expand) whose kernels read
// every size from device counters, so nothing returns to the host between
// levels or between queries.  Queries are dealt round-robin to `lanes`
// streams that run concurrently; each lane owns level tables of `cap` rows.
// The host waits once per batch; a query whose rows or elements did not fit
// its lane (ERR_OVERFLOW) is counted again on the chunked path, which has no
// size limit.
// ---------------------------------------------------------------------------
struct Lane {
  cudaStream_t st = nullptr;
  unsigned long long *ctr = nullptr, *counts = nullptr, *lvl = nullptr, *qel = nullptr;
  unsigned long long* status = nullptr;  // look-back words of the work/scan kernel
  uint32_t* tile_row = nullptr;
  uint32_t* col[MAXK][MAXK] = {};
  uint32_t* work[MAXK] = {};
  uint64_t* woff[MAXK] = {};
  uint32_t* dstart[MAXK] = {};
  uint8_t* dci[MAXK] = {};
  uint32_t epoch = 0;
};

struct LaneSet {
  uint64_t cap = 0, seg_cap = 0;
  uint32_t kmax = 0;
  std::vector<Lane> lanes;
  std::vector<void*> allocs;
  unsigned long long *r_counts = nullptr, *r_lvl = nullptr, *r_err = nullptr, *r_balg = nullptr;
  uint32_t r_cap = 0;
  PlanDev* plans = nullptr;
  uint32_t plans_cap = 0;
  TailStore tails;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
};

constexpr uint64_t kLaneCap = 1ull << 20;     // rows per lane level table
constexpr uint64_t kLaneSegment = 1ull << 26; // elements per lane expand launch
constexpr uint32_t kLanes = 8;
constexpr uint32_t kSpinLimit = 1u << 22;     // polls of a look-back wait (~0.3 s)
constexpr uint32_t kEpochMax = (1u << 20) - 1;

void free_lanes(LaneSet* ls) {
  if (!ls) return;
  for (Lane& l : ls->lanes)
    if (l.st) cudaStreamDestroy(l.st);
  for (void* p : ls->allocs) cudaFree(p);
  if (ls->ev_start) cudaEventDestroy(ls->ev_start);
  if (ls->ev_end) cudaEventDestroy(ls->ev_end);
  delete ls;
}

static int lane_alloc(LaneSet* ls, void** p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_error(MG_E_OOM, "lane scratch: cudaMalloc(%zu) failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  ls->allocs.push_back(*p);
  return MG_OK;
}

static int ensure_lanes(DevGraph* dg, uint32_t nl, uint64_t cap, uint32_t kmax) {
  LaneSet*& ls = dg->lanes;
  if (ls && (ls->lanes.size() != nl || ls->cap != cap || ls->kmax < kmax)) {
    cudaDeviceSynchronize();
    free_lanes(ls);
    ls = nullptr;
  }
  if (ls) return MG_OK;
  ls = new LaneSet();
  ls->cap = cap;
  ls->seg_cap = kLaneSegment;
  ls->kmax = std::max<uint32_t>(kmax, 8);
  MG_CK(cudaEventCreateWithFlags(&ls->ev_start, cudaEventDisableTiming));
  MG_CK(cudaEventCreateWithFlags(&ls->ev_end, cudaEventDisableTiming));
  ls->lanes.resize(nl);
  int rc;
  for (Lane& L : ls->lanes) {
    MG_CK(cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking));
    if ((rc = lane_alloc(ls, (void**)&L.ctr, C_NUM * 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&L.counts, 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&L.lvl, (MAXK + 1) * 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&L.qel, 8))) return rc;
    const uint64_t ntiles = cap / WS_ROWS + 2;
    if ((rc = lane_alloc(ls, (void**)&L.status, ntiles * 8))) return rc;
    MG_CK(cudaMemset(L.status, 0, ntiles * 8));
    if ((rc = lane_alloc(ls, (void**)&L.tile_row, (ls->seg_cap / EXPAND_BLOCK + 2) * 4))) return rc;
    for (uint32_t l = 0; l < ls->kmax; ++l) {
      const uint64_t rows = l == 0 ? 1 : cap;
      for (uint32_t j = 0; j < l; ++j)
        if ((rc = lane_alloc(ls, (void**)&L.col[l][j], rows * 4))) return rc;
      if ((rc = lane_alloc(ls, (void**)&L.work[l], rows * 4))) return rc;
      if ((rc = lane_alloc(ls, (void**)&L.woff[l], (rows + 1) * 8))) return rc;
      if ((rc = lane_alloc(ls, (void**)&L.dstart[l], rows * 4))) return rc;
      if ((rc = lane_alloc(ls, (void**)&L.dci[l], rows))) return rc;
    }
  }
  return MG_OK;
}

// Last level a plan expands in count mode: k-1, or k-2 when the last
// position is closed in place, or k-3 when a pendant tail is closed from
// dense aggregates.
static int last_level(const PlanDev& P, bool dense, bool star) {
  int l = int(P.k) - 1;
  if (P.k >= 2 && P.last_o1) l = int(P.k) - 2;
  if ((dense && P.tail2) || (star && P.star2)) l = int(P.k) - 3;
  return l;
}

static int subiso_batch_lanes(DevGraph* dg, std::vector<PlanDev>& plans, const mg_opts& o,
                              uint64_t* counts_out, uint64_t* level_rows_out, RunResult* res) {
  const uint32_t nq = uint32_t(plans.size());
  uint32_t kmax = 1;
  for (auto& p : plans) kmax = std::max(kmax, p.k);
  const uint32_t nl = o.lanes ? o.lanes : kLanes;
  if (nl > 64) return set_error(MG_E_ARG, "lanes=%u: at most 64", nl);
  uint64_t cap = o.chunk_rows ? o.chunk_rows : kLaneCap;
  if (cap > (1ull << 31)) return set_error(MG_E_ARG, "chunk_rows above 2^31");
  int rc = ensure_lanes(dg, nl, cap, kmax);
  if (rc) return rc;
  LaneSet* ls = dg->lanes;
  cudaStream_t st = dg->stream;
  const unsigned sms = dg->sms;

  if (ls->plans_cap < nq) {
    if ((rc = lane_alloc(ls, (void**)&ls->plans, uint64_t(nq) * sizeof(PlanDev)))) return rc;
    ls->plans_cap = nq;
  }
  if (ls->r_cap < nq) {
    if ((rc = lane_alloc(ls, (void**)&ls->r_counts, uint64_t(nq) * 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&ls->r_lvl, uint64_t(nq) * (MAXK + 1) * 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&ls->r_err, uint64_t(nq) * 8))) return rc;
    if ((rc = lane_alloc(ls, (void**)&ls->r_balg, uint64_t(nq) * 16))) return rc;
    ls->r_cap = nq;
  }
  Workspace* ws = dg->ws;  // timing events live with the graph's workspace
  if (!ws && (rc = ensure_ws(dg, 1ull << 16, 1, 1))) return rc;
  ws = dg->ws;
  MG_CK(cudaEventRecord(ws->ev0, st));
  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  // Pendant tails closed from hub aggregates (their table is filled on the
  // graph's stream before the lanes start).
  if (o.no_tail != 1) {
    rc = setup_tails(dg, plans, ls->tails,
                     [&](void** p, size_t bytes) { return lane_alloc(ls, p, bytes); }, st, &a,
                     &res->launches);
    if (rc) return rc;
  } else {
    for (PlanDev& p : plans) p.tail2 = 0;
  }
  MG_CK(cudaMemcpyAsync(ls->plans, plans.data(), uint64_t(nq) * sizeof(PlanDev),
                        cudaMemcpyHostToDevice, st));
  MG_CK(cudaEventRecord(ls->ev_start, st));

  a.g = dg->g;
  a.count_mode = 1;
  a.star = o.no_tail != 1;
  a.filters = o.filters & MG_FILTER_ALL;
  a.grab = o.grab;
  a.root_step = 1;
  a.probe_min = o.probe_min ? o.probe_min : kProbeMin;
  a.q_budget = o.max_elements;
  a.lane = 1;
  a.cap_rows = cap;
  a.seg_cap = ls->seg_cap;
  a.spin_limit = kSpinLimit;
  a.nq = 1;
  for (Lane& L : ls->lanes) {
    MG_CK(cudaStreamWaitEvent(L.st, ls->ev_start, 0));
    MG_CK(cudaMemsetAsync(L.ctr, 0, C_NUM * 8, L.st));
    MG_CK(cudaMemsetAsync(L.counts, 0, 8, L.st));
    MG_CK(cudaMemsetAsync(L.lvl, 0, (MAXK + 1) * 8, L.st));
    MG_CK(cudaMemsetAsync(L.qel, 0, 8, L.st));
  }
  const unsigned g_ws = sms * 2, g_tr = sms * 2, g_ex = sms * 4;
  for (uint32_t j = 0; j < nq; ++j) {
    Lane& L = ls->lanes[j % nl];
    const PlanDev& P = plans[j];
    a.plans = ls->plans + j;
    a.ctr = L.ctr;
    a.counts = L.counts;
    a.lvl_rows = L.lvl;
    a.q_elems = L.qel;
    a.scan_status = L.status;
    a.tile_row = L.tile_row;
    const int last = P.zero ? -1 : last_level(P, a.tail_dense != 0, a.star != 0);
    for (int l = 0; l <= last; ++l) {
      a.level = uint32_t(l);
      TabPtrs t{};
      for (int c = 0; c < l; ++c) t.col[c] = L.col[l][c];
      a.in = t;
      a.work = L.work[l];
      a.woff = L.woff[l];
      a.dstart = L.dstart[l];
      a.dci = L.dci[l];
      if (++L.epoch > kEpochMax) {
        MG_CK(cudaMemsetAsync(L.status, 0, (cap / WS_ROWS + 2) * 8, L.st));
        L.epoch = 1;
      }
      k_work_scan<<<g_ws, 256, 0, L.st>>>(a, L.epoch);
      k_tile_rows_lane<<<g_tr, 256, 0, L.st>>>(a);
      const bool writes = l < last;
      TabPtrs out{};
      if (writes)
        for (int c = 0; c <= l; ++c) out.col[c] = L.col[l + 1][c];
      a.out = out;
      a.out_cap = writes ? cap : 0;
      a.out_slot = C_LOUT + l;
      a.tile_slot = C_LTILE + l;
      launch_expand(a, &P, 1, true, writes, g_ex, L.st);
      res->launches += 3;
      res->expand_launches++;
    }
    k_lane_done<<<1, 32, 0, L.st>>>(L.ctr, L.counts, L.lvl, L.qel, o.max_elements, j,
                                   ls->r_counts, ls->r_lvl, ls->r_err, ls->r_balg);
    res->launches++;
  }
  MG_CK(cudaGetLastError());
  for (Lane& L : ls->lanes) {
    MG_CK(cudaEventRecord(ls->ev_end, L.st));
    MG_CK(cudaStreamWaitEvent(st, ls->ev_end, 0));
  }
  MG_CK(cudaEventRecord(ws->ev1, st));
  std::vector<unsigned long long> err(nq), cnt(nq), lv(uint64_t(nq) * (MAXK + 1)),
      balg(uint64_t(nq) * 2);
  MG_CK(cudaMemcpyAsync(cnt.data(), ls->r_counts, uint64_t(nq) * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(err.data(), ls->r_err, uint64_t(nq) * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(lv.data(), ls->r_lvl, lv.size() * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(balg.data(), ls->r_balg, balg.size() * 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  float ms = 0;
  MG_CK(cudaEventElapsedTime(&ms, ws->ev0, ws->ev1));
  res->ms = ms;
  for (uint32_t j = 0; j < nq; ++j) {
    if (err[j]) continue;  // charged by its re-run below
    res->balg += balg[2ull * j];
    res->balgc += balg[2ull * j + 1];
  }
  for (uint32_t j = 0; j < nq; ++j) {
    if (err[j] & ERR_TIMEOUT)
      return set_error(MG_E_TIMEOUT, "query %u: a lane's device wait gave up", j);
    if (err[j] & ERR_OVERFLOW) {
      // Did not fit its lane: count it again on the chunked path.
      std::vector<PlanDev> one(1, plans[j]);
      RunResult r1;
      uint64_t c1 = 0;
      std::vector<uint64_t> l1(MAXK + 1, 0);
      mg_opts o1 = o;
      o1.chunk_rows = 0;
      rc = run_levels(dg, one, true, nullptr, o1, &c1, &r1, l1.data());
      if (rc == MG_E_LIMIT && o.max_elements) {
        // Past the per-query budget on the chunked path as well: unknown, as a
        // query over budget in its lane reports.
        cnt[j] = ~0ull;
        for (uint32_t i = 0; i <= MAXK; ++i) lv[uint64_t(j) * (MAXK + 1) + i] = 0;
        res->reruns++;
        continue;
      }
      if (rc) return rc;
      cnt[j] = c1;
      for (uint32_t i = 0; i <= MAXK; ++i) lv[uint64_t(j) * (MAXK + 1) + i] = l1[i];
      res->balg += r1.balg;
      res->balgc += r1.balgc;
      res->ms += r1.ms;
      res->launches += r1.launches;
      res->reruns++;
    }
  }
  for (uint32_t j = 0; j < nq; ++j) counts_out[j] = cnt[j];
  if (level_rows_out)
    for (uint64_t x = 0; x < lv.size(); ++x) level_rows_out[x] = lv[x];
  return MG_OK;
}

// Self-test of the bounded device wait: one work/scan launch of a lane at
// level 1 over 2 * WS_ROWS rows of the first query vertex's bucket, with the
// counter that hands out tiles already past tile 0, so the block of tile 1
// waits for a predecessor nobody publishes.  The wait gives up after
// `spin_limit` polls and the launch ends with ERR_TIMEOUT in its error word.
static int selftest_wait(DevGraph* dg, const mg_csr_view* q, uint32_t spin_limit,
                         uint64_t* err_bits) {
  PlanDev P;
  mg_opts o;
  mg_opts_default(&o);
  int rc = prepare(dg, q, o, &P);
  if (rc) return rc;
  if (P.k < 2 || P.ncons[1] == 0)
    return set_error(MG_E_ARG, "self-test query needs a second vertex joined to the first");
  if ((rc = ensure_lanes(dg, 1, kLaneCap, std::max<uint32_t>(P.k, 2)))) return rc;
  LaneSet* ls = dg->lanes;
  Lane& L = ls->lanes[0];
  if (ls->plans_cap < 1) {
    if ((rc = lane_alloc(ls, (void**)&ls->plans, sizeof(PlanDev)))) return rc;
    ls->plans_cap = 1;
  }
  cudaStream_t st = L.st;
  const uint64_t rows = 2 * WS_ROWS;
  std::vector<unsigned long long> ctr(C_NUM, 0);
  ctr[C_LOUT + 0] = rows;  // level-1 table holds `rows` rows
  ctr[C_LSCAN + 1] = 1;    // tile 0 of level 1 is never handed out
  MG_CK(cudaMemcpyAsync(ls->plans, &P, sizeof(PlanDev), cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemcpyAsync(L.ctr, ctr.data(), C_NUM * 8, cudaMemcpyHostToDevice, st));
  // every row holds the first vertex of the bucket of position 0
  const uint32_t b0 = dg->h_bucket_off[P.label[0]];
  std::vector<uint32_t> col(rows, 0);
  MG_CK(cudaMemcpyAsync(col.data(), dg->g.bucket_vid + b0, 4, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  for (uint64_t r = 1; r < rows; ++r) col[r] = col[0];
  MG_CK(cudaMemcpyAsync(L.col[1][0], col.data(), rows * 4, cudaMemcpyHostToDevice, st));
  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = dg->g;
  a.plans = ls->plans;
  a.ctr = L.ctr;
  a.counts = L.counts;
  a.lvl_rows = L.lvl;
  a.q_elems = L.qel;
  a.level = 1;
  a.in.col[0] = L.col[1][0];
  a.work = L.work[1];
  a.woff = L.woff[1];
  a.dstart = L.dstart[1];
  a.dci = L.dci[1];
  a.lane = 1;
  a.cap_rows = ls->cap;
  a.seg_cap = ls->seg_cap;
  a.scan_status = L.status;
  a.spin_limit = spin_limit;
  a.root_step = 1;
  if (++L.epoch > kEpochMax) {
    MG_CK(cudaMemsetAsync(L.status, 0, (ls->cap / WS_ROWS + 2) * 8, st));
    L.epoch = 1;
  }
  k_work_scan<<<2, 256, 0, st>>>(a, L.epoch);
  MG_CK(cudaGetLastError());
  unsigned long long err = 0;
  MG_CK(cudaMemcpyAsync(&err, L.ctr + C_ERR, 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemsetAsync(L.ctr, 0, C_NUM * 8, st));
  MG_CK(cudaStreamSynchronize(st));
  *err_bits = err;
  return MG_OK;
}

int subiso_batch(DevGraph* dg, const mg_csr_view* const* qs, uint32_t nq, const mg_opts* opts,
                 uint64_t* counts, mg_stats* st, const uint32_t* orders = nullptr,
                 uint64_t* level_rows = nullptr) {
  const mg_opts o = resolve_opts(opts);
  if (o.matrix_filter)
    return set_error(MG_E_ARG, "matrix_filter applies to single-query count and emit only");
  std::vector<PlanDev> plans(nq);
  std::vector<uint32_t> learned;
  if (!orders && o.order == MG_ORDER_LEARNED && o.model) {
    // One inference launch plans the whole batch.
    int rc = ensure_full_stats(dg);
    if (rc) return rc;
    std::vector<QueryGraph> Q(nq);
    std::vector<const QueryGraph*> qp(nq);
    for (uint32_t i = 0; i < nq; ++i) {
      if ((rc = normalise_query(qs[i], &Q[i])))
        return set_error(rc, "query %u: %s", i, last_error_cstr());
      qp[i] = &Q[i];
    }
    std::vector<std::array<uint32_t, MAXK>> ord;
    if ((rc = order_learned_batch(o.model, qp, dg->stats, ord))) return rc;
    learned.resize(uint64_t(nq) * MAXK);
    for (uint32_t i = 0; i < nq; ++i)
      std::memcpy(&learned[uint64_t(i) * MAXK], ord[i].data(), MAXK * 4);
    orders = learned.data();
  }
  for (uint32_t i = 0; i < nq; ++i) {
    mg_opts oi = o;
    if (orders) {
      oi.order = MG_ORDER_GIVEN;
      oi.given_order = orders + uint64_t(i) * MAXK;
    }
    int rc = prepare(dg, qs[i], oi, &plans[i]);
    if (rc) return set_error(rc, "query %u: %s", i, last_error_cstr());
  }
  RunResult res;
  int rc = o.lanes == MG_LANES_SHARED
               ? run_levels(dg, plans, true, nullptr, o, counts, &res, level_rows)
               : subiso_batch_lanes(dg, plans, o, counts, level_rows, &res);
  if (rc) return rc;
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->balg_bytes = res.balg;
    st->balg_count_bytes = res.balgc;
    st->device_ms = res.ms;
    st->launches = res.launches;
    st->chunks = res.chunks;
    st->elements = res.elements;
    st->expand_ms = res.expand_ms;
    st->expand_launches = res.expand_launches;
  }
  return MG_OK;
}

}  // namespace mg

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* mg_last_error(void) { return mg::last_error_cstr(); }
const char* mg_version(void) { return "mg_subiso 0.1 (sm_100a)"; }

void mg_opts_default(mg_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->order = MG_ORDER_REFERENCE;
  o->filters = MG_FILTER_ALL;
}

#define MG_ENTRY(dgraph)                                              \
  mg::clear_error();                                                  \
  if (!(dgraph)) return mg::set_error(MG_E_ARG, "null graph handle"); \
  auto* dg = static_cast<mg::DevGraph*>(dgraph);                      \
  std::lock_guard<std::mutex> lock(dg->mu);                           \
  mg::DeviceGuard guard(dg->device)

int mg_plan_order(void* dgraph, const mg_csr_view* q, const mg_opts* opts, uint32_t* order,
                  uint32_t* k) {
  mg::clear_error();
  if (!q || !order || !k) return mg::set_error(MG_E_ARG, "null argument");
  mg::QueryGraph Q;
  int rc = mg::normalise_query(q, &Q);
  if (rc) return rc;
  const mg_opts o = mg::resolve_opts(opts);
  if (!dgraph) {
    if (o.order != MG_ORDER_REFERENCE && o.order != MG_ORDER_GIVEN)
      return mg::set_error(MG_E_ARG, "this order needs a graph handle");
    rc = mg::choose_order(nullptr, Q, o, order);
  } else {
    auto* dg = static_cast<mg::DevGraph*>(dgraph);
    std::lock_guard<std::mutex> lock(dg->mu);
    mg::DeviceGuard guard(dg->device);
    rc = mg::choose_order(dg, Q, o, order);
  }
  if (rc) return rc;
  *k = Q.k;
  return MG_OK;
}

int mg_subiso_count_ex(void* dgraph, const mg_csr_view* q, const mg_opts* opts, uint64_t* count,
                       mg_stats* st) {
  MG_ENTRY(dgraph);
  if (!q || !count) return mg::set_error(MG_E_ARG, "null argument");
  try {
    return mg::subiso_count(dg, q, opts, count, st);
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_subiso_count(void* dgraph, const mg_csr_view* q, const mg_opts* opts, uint64_t* count) {
  return mg_subiso_count_ex(dgraph, q, opts, count, nullptr);
}

int mg_subiso_emit_ex(void* dgraph, const mg_csr_view* q, const mg_opts* opts, uint32_t* rows,
                      uint64_t cap_rows, uint64_t* n_rows, mg_stats* st) {
  MG_ENTRY(dgraph);
  if (!q || !n_rows || (cap_rows && !rows)) return mg::set_error(MG_E_ARG, "null argument");
  try {
    return mg::subiso_emit(dg, q, opts, rows, cap_rows, n_rows, st);
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_subiso_emit(void* dgraph, const mg_csr_view* q, const mg_opts* opts, uint32_t* rows,
                   uint64_t cap_rows, uint64_t* n_rows) {
  return mg_subiso_emit_ex(dgraph, q, opts, rows, cap_rows, n_rows, nullptr);
}

int mg_subiso_batch_count_ex(void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                             const mg_opts* opts, uint64_t* counts, mg_stats* st) {
  MG_ENTRY(dgraph);
  if (!qs || !counts || nq == 0) return mg::set_error(MG_E_ARG, "null argument or empty batch");
  try {
    return mg::subiso_batch(dg, qs, nq, opts, counts, st);
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_subiso_batch_count(void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                          const mg_opts* opts, uint64_t* counts) {
  return mg_subiso_batch_count_ex(dgraph, qs, nq, opts, counts, nullptr);
}

int mg_subiso_batch_count_orders(void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                                 const uint32_t* orders, const mg_opts* opts, uint64_t* counts,
                                 uint64_t* level_rows, mg_stats* st) {
  MG_ENTRY(dgraph);
  if (!qs || !counts || nq == 0) return mg::set_error(MG_E_ARG, "null argument or empty batch");
  try {
    return mg::subiso_batch(dg, qs, nq, opts, counts, st, orders, level_rows);
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_plan_orders(void* dgraph, const mg_csr_view* const* qs, uint32_t nq, const mg_opts* opts,
                   uint32_t* orders) {
  MG_ENTRY(dgraph);
  if (!qs || !orders || nq == 0) return mg::set_error(MG_E_ARG, "null argument or empty batch");
  try {
    const mg_opts o = mg::resolve_opts(opts);
    std::vector<mg::QueryGraph> Q(nq);
    for (uint32_t i = 0; i < nq; ++i) {
      int rc = mg::normalise_query(qs[i], &Q[i]);
      if (rc) return mg::set_error(rc, "query %u: %s", i, mg::last_error_cstr());
    }
    std::memset(orders, 0, uint64_t(nq) * MG_MAX_QUERY_VERTICES * 4);
    if (o.order == MG_ORDER_LEARNED && o.model) {
      int rc = mg::ensure_full_stats(dg);
      if (rc) return rc;
      std::vector<const mg::QueryGraph*> qp(nq);
      for (uint32_t i = 0; i < nq; ++i) qp[i] = &Q[i];
      std::vector<std::array<uint32_t, MG_MAX_QUERY_VERTICES>> ord;
      if ((rc = mg::order_learned_batch(o.model, qp, dg->stats, ord))) return rc;
      for (uint32_t i = 0; i < nq; ++i)
        std::memcpy(orders + uint64_t(i) * MG_MAX_QUERY_VERTICES, ord[i].data(), Q[i].k * 4);
      return MG_OK;
    }
    for (uint32_t i = 0; i < nq; ++i) {
      int rc = mg::choose_order(dg, Q[i], o, orders + uint64_t(i) * MG_MAX_QUERY_VERTICES);
      if (rc) return rc;
    }
    return MG_OK;
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_selftest_wait_timeout(void* dgraph, const mg_csr_view* q, uint32_t spin_limit,
                             int* status) {
  MG_ENTRY(dgraph);
  if (!q || !status || spin_limit == 0) return mg::set_error(MG_E_ARG, "bad argument");
  uint64_t err = 0;
  int rc = mg::selftest_wait(dg, q, spin_limit, &err);
  if (rc) return rc;
  *status = (err & mg::ERR_TIMEOUT) ? MG_E_TIMEOUT : MG_OK;
  return MG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free count (mg_subiso_count_noalloc)
//
// For callers that cannot allocate device memory when they ask for a count:
// processes whose device memory is owned by another allocator (a framework's
// caching allocator that has reserved nearly all HBM, a fixed arena), or
// latency-critical paths that must not pay cudaMalloc/cudaFree and the
// device-wide synchronisation cudaFree implies.  The level tables, scan
// scratch, counters and the plan live in the file-scope array below, sized
// once at load time and held by every GPU that loads the library until the
// process exits.  The data graph must already be resident (mg_graph_upload).
// ---------------------------------------------------------------------------
namespace mg {

static __device__ __align__(256) unsigned char g_noalloc_scratch[MG_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch per device, looked up once per device
// (with that device current) by the first call on it.
std::mutex g_noalloc_mu;  // one call at a time: every call shares the array
void* g_noalloc_ptr[256] = {};

int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 256) return set_error(MG_E_ARG, "device %d out of range", device);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(MG_E_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) on device %d: %s",
                       device, cudaGetErrorString(e));
    g_noalloc_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
  return MG_OK;
}

// Carves the level tables of a single-query count out of `base`; returns the
// bytes used (a size above MG_NOALLOC_SCRATCH_BYTES means it does not fit).
struct NoallocLayout {
  unsigned long long* ctr;
  unsigned long long* counts;
  unsigned long long* lvl_rows;
  PlanDev* plan;
  uint64_t* bsum;
  uint32_t* tile_row;
  uint32_t* col[MAXK][MAXK];
  uint32_t* work[MAXK];
  uint64_t* woff[MAXK];
  uint32_t* dstart[MAXK];
  uint8_t* dci[MAXK];
};

// Elements per expand launch of a level whose survivors are not stored.
constexpr uint64_t kNoallocSegment = 1ull << 24;

uint64_t noalloc_carve(unsigned char* base, uint64_t cap, uint32_t k, NoallocLayout* L) {
  uint64_t off = 0;
  auto take = [&](uint64_t bytes) -> unsigned char* {
    off = (off + 255) & ~uint64_t(255);
    unsigned char* p = base ? base + off : nullptr;
    off += bytes;
    return p;
  };
  L->ctr = reinterpret_cast<unsigned long long*>(take(C_NUM * 8));
  L->counts = reinterpret_cast<unsigned long long*>(take(8));
  L->lvl_rows = reinterpret_cast<unsigned long long*>(take((MAXK + 1) * 8));
  L->plan = reinterpret_cast<PlanDev*>(take(sizeof(PlanDev)));
  L->bsum = reinterpret_cast<uint64_t*>(take((cap / SCAN_TILE + 2) * 8));
  L->tile_row = reinterpret_cast<uint32_t*>(take((kNoallocSegment / EXPAND_BLOCK + 2) * 4));
  for (uint32_t l = 0; l < k; ++l) {
    const uint64_t rows = l == 0 ? 1 : cap;
    for (uint32_t j = 0; j < l; ++j) L->col[l][j] = reinterpret_cast<uint32_t*>(take(rows * 4));
    L->work[l] = reinterpret_cast<uint32_t*>(take(rows * 4));
    L->woff[l] = reinterpret_cast<uint64_t*>(take((rows + 1) * 8));
    L->dstart[l] = reinterpret_cast<uint32_t*>(take(rows * 4));
    L->dci[l] = reinterpret_cast<uint8_t*>(take(rows));
  }
  return off;
}

int noalloc_count(DevGraph* dg, const mg_csr_view* q, const mg_opts* opts, uint64_t* count) {
  mg_opts o;
  mg_opts_default(&o);
  if (opts) o = *opts;
  // Every argument is checked before any work is queued on the shared array.
  int rc = check_opts(o);
  if (rc) return rc;
  if (o.matrix_filter)
    return set_error(MG_E_ARG, "mg_subiso_count_noalloc does not apply a matrix filter");
  QueryGraph Q;
  rc = normalise_query(q, &Q);  // the allocating entry points' normaliser
  if (rc) return rc;
  uint32_t order[MAXK];
  if (o.order == MG_ORDER_REFERENCE) {
    order_reference(Q, order);
  } else if (o.order == MG_ORDER_STRONG) {
    order_strong(Q, dg->stats, order);
  } else if (o.order == MG_ORDER_GIVEN) {
    if (!o.given_order) return set_error(MG_E_ARG, "MG_ORDER_GIVEN without given_order");
    std::memcpy(order, o.given_order, Q.k * 4);
    if (!order_is_permutation(order, Q.k))
      return set_error(MG_E_ARG, "given_order is not a permutation of 0..%u", Q.k - 1);
  } else {
    return set_error(MG_E_ARG, "mg_subiso_count_noalloc supports the reference, strong and "
                               "given orders only");
  }
  PlanDev P;
  if ((rc = build_plan(dg, Q, order, &P))) return rc;
  const uint32_t k = P.k;

  // Rows per level table: the largest power of two whose layout fits, or the
  // caller's chunk_rows, which must fit.
  NoallocLayout L;
  uint64_t cap = 0;
  if (o.chunk_rows) {
    if (o.chunk_rows > (1ull << 31) ||
        noalloc_carve(nullptr, o.chunk_rows, k, &L) > MG_NOALLOC_SCRATCH_BYTES)
      return set_error(MG_E_LIMIT,
                       "chunk_rows=%llu for a %u-vertex query needs %llu bytes of scratch; the "
                       "static scratch holds %llu bytes",
                       (unsigned long long)o.chunk_rows, k,
                       (unsigned long long)noalloc_carve(nullptr, std::min<uint64_t>(
                           o.chunk_rows, 1ull << 31), k, &L),
                       (unsigned long long)MG_NOALLOC_SCRATCH_BYTES);
    cap = o.chunk_rows;
  } else {
    for (uint64_t c = 1ull << 22; c >= 64; c >>= 1)
      if (noalloc_carve(nullptr, c, k, &L) <= MG_NOALLOC_SCRATCH_BYTES) {
        cap = c;
        break;
      }
    if (!cap)
      return set_error(MG_E_LIMIT, "a %u-vertex query does not fit the %llu-byte static scratch",
                       k, (unsigned long long)MG_NOALLOC_SCRATCH_BYTES);
  }
  unsigned char* base = nullptr;
  if ((rc = noalloc_scratch(dg->device, &base))) return rc;
  noalloc_carve(base, cap, k, &L);

  cudaStream_t st = dg->stream;
  // The array keeps the previous call's contents: counters start at zero.
  MG_CK(cudaMemcpyAsync(L.plan, &P, sizeof(PlanDev), cudaMemcpyHostToDevice, st));
  MG_CK(cudaMemsetAsync(L.counts, 0, 8, st));
  MG_CK(cudaMemsetAsync(L.lvl_rows, 0, (MAXK + 1) * 8, st));
  MG_CK(cudaMemsetAsync(L.ctr, 0, C_NUM * 8, st));

  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = dg->g;
  a.plans = L.plan;
  a.ctr = L.ctr;
  a.counts = L.counts;
  a.lvl_rows = L.lvl_rows;
  a.count_mode = 1;
  a.filters = o.filters & MG_FILTER_ALL;
  a.nq = 1;
  a.grab = o.grab;
  a.tile_row = L.tile_row;
  a.root_step = o.root_step > 1 ? o.root_step : 1u;
  a.probe_min = o.probe_min ? o.probe_min : kProbeMin;
  a.out_slot = C_OUT;
  a.tile_slot = C_TILE;
  if (o.root_end || a.root_step > 1) {
    a.root_begin = o.root_begin;
    a.root_end = o.root_end ? o.root_end : ~0ull;
  }
  bool writes[MAXK] = {};
  for (uint32_t l = 0; l < k; ++l)
    writes[l] = P.k > l + 1 && !(P.k == l + 2 && P.last_o1);
  auto tab = [&](uint32_t l) {
    TabPtrs t{};
    for (uint32_t j = 0; j < l; ++j) t.col[j] = L.col[l][j];
    return t;
  };
  const unsigned sms = dg->sms;
  uint64_t T[MAXK] = {}, cur[MAXK] = {}, host_u64 = 0, elements = 0;
  uint32_t R[MAXK] = {};
  R[0] = 1;
  int lvl = 0;
  bool need_work = true;
  while (true) {
    a.level = uint32_t(lvl);
    a.R = R[lvl];
    a.in = tab(lvl);
    a.work = L.work[lvl];
    a.woff = L.woff[lvl];
    a.dstart = L.dstart[lvl];
    a.dci = L.dci[lvl];
    if (need_work) {
      k_work<<<grid_for(R[lvl], 256, sms * 16), 256, 0, st>>>(a);
      const uint32_t nb = (R[lvl] + SCAN_TILE - 1) / SCAN_TILE;
      k_scan_reduce<<<nb, 256, 0, st>>>(L.work[lvl], R[lvl], L.bsum);
      k_scan_bsum<<<1, 1024, 0, st>>>(L.bsum, nb, L.woff[lvl] + R[lvl]);
      k_scan_apply<<<nb, 256, 0, st>>>(L.work[lvl], R[lvl], L.bsum, L.woff[lvl]);
      MG_CK(cudaMemcpyAsync(&host_u64, L.woff[lvl] + R[lvl], 8, cudaMemcpyDeviceToHost, st));
      MG_CK(cudaStreamSynchronize(st));
      T[lvl] = host_u64;
      cur[lvl] = 0;
      need_work = false;
    }
    if (cur[lvl] < T[lvl]) {
      const uint64_t t0 = cur[lvl];
      const uint64_t t1 = writes[lvl] ? std::min(T[lvl], t0 + cap) : T[lvl];
      elements += t1 - t0;
      if (o.max_elements && elements > o.max_elements) {
        cudaStreamSynchronize(st);  // nothing of this call stays queued on the array
        return set_error(MG_E_LIMIT, "work budget of %llu candidate elements exceeded",
                         (unsigned long long)o.max_elements);
      }
      a.out = writes[lvl] ? tab(lvl + 1) : TabPtrs{};
      a.out_cap = writes[lvl] ? cap : 0;
      MG_CK(cudaMemsetAsync(L.ctr + C_OUT, 0, 8, st));
      const uint64_t seg = writes[lvl] ? std::min<uint64_t>(cap, kNoallocSegment) : kNoallocSegment;
      for (uint64_t s0 = t0; s0 < t1; s0 += seg) {
        const uint64_t s1 = std::min(t1, s0 + seg);
        const uint32_t ntiles = uint32_t((s1 - s0 + EXPAND_BLOCK - 1) / EXPAND_BLOCK);
        a.t0 = s0;
        a.t1 = s1;
        k_tile_rows<<<grid_for(uint64_t(ntiles) + 1, 256, sms * 16), 256, 0, st>>>(
            L.woff[lvl], R[lvl], s0, s1, ntiles, L.tile_row);
        MG_CK(cudaMemsetAsync(L.ctr + C_TILE, 0, 8, st));
        launch_expand(a, &P, 1, true, writes[lvl],
                      grid_for(s1 - s0, EXPAND_BLOCK, sms * 8), st);
      }
      MG_CK(cudaGetLastError());
      cur[lvl] = t1;
      if (writes[lvl]) {
        MG_CK(cudaMemcpyAsync(&host_u64, L.ctr + C_OUT, 8, cudaMemcpyDeviceToHost, st));
        MG_CK(cudaStreamSynchronize(st));
        if (host_u64 > cap)
          return set_error(MG_E_CUDA, "level table overflow (%llu > %llu)",
                           (unsigned long long)host_u64, (unsigned long long)cap);
        if (host_u64 > 0) {
          R[lvl + 1] = uint32_t(host_u64);
          ++lvl;
          need_work = true;
        }
      }
    } else {
      if (lvl == 0) break;
      --lvl;
    }
  }
  unsigned long long err = 0, c = 0;
  MG_CK(cudaMemcpyAsync(&err, L.ctr + C_ERR, 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaMemcpyAsync(&c, L.counts, 8, cudaMemcpyDeviceToHost, st));
  MG_CK(cudaStreamSynchronize(st));
  MG_CK(cudaGetLastError());
  if (err & ERR_OVERFLOW) return set_error(MG_E_CUDA, "device table overflow");
  *count = c;
  return MG_OK;
}

}  // namespace
}  // namespace mg

extern "C" int mg_subiso_count_noalloc(void* dgraph, const mg_csr_view* q, const mg_opts* opts,
                                       uint64_t* count) {
  mg::clear_error();
  if (!dgraph || !q || !count) return mg::set_error(MG_E_ARG, "null argument");
  auto* dg = static_cast<mg::DevGraph*>(dgraph);
  std::lock_guard<std::mutex> glock(mg::g_noalloc_mu);
  std::lock_guard<std::mutex> lock(dg->mu);
  mg::DeviceGuard guard(dg->device);
  return mg::noalloc_count(dg, q, opts, count);
}
