// Device-side data layout of a resident data graph and of matching plans.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <memory>

#include "mg_internal.h"

namespace mg {

constexpr int MAXK = MG_MAX_QUERY_VERTICES;
constexpr int WMAX = MG_MAX_LABELS / 32;
constexpr uint8_t DCI_BUCKET = 0xFF;
constexpr uint32_t FULL = 0xFFFFFFFFu;

// Error bits raised by kernels (read back by the host after each call).
constexpr uint32_t ERR_OVERFLOW = 1u;   // a table write exceeded its capacity
constexpr uint32_t ERR_RANGE = 2u;      // an adjacency id outside [0, n)
constexpr uint32_t ERR_TIMEOUT = 4u;    // a bounded device wait gave up

// Read-only view of a resident graph, passed by value to kernels.
//   adj[d]   : adjacency of direction d (0 = out, 1 = in), each vertex's list
//              ordered by (label, id): label slices are contiguous and sorted
//   loff[d]  : n*L+1 slice starts; slice (v, l) = [loff[v*L+l], loff[v*L+l+1])
//   nlb[d]   : n*W neighbour-label bits (bit l: v has a d-neighbour labelled l)
//   deg[d]   : distinct d-neighbours
//   label    : compact labels 0..L-1
//   bucket_* : vertices grouped by label (ascending id inside a bucket)
//   selfbits : bit v set when (v, v) is an edge
//   globalid : local id -> global id of the reference format
struct GraphDev {
  uint32_t n, L, W, symmetric;
  const uint32_t* adj[2];
  const uint32_t* loff[2];
  const uint32_t* nlb[2];
  const uint32_t* deg[2];
  const uint32_t* label;
  const uint32_t* bucket_off;
  const uint32_t* bucket_vid;
  const uint32_t* bucket_pos;  // index of every vertex inside its label bucket
  const uint32_t* selfbits;
  const uint32_t* globalid;
  // Hub bitmaps per direction (nullptr: none): hub_slot[d][v] is v's row in
  // hub_bits[d] or NO_HUB; a row holds hub_words words, bit x set when x is a
  // d-neighbour of v.
  const uint16_t* hub_slot[2];
  const uint32_t* hub_bits[2];
  const uint32_t* hub_vid[2];  // vertex of each hub slot
  uint32_t n_hubs[2];
  uint32_t hub_words;
};
constexpr uint16_t NO_HUB = 0xFFFF;

// Matching plan of one query for one order.  Position i matches query vertex
// perm[i].  cons[i][c] = pos | dir << 8: the candidate for position i must be
// in the dir-adjacency of the vertex matched at position pos (< i).
struct PlanDev {
  uint32_t k;
  uint32_t last_o1;         // last position has one constraint, no self-loop
  uint32_t selfloop_mask;   // bit i: query vertex perm[i] has a self-loop
  uint32_t zero;            // 1: some label of the query is absent (count 0)
  uint32_t label[MAXK];
  uint32_t ncons[MAXK];
  uint32_t cons[MAXK][MAXK];
  uint32_t req[2][MAXK];               // degree requirement per direction
  uint32_t nlbq[2][MAXK][WMAX];        // required neighbour-label bits
  uint32_t samelab[MAXK];              // positions j < i with the same label
  uint32_t guar[MAXK];                 // last position: m(j) surely in slice
  uint32_t perm[MAXK];
  // Two-position pendant tail (count mode): position a = k-2 has the single
  // backward neighbour tail_p (direction tail_da), position b = k-1 has the
  // single backward neighbour a (direction tail_db), neither has a self-loop,
  // and every earlier position labelled like b is tail_p itself with
  // matching directions.  Rows of prefix length k-2 are then counted in
  // closed form from a per-vertex two-hop aggregate.
  uint32_t tail2;
  uint32_t tail_p, tail_da, tail_db;
  uint32_t tail_Ia;  // positions i < a labelled like position a
  uint32_t tail_J;   // positions j < a labelled like position b
  uint32_t tail_kid; // index of (da, la, db, lb) in the call's tail-key table
  // Two final leaves of one anchor (count mode): positions k-2 and k-1 each
  // have the single backward neighbour star_p (< k-2) in direction star_d and
  // no self-loop, and no edge between them.  A prefix of length k-2 then has
  // A = |S_a| minus its matches inside S_a choices for k-2 and, for k-1,
  // A - 1 when both carry one label (the same slice) or the free entries of
  // the other label's slice; it is counted while position k-3 expands.
  uint32_t star2;
  uint32_t star_p, star_d;
};

// Signature of a two-hop aggregate: A(y) = sum over the da-slice of y labelled
// la of the db-slice lengths labelled lb.  Queries of one call sharing a
// signature share the hub table of aggregates.
struct TailKey {
  uint32_t da, la, db, lb;
  uint32_t lp;     // label of m_p: only hubs with this label get aggregates
  uint32_t pad;
  uint64_t base;   // first entry of this key's hub table (~0: none)
  uint64_t lazy;   // first entry of this key's lazily filled table over the
                   // bucket of label lp (~0: none, sum in place)
};

struct Workspace;  // enumeration scratch (mg_enum.cu)
struct LaneSet;    // batch lane pipelines (mg_enum.cu)

// Host object behind the opaque dgraph handle.
struct DevGraph {
  int device = 0;
  unsigned sms = 1;  // multiprocessors of the device (grid sizing)
  cudaStream_t stream = nullptr;
  GraphDev g{};
  mg_graph_info info{};
  GraphStats stats;
  bool stats_full = false;   // degree / label-pair statistics computed
  std::vector<uint32_t> h_bucket_off;
  std::vector<void*> allocs;
  Workspace* ws = nullptr;
  LaneSet* lanes = nullptr;
  std::mutex mu;
  ~DevGraph();
};

int ensure_full_stats(DevGraph* dg);

// Makes device d current for a scope and restores the caller's device.
struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int d) {
    cudaGetDevice(&prev);
    cudaSetDevice(d);
  }
  ~DeviceGuard() { cudaSetDevice(prev); }
};

// Keep bits (ceil(n/32) words) of the vertices of label bucket `lab` for query
// vertex u under a matrix filter (mg_matrix_filter.cu); synchronises st.
int matrix_filter_roots(void* filter, const DevGraph* dg, uint32_t u, uint32_t lab,
                        uint32_t* bits, cudaStream_t st);

#define MG_CK(call)                                                          \
  do {                                                                       \
    cudaError_t _e = (call);                                                 \
    if (_e != cudaSuccess)                                                   \
      return ::mg::set_error(MG_E_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, \
                             #call, cudaGetErrorString(_e));                 \
  } while (0)

// cudaMalloc that records the allocation on the graph and maps failure to
// MG_E_OOM.
int dev_alloc(DevGraph* dg, void** p, size_t bytes);

}  // namespace mg
