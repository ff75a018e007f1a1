// Internal declarations shared by the host C++ and CUDA sources of
// libmg_subiso.so.  Nothing here crosses the C-ABI.
#pragma once

#include <array>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <string>
#include <vector>
#include <mutex>

#include "mg_subiso.h"

namespace mg {

// ---- errors: thread-local message, negative status codes ------------------
int set_error(int code, const char* fmt, ...);
void clear_error();

int validate_csr_view(const mg_csr_view* v);

// ---- host CSR in the reference layout --------------------------------------
// Arrays exactly as graphs/0.bin + label/0.bin of the reference
// (core/data_structures/immutable_csr.cu:103-166).  When in_is_out is set the
// in-arrays are not stored and the view aliases the out-arrays.
struct HostCSR {
  uint32_t n = 0, max_vid = 0, min_vid = 0, m_in = 0, m_out = 0;
  bool in_is_out = false;
  std::vector<uint32_t> globalid, indeg, outdeg, in_off, out_off, in_edges,
      out_edges, eg_by_l, l_by_g, labels;
  void fill_view(mg_csr_view* v) const;
};

// Builds a HostCSR over vertices 0..n-1 from directed pairs; adjacency lists
// are sorted.  Multi-threaded.
int build_csr_from_pairs(uint32_t n, const uint32_t* src, const uint32_t* dst,
                         uint64_t m, const uint32_t* labels, uint32_t flags,
                         HostCSR* out);

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers:
// as easy as 1, 2, 3", SC'11), counter-based: (key, counter) -> 4 words -------
struct Philox4 {
  uint32_t v[4];
};
Philox4 philox4x32_10(uint64_t key, uint64_t ctr_lo, uint64_t ctr_hi);
// Uniform double in [0,1) from two 32-bit words (53 bits).
inline double u53(uint32_t a, uint32_t b) {
  uint64_t x = (uint64_t(a) << 21) ^ (uint64_t(b) >> 11);
  x &= ((uint64_t(1) << 53) - 1);
  return double(x) * (1.0 / 9007199254740992.0);
}
// Sequential stream of words from (seed, stream).
struct RngStream {
  uint64_t seed, stream, ctr = 0;
  Philox4 buf{};
  int used = 4;
  RngStream(uint64_t s, uint64_t st) : seed(s), stream(st) {}
  uint32_t next() {
    if (used == 4) {
      buf = philox4x32_10(seed, ctr++, stream);
      used = 0;
    }
    return buf.v[used++];
  }
  // Uniform integer in [0, n) by multiply-shift of a 32-bit word.
  uint32_t below(uint32_t n) { return uint32_t((uint64_t(next()) * n) >> 32); }
  double uniform() {
    uint32_t a = next();
    uint32_t b = next();
    return u53(a, b);
  }
};

// ---- normalised query -------------------------------------------------------
// Local ids 0..k-1 (CSR row order), edge sets as bit masks, raw labels, and
// the distinct directed edges in CSR order.  Fixed-size storage: normalising
// a query touches no heap, so allocation-free entry points share it.
struct QueryGraph {
  uint32_t k = 0;
  uint32_t label_raw[MG_MAX_QUERY_VERTICES];
  uint32_t out_mask[MG_MAX_QUERY_VERTICES];  // bit w set: edge u -> w
  uint32_t in_mask[MG_MAX_QUERY_VERTICES];   // bit w set: edge w -> u
  uint32_t n_edges = 0;
  uint8_t edge_u[MG_MAX_QUERY_VERTICES * MG_MAX_QUERY_VERTICES];
  uint8_t edge_w[MG_MAX_QUERY_VERTICES * MG_MAX_QUERY_VERTICES];
};
int normalise_query(const mg_csr_view* q, QueryGraph* out);

// Graph-level statistics used by orders and the order model (host side).
struct GraphStats {
  uint32_t n = 0, L = 0;
  bool symmetric = true;
  std::vector<uint32_t> label_values;      // compact id -> raw label
  std::vector<uint64_t> label_count;       // vertices per compact label
  std::vector<double> label_deg_mean, label_deg_max, label_deg_p99;
  std::vector<uint64_t> label_pair_edges;  // L*L directed edge counts
  std::vector<uint64_t> label_nlb_density; // sum over vertices of popc(NLB)
  int compact_label(uint32_t raw) const;   // -1 if absent
};

// Orders (query-local ids).  Reference: core/data_structures/
// woj_exec_plan.cuh:36-45 and kernel_woj_subsio.cu:1006-1008.
void order_reference(const QueryGraph& q, uint32_t* order);
void order_strong(const QueryGraph& q, const GraphStats& gs, uint32_t* order);
bool order_is_permutation(const uint32_t* order, uint32_t k);

// Learned order model (mg_order_model.cu).
int order_learned(void* model, const QueryGraph& q, const GraphStats& gs,
                  uint32_t* order);
// Device named by MATRIXGRAPH_CUDA_DEVICE, else the current one (mg_graph.cu).
int env_or_current_device(int* dev);

int order_learned_batch(void* model, const std::vector<const QueryGraph*>& qs,
                        const GraphStats& gs,
                        std::vector<std::array<uint32_t, MG_MAX_QUERY_VERTICES>>& orders);

}  // namespace mg
