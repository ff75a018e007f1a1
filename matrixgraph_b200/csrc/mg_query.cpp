// Query normalisation and matching orders.
#include <algorithm>
#include <cstring>

#include "mg_internal.h"

namespace mg {

// Pattern graphs use the data-graph CSR format (SubIso::LoadData reads both
// with ImmutableCSR::Read, core/task/gpu_task/subiso.cu:101-110).  Adjacency
// entries are global ids; they are mapped back to local ids through
// globalid[] (core/util/format_converter.cuh:166-184).
int normalise_query(const mg_csr_view* q, QueryGraph* out) {
  int rc = validate_csr_view(q);
  if (rc) return rc;
  if (q->n == 0) return set_error(MG_E_ARG, "empty query");
  if (q->n > MG_MAX_QUERY_VERTICES)
    return set_error(MG_E_LIMIT, "query has %u vertices; at most %d supported", q->n,
                     MG_MAX_QUERY_VERTICES);
  QueryGraph& Q = *out;
  Q.k = q->n;
  // Global -> local id by a linear scan (k <= 16): no heap.
  auto local = [&](uint32_t gid) -> uint32_t {
    for (uint32_t x = 0; x < q->n; ++x)
      if (q->globalid[x] == gid) return x;
    return UINT32_MAX;
  };
  for (uint32_t i = 0; i < q->n; ++i) {
    if (local(q->globalid[i]) != i)
      return set_error(MG_E_FORMAT, "query globalid %u repeated", q->globalid[i]);
    Q.label_raw[i] = q->labels[i];
    Q.out_mask[i] = Q.in_mask[i] = 0;
  }
  Q.n_edges = 0;
  for (uint32_t u = 0; u < q->n; ++u) {
    for (uint32_t e = q->out_off[u]; e < q->out_off[u + 1]; ++e) {
      const uint32_t w = local(q->out_edges[e]);
      if (w == UINT32_MAX)
        return set_error(MG_E_FORMAT, "query out-edge to unknown vertex %u", q->out_edges[e]);
      if (!(Q.out_mask[u] >> w & 1)) {
        Q.edge_u[Q.n_edges] = uint8_t(u);
        Q.edge_w[Q.n_edges] = uint8_t(w);
        ++Q.n_edges;
      }
      Q.out_mask[u] |= 1u << w;
      Q.in_mask[w] |= 1u << u;
    }
  }
  // In-edges must describe the same edge set (both arrays are part of the
  // reference format; a pattern whose in-arrays disagree is malformed).
  if (q->m_in > 0) {
    uint32_t in_mask[MG_MAX_QUERY_VERTICES] = {0};
    for (uint32_t u = 0; u < q->n; ++u)
      for (uint32_t e = q->in_off[u]; e < q->in_off[u + 1]; ++e) {
        const uint32_t w = local(q->in_edges[e]);
        if (w == UINT32_MAX)
          return set_error(MG_E_FORMAT, "query in-edge from unknown vertex %u", q->in_edges[e]);
        in_mask[u] |= 1u << w;
      }
    for (uint32_t u = 0; u < q->n; ++u)
      if (in_mask[u] != Q.in_mask[u])
        return set_error(MG_E_FORMAT, "query in-edges disagree with out-edges at vertex %u", u);
  }
  return MG_OK;
}

int GraphStats::compact_label(uint32_t raw) const {
  auto it = std::lower_bound(label_values.begin(), label_values.end(), raw);
  if (it == label_values.end() || *it != raw) return -1;
  return int(it - label_values.begin());
}

bool order_is_permutation(const uint32_t* order, uint32_t k) {
  uint32_t seen = 0;
  for (uint32_t i = 0; i < k; ++i) {
    if (order[i] >= k || (seen >> order[i] & 1)) return false;
    seen |= 1u << order[i];
  }
  return true;
}

// Vertex-introduction order of the reference WOJ chain: directed pattern
// edges in CSR order (woj_exec_plan.cuh:36-45); the first edge places both
// endpoints, later edges place an endpoint the first time the edge touches
// the placed prefix.  The reference skips edges that are disconnected at
// their turn and never revisits them (kernel_woj_subsio.cu:1006-1008); here
// the edge list is rescanned until nothing changes, and an unreachable
// vertex (another component) starts a new scan from the lowest id.
void order_reference(const QueryGraph& q, uint32_t* order) {
  uint32_t placed = 0, n = 0;
  auto place = [&](uint32_t v) {
    if (!(placed >> v & 1)) {
      placed |= 1u << v;
      order[n++] = v;
    }
  };
  if (q.n_edges) {
    place(q.edge_u[0]);
    place(q.edge_w[0]);
  }
  while (n < q.k) {
    bool changed = true;
    while (changed) {
      changed = false;
      for (uint32_t e = 0; e < q.n_edges; ++e) {
        bool a = placed >> q.edge_u[e] & 1, b = placed >> q.edge_w[e] & 1;
        if (a && !b) {
          place(q.edge_w[e]);
          changed = true;
        } else if (b && !a) {
          place(q.edge_u[e]);
          changed = true;
        }
      }
    }
    if (n < q.k) {
      for (uint32_t v = 0; v < q.k; ++v)
        if (!(placed >> v & 1)) {
          place(v);
          break;
        }
    }
  }
}

// Classical strong heuristic: start at the vertex with the fewest label
// candidates (ties: larger degree, then lower id); then repeatedly take the
// unplaced vertex with the most placed neighbours (ties: fewer candidates,
// larger degree, lower id).
void order_strong(const QueryGraph& q, const GraphStats& gs, uint32_t* order) {
  auto cand = [&](uint32_t u) -> uint64_t {
    int c = gs.compact_label(q.label_raw[u]);
    return c < 0 ? 0 : gs.label_count[c];
  };
  auto nbr = [&](uint32_t u) { return (q.out_mask[u] | q.in_mask[u]) & ~(1u << u); };
  uint32_t placed = 0;
  for (uint32_t i = 0; i < q.k; ++i) {
    int best = -1;
    uint64_t bc = 0;
    int bb = -1, bd = -1;
    for (uint32_t u = 0; u < q.k; ++u) {
      if (placed >> u & 1) continue;
      int back = __builtin_popcount(nbr(u) & placed);
      int deg = __builtin_popcount(nbr(u));
      uint64_t c = cand(u);
      bool better;
      if (best < 0) better = true;
      else if (i > 0 && back != bb) better = back > bb;
      else if (c != bc) better = c < bc;
      else better = deg > bd;
      if (better) {
        best = int(u);
        bc = c;
        bb = back;
        bd = deg;
      }
    }
    order[i] = uint32_t(best);
    placed |= 1u << best;
  }
}

}  // namespace mg
