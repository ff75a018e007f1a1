// GAR pattern match over edge lists: the C entry matrixgraph_gar_match.
//
// The reference builds one candidate-edge list per pattern edge with vertex
// filters and joins them edge by edge into a capped frontier of partial
// matches (core/task/gpu_task/kernel/kernel_gar_match.cu:365-640), then
// groups the complete matches by pivot (:640-700).  Here the data edges that
// some pattern edge can use are gathered into a reference-layout CSR (the
// matching instance), the pattern is matched on the GPU by the label-sliced
// enumeration engine (count pass, then emit passes over level-0 ranges that
// fit the host budget), and the node columns are grouped by pivot on the
// host with the reference's ordering and capacity rules.
//
// Edge labels.  When the pattern uses a single edge label, or the data
// graph carries none, only the usable data edges enter the CSR and the match
// is a vertex-labelled one.  With two or more edge labels every usable data
// edge (s, d, l) becomes a vertex labelled by l with the edges s -> x -> d,
// and every distinct pattern edge likewise.  Distinct pattern edges differ
// in an endpoint or in the label, so an injective node map sends them to
// distinct data edges: the node columns of the subdivided matches are
// exactly the GAR matches, each once.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <tuple>
#include <vector>

#include "mg_gar_match.h"
#include "mg_internal.h"

namespace mg {
namespace {

struct GarOut {
  int* num_conditions;
  uint32_t* row_pivot_id;
  int32_t* row_cond_j;
  int32_t* row_pos;
  int32_t* row_offset;
  int32_t* row_count;
  int row_capacity;
  int* row_size;
  uint32_t* matched;
  int match_capacity;
  int* match_size;
};

// State the reference leaves when no match is written
// (kernel_gar_match.cu:497-508).
void put_empty(const GarOut& o) {
  if (o.num_conditions) *o.num_conditions = 1;
  if (o.row_size) *o.row_size = 0;
  if (o.match_size) *o.match_size = 0;
}

struct GarInputs {
  const uint32_t* v_id;
  const int32_t* v_label;
  int n;
  const uint32_t* src;
  const uint32_t* dst;
  const int32_t* elab;
  int m;
  const int32_t* p_lab;
  int p_n;
  const int32_t* p_src;
  const int32_t* p_dst;
  const int32_t* p_elab;
  int p_m;
};

// Matching instance of one (graph, pattern) pair.  Query vertices 0..k-1 are
// the pattern nodes; data vertices 0..n-1 are the graph's local indices.
struct GarInstance {
  bool empty = true;  // the answer is empty without matching
  uint32_t k = 0;     // pattern nodes
  HostCSR data;
  HostCSR* query = nullptr;  // owner returned by mg_query_from_edges
  mg_csr_view qv{};
  ~GarInstance() {
    if (query) mg_csr_dir_close(query);
  }
};

int build_instance(const GarInputs& in, GarInstance* I) {
  I->empty = true;
  // Inputs for which the reference finds no candidate edge, or no complete
  // match, give the empty result (kernel_gar_match.cu:386-387, :509-522): no
  // pattern edge, no data edge, a missing array, a pattern edge with an
  // endpoint out of range.
  if (in.p_n <= 0 || in.p_m <= 0) return MG_OK;
  if (in.n <= 0 || in.m <= 0 || !in.src || !in.dst || !in.p_src || !in.p_dst || !in.p_lab ||
      !in.v_label)
    return MG_OK;
  const uint32_t n = uint32_t(in.n), k = uint32_t(in.p_n);
  for (int j = 0; j < in.p_m; ++j)
    if (in.p_src[j] < 0 || in.p_src[j] >= in.p_n || in.p_dst[j] < 0 || in.p_dst[j] >= in.p_n)
      return MG_OK;
  if (k > MG_MAX_QUERY_VERTICES)
    return set_error(MG_E_LIMIT, "pattern has %u nodes; at most %d supported", k,
                     MG_MAX_QUERY_VERTICES);

  // Compact pattern node labels 0..Lp-1; data vertices with any other label
  // get Lp and can match no node.
  std::vector<int32_t> plabels;
  for (uint32_t u = 0; u < k; ++u)
    if (std::find(plabels.begin(), plabels.end(), in.p_lab[u]) == plabels.end())
      plabels.push_back(in.p_lab[u]);
  const uint32_t Lp = uint32_t(plabels.size());
  auto lab_of = [&](int32_t raw) -> uint32_t {
    for (uint32_t i = 0; i < Lp; ++i)
      if (plabels[i] == raw) return i;
    return Lp;
  };
  std::vector<uint32_t> qlab(k);
  for (uint32_t u = 0; u < k; ++u) qlab[u] = lab_of(in.p_lab[u]);

  // Edge labels of the pattern (compact 0..D-1).  Without data edge labels
  // every data edge serves every pattern edge.
  const bool use_elab = in.elab != nullptr;
  std::vector<int32_t> elabels;
  std::vector<uint32_t> pe_lab(in.p_m, 0);
  if (use_elab) {
    for (int j = 0; j < in.p_m; ++j) {
      const int32_t l = in.p_elab ? in.p_elab[j] : 0;
      auto it = std::find(elabels.begin(), elabels.end(), l);
      pe_lab[j] = uint32_t(it - elabels.begin());
      if (it == elabels.end()) elabels.push_back(l);
    }
  }
  const uint32_t D = use_elab ? uint32_t(elabels.size()) : 1u;
  const bool subdivide = D >= 2;

  // Usable (source label, target label, edge label) triples.
  auto key = [&](uint32_t cs, uint32_t cd, uint32_t e) {
    return (uint64_t(cs) * Lp + cd) * D + e;
  };
  std::vector<uint8_t> usable(uint64_t(Lp) * Lp * D, 0);
  for (int j = 0; j < in.p_m; ++j) usable[key(qlab[in.p_src[j]], qlab[in.p_dst[j]], pe_lab[j])] = 1;

  std::vector<uint32_t> vlab(n);
  for (uint32_t v = 0; v < n; ++v) vlab[v] = lab_of(in.v_label[v]);

  // Usable data edges, and per triple whether a self-loop (bit 0) or a
  // non-loop edge (bit 1) was seen: a pattern self-loop maps only onto a
  // data self-loop, any other pattern edge only onto a non-loop edge.
  std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> kept;
  std::vector<uint8_t> seen(usable.size(), 0);
  for (int e = 0; e < in.m; ++e) {
    const uint32_t s = in.src[e], d = in.dst[e];
    if (s >= n || d >= n) continue;
    const uint32_t cs = vlab[s], cd = vlab[d];
    if (cs == Lp || cd == Lp) continue;
    uint32_t el = 0;
    if (use_elab) {
      auto it = std::find(elabels.begin(), elabels.end(), in.elab[e]);
      if (it == elabels.end()) continue;
      el = uint32_t(it - elabels.begin());
    }
    const uint64_t kk = key(cs, cd, el);
    if (!usable[kk]) continue;
    seen[kk] |= s == d ? 1 : 2;
    kept.emplace_back(s, d, el);
  }
  // A pattern edge without a usable data edge, or a node on no pattern edge,
  // leaves every partial match incomplete: empty result.
  uint32_t covered = 0;
  for (int j = 0; j < in.p_m; ++j) {
    const uint32_t s = uint32_t(in.p_src[j]), d = uint32_t(in.p_dst[j]);
    covered |= 1u << s | 1u << d;
    if (!(seen[key(qlab[s], qlab[d], pe_lab[j])] & (s == d ? 1 : 2))) return MG_OK;
  }
  if (covered != (1u << k) - 1) return MG_OK;

  // Distinct pattern edges.
  std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> pedges;
  for (int j = 0; j < in.p_m; ++j)
    pedges.emplace_back(uint32_t(in.p_src[j]), uint32_t(in.p_dst[j]), subdivide ? pe_lab[j] : 0u);
  std::sort(pedges.begin(), pedges.end());
  pedges.erase(std::unique(pedges.begin(), pedges.end()), pedges.end());

  std::vector<uint32_t> src, dst, lab(vlab), qs, qd, ql(qlab);
  uint32_t kq = k;
  if (!subdivide) {
    src.reserve(kept.size());
    dst.reserve(kept.size());
    for (auto& t : kept) {
      src.push_back(std::get<0>(t));
      dst.push_back(std::get<1>(t));
    }
    for (auto& t : pedges) {
      qs.push_back(std::get<0>(t));
      qd.push_back(std::get<1>(t));
    }
  } else {
    if (k + pedges.size() > MG_MAX_QUERY_VERTICES)
      return set_error(MG_E_LIMIT,
                       "pattern with %u nodes and %zu distinct edges over %u edge labels: "
                       "at most %d nodes plus edges supported",
                       k, pedges.size(), D, MG_MAX_QUERY_VERTICES);
    std::sort(kept.begin(), kept.end());
    kept.erase(std::unique(kept.begin(), kept.end()), kept.end());
    if (uint64_t(n) + kept.size() >= 0xFFFFFFFFull)
      return set_error(MG_E_LIMIT, "%zu usable edges on %u vertices exceed 32-bit ids",
                       kept.size(), n);
    src.reserve(2 * kept.size());
    dst.reserve(2 * kept.size());
    lab.reserve(n + kept.size());
    uint32_t x = n;
    for (auto& t : kept) {
      src.push_back(std::get<0>(t));
      dst.push_back(x);
      src.push_back(x);
      dst.push_back(std::get<1>(t));
      lab.push_back(Lp + 1 + std::get<2>(t));
      ++x;
    }
    for (auto& t : pedges) {
      qs.push_back(std::get<0>(t));
      qd.push_back(kq);
      qs.push_back(kq);
      qd.push_back(std::get<1>(t));
      ql.push_back(Lp + 1 + std::get<2>(t));
      ++kq;
    }
  }
  int rc = build_csr_from_pairs(uint32_t(lab.size()), src.data(), dst.data(), src.size(),
                                lab.data(), MG_BUILD_DEDUP, &I->data);
  if (rc) return rc;
  void* owner = nullptr;
  if ((rc = mg_query_from_edges(kq, qs.data(), qd.data(), uint32_t(qs.size()), ql.data(), 1,
                                &I->qv, &owner)))
    return rc;
  I->query = static_cast<HostCSR*>(owner);
  I->k = k;
  I->empty = false;
  return MG_OK;
}

// Distinct (pivot, value) pairs of one pattern position, packed as
// pivot << 32 | value and kept sorted.
struct PosValues {
  std::vector<uint64_t> v;
  size_t sorted = 0;
  void compact() {
    if (sorted == v.size()) return;
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    sorted = v.size();
  }
};

// Adds match rows (row_width ids, the first k of them the pattern nodes).
void add_rows(std::vector<PosValues>& pv, const uint32_t* rows, uint64_t n_rows,
              uint32_t row_width) {
  const uint32_t k = uint32_t(pv.size());
  for (uint64_t i = 0; i < n_rows; ++i) {
    const uint32_t* row = rows + i * row_width;
    const uint64_t pivot = uint64_t(row[0]) << 32;
    for (uint32_t u = 0; u < k; ++u) pv[u].v.push_back(pivot | row[u]);
  }
  for (auto& p : pv)
    if (p.v.size() > 2 * p.sorted + (uint64_t(1) << 20)) p.compact();
}

// The grouped output of gar_match_arrays.h:14-51: one row per (pivot,
// position), pivots in ascending local-index order and positions 0..k-1 under
// each, every row a slice of the id pool holding that position's distinct
// instance ids under that pivot, ascending.  Output stops at the first
// capacity reached: no row starts once row_capacity rows exist, and the row
// that reaches match_capacity keeps only the ids that still fit (possibly
// none) and ends it.
void flatten(std::vector<PosValues>& pv, const uint32_t* v_id, uint32_t n, const GarOut& out) {
  const uint32_t k = uint32_t(pv.size());
  for (auto& p : pv) p.compact();
  auto inst = [&](uint32_t v) -> uint32_t { return v_id && v < n ? v_id[v] : v; };
  int rows = 0, ids = 0;
  // Appends one row; false once the output is complete.
  auto append = [&](uint32_t pivot, uint32_t pos, const std::vector<uint32_t>& vals) -> bool {
    if (rows >= out.row_capacity) return false;
    const int64_t room = std::max<int64_t>(0, int64_t(out.match_capacity) - ids);
    const int take = int(std::min<int64_t>(room, int64_t(vals.size())));
    if (out.row_pivot_id) out.row_pivot_id[rows] = pivot;
    if (out.row_cond_j) out.row_cond_j[rows] = int32_t(pos);
    if (out.row_pos) out.row_pos[rows] = int32_t(pos);
    if (out.row_offset) out.row_offset[rows] = ids;
    if (out.row_count) out.row_count[rows] = take;
    if (out.matched && take > 0) std::memcpy(out.matched + ids, vals.data(), size_t(take) * 4);
    ids += take;
    rows += 1;
    return rows < out.row_capacity && ids < out.match_capacity;
  };
  // Position cursors walk the packed (pivot << 32 | value) lists in step.
  std::vector<size_t> at(k, 0);
  std::vector<uint32_t> vals;
  const auto& piv = pv[0].v;  // (pivot, pivot): one entry per pivot
  bool more = true;
  for (size_t pi = 0; pi < piv.size() && more; ++pi) {
    const uint64_t pivot = piv[pi] >> 32;
    for (uint32_t pos = 0; pos < k && more; ++pos) {
      const auto& p = pv[pos].v;
      size_t c = at[pos];
      while (c < p.size() && (p[c] >> 32) < pivot) ++c;
      vals.clear();
      for (; c < p.size() && (p[c] >> 32) == pivot; ++c) vals.push_back(inst(uint32_t(p[c])));
      at[pos] = c;
      std::sort(vals.begin(), vals.end());
      vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
      more = append(inst(uint32_t(pivot)), pos, vals);
    }
  }
  if (out.row_size) *out.row_size = rows;
  if (out.match_size) *out.match_size = ids;
  if (out.num_conditions) *out.num_conditions = int(k);
}

struct GraphHandle {
  void* h = nullptr;
  ~GraphHandle() {
    if (h) mg_graph_free(h);
  }
};

int gar_match(const GarInputs& in, const GarOut& out, const mg_opts* user_opts,
              uint64_t* n_matches) {
  put_empty(out);
  if (n_matches) *n_matches = 0;
  if (user_opts && user_opts->order == MG_ORDER_GIVEN)
    return set_error(MG_E_ARG, "a given matching order is not accepted for GAR patterns");
  GarInstance I;
  int rc = build_instance(in, &I);
  if (rc || I.empty) return rc;
  const uint32_t k = I.k, kq = I.qv.n;
  mg_csr_view gv;
  I.data.fill_view(&gv);

  int device = 0;
  if ((rc = env_or_current_device(&device))) return rc;
  GraphHandle dgh;
  if ((rc = mg_graph_upload(&gv, device, &dgh.h))) return rc;

  mg_opts o;
  mg_opts_default(&o);
  if (user_opts) o = *user_opts;
  o.root_begin = o.root_end = 0;
  uint64_t total = 0;
  if ((rc = mg_subiso_count_ex(dgh.h, &I.qv, &o, &total, nullptr))) return rc;
  if (n_matches) *n_matches = total;
  if (total == 0) return MG_OK;

  // Emit passes.  A level-0 range whose matches exceed the host row budget
  // (2^28 ids, or MG_GAR_EMIT_ROWS rows when set) is split in halves; one
  // root beyond 2^31 matches is refused.
  uint64_t row_budget = std::max<uint64_t>(1, (uint64_t(1) << 28) / kq);
  if (const char* s = std::getenv("MG_GAR_EMIT_ROWS"))
    if (std::strtoull(s, nullptr, 10) > 0) row_budget = std::strtoull(s, nullptr, 10);
  std::vector<PosValues> pv(k);
  std::vector<uint32_t> rows;
  auto emit_range = [&](uint64_t rb, uint64_t re, uint64_t cnt) -> int {
    mg_opts oe = o;
    oe.root_begin = rb;
    oe.root_end = re;
    rows.assign(cnt * kq, 0);
    uint64_t got = 0;
    int r = mg_subiso_emit_ex(dgh.h, &I.qv, &oe, rows.data(), cnt, &got, nullptr);
    if (r) return r;
    if (got != cnt)
      return set_error(MG_E_CUDA, "emit returned %llu rows, count %llu", (unsigned long long)got,
                       (unsigned long long)cnt);
    add_rows(pv, rows.data(), cnt, kq);
    return MG_OK;
  };
  if (total <= row_budget) {
    if ((rc = emit_range(0, 0, total))) return rc;
  } else {
    std::vector<std::pair<uint64_t, uint64_t>> todo{{0, uint64_t(gv.n)}};
    while (!todo.empty()) {
      auto [rb, re] = todo.back();
      todo.pop_back();
      mg_opts oc = o;
      oc.root_begin = rb;
      oc.root_end = re;
      uint64_t cnt = 0;
      if ((rc = mg_subiso_count_ex(dgh.h, &I.qv, &oc, &cnt, nullptr))) return rc;
      if (cnt == 0) continue;
      if (cnt <= row_budget || re - rb == 1) {
        if (cnt >= (uint64_t(1) << 31))
          return set_error(MG_E_LIMIT, "one level-0 candidate holds %llu matches",
                           (unsigned long long)cnt);
        if ((rc = emit_range(rb, re, cnt))) return rc;
      } else {
        const uint64_t mid = rb + (re - rb) / 2;
        todo.emplace_back(mid, re);
        todo.emplace_back(rb, mid);
      }
    }
  }
  std::vector<uint32_t>().swap(rows);
  flatten(pv, in.v_id, uint32_t(in.n), out);
  return MG_OK;
}

}  // namespace
}  // namespace mg

extern "C" {

int mg_gar_match_ex(const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
                    const uint32_t* g_e_src, const uint32_t* g_e_dst, const uint32_t* g_e_id,
                    const int32_t* g_e_label_idx, int g_n_edges, const int32_t* p_node_label_idx,
                    int p_n_nodes, const int32_t* p_edge_src, const int32_t* p_edge_dst,
                    const int32_t* p_edge_label_idx, int p_n_edges, int* out_num_conditions,
                    uint32_t* out_row_pivot_id, int32_t* out_row_cond_j, int32_t* out_row_pos,
                    int32_t* out_row_offset, int32_t* out_row_count, int out_row_capacity,
                    int* out_row_size, uint32_t* out_matched_v_ids, int out_match_capacity,
                    int* out_match_size, const mg_opts* opts, uint64_t* n_matches) {
  (void)g_e_id;  // carried by the interface, never read (as in the reference)
  mg::clear_error();
  const mg::GarInputs in{g_v_id,    g_v_label_idx,    g_n_vertices, g_e_src,    g_e_dst,
                         g_e_label_idx, g_n_edges,   p_node_label_idx, p_n_nodes, p_edge_src,
                         p_edge_dst, p_edge_label_idx, p_n_edges};
  const mg::GarOut out{out_num_conditions, out_row_pivot_id, out_row_cond_j, out_row_pos,
                       out_row_offset,     out_row_count,    out_row_capacity, out_row_size,
                       out_matched_v_ids,  out_match_capacity, out_match_size};
  int rc;
  try {
    rc = mg::gar_match(in, out, opts, n_matches);
  } catch (const std::bad_alloc&) {
    rc = mg::set_error(MG_E_OOM, "host allocation failed");
  }
  if (rc) mg::put_empty(out);
  return rc;
}

int matrixgraph_gar_match(const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
                          const uint32_t* g_e_src, const uint32_t* g_e_dst,
                          const uint32_t* g_e_id, const int32_t* g_e_label_idx, int g_n_edges,
                          const int32_t* p_node_label_idx, int p_n_nodes,
                          const int32_t* p_edge_src, const int32_t* p_edge_dst,
                          const int32_t* p_edge_label_idx, int p_n_edges,
                          int* out_num_conditions, uint32_t* out_row_pivot_id,
                          int32_t* out_row_cond_j, int32_t* out_row_pos, int32_t* out_row_offset,
                          int32_t* out_row_count, int out_row_capacity, int* out_row_size,
                          uint32_t* out_matched_v_ids, int out_match_capacity,
                          int* out_match_size) {
  return mg_gar_match_ex(g_v_id, g_v_label_idx, g_n_vertices, g_e_src, g_e_dst, g_e_id,
                         g_e_label_idx, g_n_edges, p_node_label_idx, p_n_nodes, p_edge_src,
                         p_edge_dst, p_edge_label_idx, p_n_edges, out_num_conditions,
                         out_row_pivot_id, out_row_cond_j, out_row_pos, out_row_offset,
                         out_row_count, out_row_capacity, out_row_size, out_matched_v_ids,
                         out_match_capacity, out_match_size, nullptr, nullptr);
}

int mg_gar_instance(const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
                    const uint32_t* g_e_src, const uint32_t* g_e_dst,
                    const int32_t* g_e_label_idx, int g_n_edges, const int32_t* p_node_label_idx,
                    int p_n_nodes, const int32_t* p_edge_src, const int32_t* p_edge_dst,
                    const int32_t* p_edge_label_idx, int p_n_edges, mg_csr_view* data,
                    void** data_owner, mg_csr_view* query, void** query_owner) {
  mg::clear_error();
  if (!data || !data_owner || !query || !query_owner)
    return mg::set_error(MG_E_ARG, "null argument");
  *data_owner = *query_owner = nullptr;
  const mg::GarInputs in{g_v_id,    g_v_label_idx,    g_n_vertices, g_e_src,    g_e_dst,
                         g_e_label_idx, g_n_edges,   p_node_label_idx, p_n_nodes, p_edge_src,
                         p_edge_dst, p_edge_label_idx, p_n_edges};
  try {
    auto I = std::make_unique<mg::GarInstance>();
    int rc = mg::build_instance(in, I.get());
    if (rc || I->empty) return rc;
    auto* d = new mg::HostCSR(std::move(I->data));
    d->fill_view(data);
    *data_owner = d;
    *query = I->qv;
    *query_owner = I->query;
    I->query = nullptr;
    return MG_OK;
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_gar_flatten(const uint32_t* rows, uint64_t n_rows, uint32_t row_width, uint32_t n_nodes,
                   const uint32_t* g_v_id, int g_n_vertices, int* out_num_conditions,
                   uint32_t* out_row_pivot_id, int32_t* out_row_cond_j, int32_t* out_row_pos,
                   int32_t* out_row_offset, int32_t* out_row_count, int out_row_capacity,
                   int* out_row_size, uint32_t* out_matched_v_ids, int out_match_capacity,
                   int* out_match_size) {
  mg::clear_error();
  const mg::GarOut out{out_num_conditions, out_row_pivot_id, out_row_cond_j, out_row_pos,
                       out_row_offset,     out_row_count,    out_row_capacity, out_row_size,
                       out_matched_v_ids,  out_match_capacity, out_match_size};
  mg::put_empty(out);
  if ((n_rows && !rows) || n_nodes == 0 || row_width < n_nodes)
    return mg::set_error(MG_E_ARG, "bad rows");
  if (n_rows == 0) return MG_OK;
  try {
    std::vector<mg::PosValues> pv(n_nodes);
    mg::add_rows(pv, rows, n_rows, row_width);
    mg::flatten(pv, g_v_id, g_n_vertices < 0 ? 0u : uint32_t(g_n_vertices), out);
    return MG_OK;
  } catch (const std::bad_alloc&) {
    mg::put_empty(out);
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

}  // extern "C"
