// Seeded synthetic inputs: Chung-Lu and R-MAT data graphs, uniform and Zipf
// vertex labels, and labelled queries whose labels come from random walks on
// the data graph.  Every draw is a pure function of (seed, index) through
// Philox4x32-10, so results do not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "mg_internal.h"

namespace mg {

// Philox4x32-10 as published by Salmon et al. (SC'11): ten rounds of two
// 32x32->64 multiplies with the round keys bumped by the Weyl constants.
Philox4 philox4x32_10(uint64_t key, uint64_t ctr_lo, uint64_t ctr_hi) {
  uint32_t c0 = uint32_t(ctr_lo), c1 = uint32_t(ctr_lo >> 32);
  uint32_t c2 = uint32_t(ctr_hi), c3 = uint32_t(ctr_hi >> 32);
  uint32_t k0 = uint32_t(key), k1 = uint32_t(key >> 32);
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = uint64_t(M0) * c0;
    uint64_t p1 = uint64_t(M1) * c2;
    uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  return Philox4{{c0, c1, c2, c3}};
}

static unsigned pick_threads(uint32_t t) {
  unsigned h = std::thread::hardware_concurrency();
  if (h == 0) h = 1;
  if (t == 0) t = h;
  return std::max(1u, std::min<unsigned>(t, 256));
}

// ---- Chung-Lu -----------------------------------------------------------------
static int gen_chung_lu(uint32_t n, double beta, double avg_deg, uint64_t seed,
                        uint32_t threads, std::vector<uint32_t>& src,
                        std::vector<uint32_t>& dst) {
  if (n < 2 || beta <= 1.0 || avg_deg <= 0)
    return set_error(MG_E_ARG, "chung-lu needs n>=2, beta>1, avg_deg>0");
  std::vector<double> w(n);
  const double ex = -1.0 / (beta - 1.0);
  double sum = 0;
  for (uint32_t i = 0; i < n; ++i) {
    w[i] = std::pow(double(i + 1), ex);
    sum += w[i];
  }
  const double target = double(n) * avg_deg;
  const double c = target / sum;
  for (auto& x : w) x *= c;
  const double S = target;
  unsigned T = pick_threads(threads);
  std::vector<std::vector<uint32_t>> ls(T), ld(T);
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < T; ++t) {
    ts.emplace_back([&, t]() {
      // Rows i interleaved across threads; the pair (i,j) uses counter i*n+j.
      for (uint64_t i = t; i < n; i += T) {
        for (uint64_t j = i + 1; j < n; ++j) {
          double p = w[i] * w[j] / S;
          if (p >= 1.0) {
            ls[t].push_back(uint32_t(i));
            ld[t].push_back(uint32_t(j));
            continue;
          }
          Philox4 r = philox4x32_10(seed, i * uint64_t(n) + j, 0x434C00ull);
          if (u53(r.v[0], r.v[1]) < p) {
            ls[t].push_back(uint32_t(i));
            ld[t].push_back(uint32_t(j));
          }
        }
      }
    });
  }
  for (auto& th : ts) th.join();
  for (unsigned t = 0; t < T; ++t) {
    src.insert(src.end(), ls[t].begin(), ls[t].end());
    dst.insert(dst.end(), ld[t].begin(), ld[t].end());
  }
  return MG_OK;
}

// ---- R-MAT ----------------------------------------------------------------------
static int gen_rmat(uint32_t scale, uint32_t ef, double a, double b, double c,
                    uint64_t seed, uint32_t threads, uint32_t* src,
                    uint32_t* dst) {
  const uint64_t m = uint64_t(ef) << scale;
  // Integer thresholds so the quadrant choice is exact integer arithmetic.
  const uint64_t two32 = 1ull << 32;
  const uint64_t ta = uint64_t(std::floor(a * double(two32)));
  const uint64_t tab = uint64_t(std::floor((a + b) * double(two32)));
  const uint64_t tabc = uint64_t(std::floor((a + b + c) * double(two32)));
  unsigned T = pick_threads(threads);
  std::vector<std::thread> ts;
  const uint64_t chunk = (m + T - 1) / T;
  for (unsigned t = 0; t < T; ++t) {
    ts.emplace_back([&, t]() {
      uint64_t lo = t * chunk, hi = std::min(m, lo + chunk);
      for (uint64_t e = lo; e < hi; ++e) {
        uint32_t s = 0, d = 0;
        Philox4 r{};
        for (uint32_t l = 0; l < scale; ++l) {
          if ((l & 3) == 0) r = philox4x32_10(seed, e, 0x524D00ull + (l >> 2));
          uint64_t u = r.v[l & 3];
          uint32_t bit = 1u << (scale - 1 - l);
          if (u < ta) {
          } else if (u < tab) {
            d |= bit;
          } else if (u < tabc) {
            s |= bit;
          } else {
            s |= bit;
            d |= bit;
          }
        }
        src[e] = s;
        dst[e] = d;
      }
    });
  }
  for (auto& th : ts) th.join();
  return MG_OK;
}

// ---- labels -----------------------------------------------------------------------
static int gen_labels(uint32_t n, uint32_t kind, uint32_t L, double s,
                      uint64_t seed, uint32_t* labels) {
  if (L == 0) return set_error(MG_E_ARG, "label count must be > 0");
  std::vector<double> cdf;
  if (kind == 1) {
    cdf.resize(L);
    double acc = 0;
    for (uint32_t k = 0; k < L; ++k) {
      acc += std::pow(double(k + 1), -s);
      cdf[k] = acc;
    }
    for (auto& x : cdf) x /= acc;
    cdf[L - 1] = 1.0;
  }
  for (uint64_t v = 0; v < n; ++v) {
    Philox4 r = philox4x32_10(seed, v, 0x4C4200ull);
    if (kind == 0) {
      labels[v] = uint32_t((uint64_t(r.v[0]) * L) >> 32);
    } else {
      double u = u53(r.v[0], r.v[1]);
      labels[v] = uint32_t(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
      if (labels[v] >= L) labels[v] = L - 1;
    }
  }
  return MG_OK;
}

// ---- queries ------------------------------------------------------------------------
// Maps a global id of the data graph to its local id (identity fast path).
struct G2L {
  const mg_csr_view* g;
  std::vector<uint32_t> map;
  bool ident = true;
  explicit G2L(const mg_csr_view* gv) : g(gv) {
    for (uint32_t i = 0; i < g->n; ++i)
      if (g->globalid[i] != i) {
        ident = false;
        break;
      }
    if (!ident) {
      map.assign(uint64_t(g->max_vid) + 1, 0xFFFFFFFFu);
      for (uint32_t i = 0; i < g->n; ++i)
        if (g->globalid[i] <= g->max_vid) map[g->globalid[i]] = i;
    }
  }
  uint32_t operator()(uint32_t gid) const {
    if (ident) return gid;
    return gid < map.size() ? map[gid] : 0xFFFFFFFFu;
  }
};

// Labels by a random walk along the BFS spanning tree of the query from 0.
static int walk_labels(const mg_csr_view* g, uint32_t k,
                       const std::vector<uint32_t>& adjmask, uint64_t seed,
                       std::vector<uint32_t>& qlab) {
  if (g->n == 0 || g->m_out == 0) return set_error(MG_E_ARG, "data graph has no edges");
  G2L g2l(g);
  RngStream rng(seed, 0x57414C4Bull);
  uint32_t start = 0;
  bool found = false;
  for (int tries = 0; tries < 1 << 20; ++tries) {
    uint32_t v = rng.below(g->n);
    if (g->out_off[v + 1] > g->out_off[v]) {
      start = v;
      found = true;
      break;
    }
  }
  if (!found) return set_error(MG_E_ARG, "no vertex with out-degree > 0 found");
  std::vector<uint32_t> img(k, 0xFFFFFFFFu), queue;
  img[0] = start;
  queue.push_back(0);
  for (size_t h = 0; h < queue.size(); ++h) {
    uint32_t p = queue[h];
    for (uint32_t c = 0; c < k; ++c) {
      if (!(adjmask[p] >> c & 1) || img[c] != 0xFFFFFFFFu) continue;
      uint32_t x = img[p];
      uint32_t deg = g->out_off[x + 1] - g->out_off[x];
      if (deg == 0) {
        img[c] = x;  // dead end: stay (label copied from x)
      } else {
        uint32_t nb = g->out_edges[g->out_off[x] + rng.below(deg)];
        uint32_t l = g2l(nb);
        img[c] = (l == 0xFFFFFFFFu) ? x : l;
      }
      queue.push_back(c);
    }
  }
  qlab.resize(k);
  for (uint32_t u = 0; u < k; ++u) {
    uint32_t x = img[u] == 0xFFFFFFFFu ? start : img[u];
    qlab[u] = g->labels[x];
  }
  return MG_OK;
}

static int make_query(uint32_t k, const std::vector<std::pair<uint32_t, uint32_t>>& und,
                      const std::vector<uint32_t>& lab, bool directed, HostCSR* q) {
  std::vector<uint32_t> s, d;
  for (auto& e : und) {
    s.push_back(e.first);
    d.push_back(e.second);
  }
  uint32_t flags = MG_BUILD_DEDUP | (directed ? 0u : MG_BUILD_SYMMETRIZE);
  int rc = build_csr_from_pairs(k, s.data(), d.data(), s.size(), lab.data(), flags, q);
  if (rc) return rc;
  if (q->in_is_out) {  // queries are stored with explicit in-arrays
    q->in_off = q->out_off;
    q->in_edges = q->out_edges;
    q->in_is_out = false;
  }
  return MG_OK;
}

}  // namespace mg

extern "C" {

int mg_gen_chung_lu(uint32_t n, double beta, double avg_deg, uint64_t seed,
                    uint32_t threads, uint32_t** src, uint32_t** dst, uint64_t* m) {
  mg::clear_error();
  if (!src || !dst || !m) return mg::set_error(MG_E_ARG, "null argument");
  std::vector<uint32_t> s, d;
  int rc = mg::gen_chung_lu(n, beta, avg_deg, seed, threads, s, d);
  if (rc) return rc;
  *m = s.size();
  *src = static_cast<uint32_t*>(std::malloc(std::max<size_t>(1, s.size()) * 4));
  *dst = static_cast<uint32_t*>(std::malloc(std::max<size_t>(1, d.size()) * 4));
  if (!*src || !*dst) return mg::set_error(MG_E_OOM, "host allocation failed");
  std::memcpy(*src, s.data(), s.size() * 4);
  std::memcpy(*dst, d.data(), d.size() * 4);
  return MG_OK;
}

int mg_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                uint64_t seed, uint32_t threads, uint32_t** src, uint32_t** dst,
                uint64_t* m) {
  mg::clear_error();
  if (!src || !dst || !m) return mg::set_error(MG_E_ARG, "null argument");
  if (scale == 0 || scale > 31 || edge_factor == 0)
    return mg::set_error(MG_E_ARG, "rmat needs 1 <= scale <= 31, edge_factor > 0");
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return mg::set_error(MG_E_ARG, "rmat probabilities invalid");
  const uint64_t mm = uint64_t(edge_factor) << scale;
  *src = static_cast<uint32_t*>(std::malloc(mm * 4));
  *dst = static_cast<uint32_t*>(std::malloc(mm * 4));
  if (!*src || !*dst) {
    std::free(*src);
    std::free(*dst);
    return mg::set_error(MG_E_OOM, "host allocation of %llu edges failed", (unsigned long long)mm);
  }
  *m = mm;
  return mg::gen_rmat(scale, edge_factor, a, b, c, seed, threads, *src, *dst);
}

void mg_free_buffer(void* p) { std::free(p); }

int mg_gen_labels(uint32_t n, uint32_t kind, uint32_t L, double s, uint64_t seed,
                  uint32_t* labels) {
  mg::clear_error();
  if (!labels && n) return mg::set_error(MG_E_ARG, "null labels");
  return mg::gen_labels(n, kind, L, s, seed, labels);
}

int mg_gen_query_walk(const mg_csr_view* g, uint32_t k, const uint32_t* eu,
                      const uint32_t* ev, uint32_t ne, uint64_t seed,
                      mg_csr_view* out, void** owner) {
  mg::clear_error();
  if (!g || !out || !owner || (ne && (!eu || !ev)))
    return mg::set_error(MG_E_ARG, "null argument");
  if (k == 0 || k > MG_MAX_QUERY_VERTICES) return mg::set_error(MG_E_LIMIT, "k=%u out of range", k);
  std::vector<std::pair<uint32_t, uint32_t>> und;
  std::vector<uint32_t> adj(k, 0);
  for (uint32_t i = 0; i < ne; ++i) {
    if (eu[i] >= k || ev[i] >= k) return mg::set_error(MG_E_ARG, "query edge out of range");
    und.emplace_back(eu[i], ev[i]);
    adj[eu[i]] |= 1u << ev[i];
    adj[ev[i]] |= 1u << eu[i];
  }
  std::vector<uint32_t> lab;
  int rc = mg::walk_labels(g, k, adj, seed, lab);
  if (rc) return rc;
  auto* q = new mg::HostCSR();
  rc = mg::make_query(k, und, lab, false, q);
  if (rc) {
    delete q;
    return rc;
  }
  q->fill_view(out);
  *owner = q;
  return MG_OK;
}

int mg_gen_query_random(const mg_csr_view* g, uint32_t k, double p_extra,
                        uint64_t seed, mg_csr_view* out, void** owner) {
  mg::clear_error();
  if (!g || !out || !owner) return mg::set_error(MG_E_ARG, "null argument");
  if (k == 0 || k > MG_MAX_QUERY_VERTICES) return mg::set_error(MG_E_LIMIT, "k=%u out of range", k);
  mg::RngStream rng(seed, 0x51525900ull);
  std::vector<std::pair<uint32_t, uint32_t>> und;
  std::vector<uint32_t> adj(k, 0);
  for (uint32_t j = 1; j < k; ++j) {
    uint32_t p = rng.below(j);
    und.emplace_back(p, j);
    adj[p] |= 1u << j;
    adj[j] |= 1u << p;
  }
  for (uint32_t i = 0; i < k; ++i)
    for (uint32_t j = i + 1; j < k; ++j) {
      if (adj[i] >> j & 1) continue;
      if (rng.uniform() < p_extra) {
        und.emplace_back(i, j);
        adj[i] |= 1u << j;
        adj[j] |= 1u << i;
      }
    }
  std::vector<uint32_t> lab;
  int rc = mg::walk_labels(g, k, adj, seed ^ 0x9E3779B97F4A7C15ull, lab);
  if (rc) return rc;
  auto* q = new mg::HostCSR();
  rc = mg::make_query(k, und, lab, false, q);
  if (rc) {
    delete q;
    return rc;
  }
  q->fill_view(out);
  *owner = q;
  return MG_OK;
}

int mg_query_from_edges(uint32_t k, const uint32_t* eu, const uint32_t* ev, uint32_t ne,
                        const uint32_t* labels, int directed, mg_csr_view* out,
                        void** owner) {
  mg::clear_error();
  if (!out || !owner || !labels || (ne && (!eu || !ev)))
    return mg::set_error(MG_E_ARG, "null argument");
  if (k == 0 || k > MG_MAX_QUERY_VERTICES) return mg::set_error(MG_E_LIMIT, "k=%u out of range", k);
  std::vector<std::pair<uint32_t, uint32_t>> und;
  for (uint32_t i = 0; i < ne; ++i) {
    if (eu[i] >= k || ev[i] >= k) return mg::set_error(MG_E_ARG, "query edge out of range");
    und.emplace_back(eu[i], ev[i]);
  }
  std::vector<uint32_t> lab(labels, labels + k);
  auto* q = new mg::HostCSR();
  int rc = mg::make_query(k, und, lab, directed != 0, q);
  if (rc) {
    delete q;
    return rc;
  }
  q->fill_view(out);
  *owner = q;
  return MG_OK;
}

}  // extern "C"
