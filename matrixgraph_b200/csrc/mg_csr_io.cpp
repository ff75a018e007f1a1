// Reference CSR directory format: reader, writer and builders.
//
// Layout follows ImmutableCSR::Read / Write / ParseBasePtr
// (core/data_structures/immutable_csr.cu:79-247) and the meta.yaml schema of
// core/common/yaml_config.h:43-110 / core/data_structures/metadata.h:39-66.
// The YAML subset written by that schema is parsed by a small reader written
// here (no yaml-cpp).
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <thread>
#include <unordered_map>
#include <sys/stat.h>

#include "mg_internal.h"

namespace mg {

static thread_local std::string g_err;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
void clear_error() { g_err.clear(); }
const char* last_error_cstr() { return g_err.c_str(); }

void HostCSR::fill_view(mg_csr_view* v) const {
  std::memset(v, 0, sizeof(*v));
  v->n = n;
  v->max_vid = max_vid;
  v->min_vid = min_vid;
  v->m_in = m_in;
  v->m_out = m_out;
  v->globalid = globalid.data();
  v->indeg = indeg.data();
  v->outdeg = outdeg.data();
  v->out_off = out_off.data();
  v->out_edges = out_edges.data();
  if (in_is_out) {
    v->in_off = out_off.data();
    v->in_edges = out_edges.data();
  } else {
    v->in_off = in_off.data();
    v->in_edges = in_edges.data();
  }
  v->edges_globalid_by_localid = eg_by_l.empty() ? nullptr : eg_by_l.data();
  v->localid_by_globalid = l_by_g.empty() ? nullptr : l_by_g.data();
  v->labels = labels.data();
}

// ---- minimal YAML reader for the GraphMetadata schema -----------------------
namespace {

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r");
  return s.substr(a, b - a + 1);
}

bool parse_u32(const std::string& s, uint32_t* out) {
  std::string t = trim(s);
  if (t.size() >= 2 && (t[0] == '"' || t[0] == '\''))
    t = t.substr(1, t.size() - 2);
  if (t.empty()) return false;
  uint64_t v = 0;
  for (char c : t) {
    if (c < '0' || c > '9') return false;
    v = v * 10 + uint64_t(c - '0');
    if (v > 0xFFFFFFFFull) return false;
  }
  *out = uint32_t(v);
  return true;
}

struct Meta {
  std::map<std::string, std::string> top;                 // GraphMetadata.*
  std::vector<std::map<std::string, std::string>> subs;   // subgraphs[*]
};

// Flow map "{a: 1, b: 2}" -> pairs.
void parse_flow_map(const std::string& s, std::map<std::string, std::string>* m) {
  std::string t = trim(s);
  if (!t.empty() && t.front() == '{') t = t.substr(1);
  if (!t.empty() && t.back() == '}') t.pop_back();
  std::stringstream ss(t);
  std::string item;
  while (std::getline(ss, item, ',')) {
    size_t c = item.find(':');
    if (c == std::string::npos) continue;
    (*m)[trim(item.substr(0, c))] = trim(item.substr(c + 1));
  }
}

int parse_meta(const std::string& text, Meta* meta) {
  std::stringstream ss(text);
  std::string line;
  bool in_gm = false, in_subs = false;
  size_t subs_indent = 0;
  while (std::getline(ss, line)) {
    size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    if (trim(line).empty() || trim(line) == "---" || trim(line) == "...")
      continue;
    size_t indent = line.find_first_not_of(' ');
    std::string body = line.substr(indent);
    if (indent == 0) {
      in_subs = false;
      std::string key = trim(body.substr(0, body.find(':')));
      in_gm = (key == "GraphMetadata");
      continue;
    }
    if (!in_gm) continue;
    bool item = false;
    if (body.rfind("- ", 0) == 0 || body == "-") {
      item = true;
      body = trim(body.substr(1));
      indent += 2;
    }
    if (in_subs && indent <= subs_indent && !item) in_subs = false;
    if (item && in_subs) {
      meta->subs.emplace_back();
      if (!body.empty() && body[0] == '{') {
        parse_flow_map(body, &meta->subs.back());
        continue;
      }
    }
    if (body.empty()) continue;
    size_t c = body.find(':');
    if (c == std::string::npos) return -1;
    std::string key = trim(body.substr(0, c));
    std::string val = trim(body.substr(c + 1));
    if (in_subs) {
      if (meta->subs.empty()) return -1;
      meta->subs.back()[key] = val;
      continue;
    }
    if (key == "subgraphs") {
      in_subs = true;
      subs_indent = indent;
      if (!val.empty() && val[0] == '[') {  // flow sequence
        std::string inner = val.substr(1, val.rfind(']') - 1);
        size_t p = 0;
        while ((p = inner.find('{', p)) != std::string::npos) {
          size_t e = inner.find('}', p);
          if (e == std::string::npos) return -1;
          meta->subs.emplace_back();
          parse_flow_map(inner.substr(p, e - p + 1), &meta->subs.back());
          p = e + 1;
        }
        in_subs = false;
      }
      continue;
    }
    meta->top[key] = val;
  }
  return 0;
}

bool file_size(const std::string& p, uint64_t* sz) {
  struct stat st;
  if (stat(p.c_str(), &st) != 0) return false;
  *sz = uint64_t(st.st_size);
  return true;
}

bool read_exact(std::ifstream& f, void* dst, uint64_t bytes) {
  char* p = static_cast<char*>(dst);
  while (bytes > 0) {
    uint64_t chunk = std::min<uint64_t>(bytes, 1ull << 30);
    f.read(p, std::streamsize(chunk));
    if (uint64_t(f.gcount()) != chunk) return false;
    p += chunk;
    bytes -= chunk;
  }
  return true;
}

bool write_all(std::ofstream& f, const void* src, uint64_t bytes) {
  const char* p = static_cast<const char*>(src);
  while (bytes > 0) {
    uint64_t chunk = std::min<uint64_t>(bytes, 1ull << 30);
    f.write(p, std::streamsize(chunk));
    if (!f) return false;
    p += chunk;
    bytes -= chunk;
  }
  return true;
}

}  // namespace

// Validates internal consistency of a reference-layout view.
static int validate_view(const mg_csr_view* v) {
  if (!v) return set_error(MG_E_ARG, "null csr view");
  if (v->n > 0 && (!v->globalid || !v->out_off || !v->in_off || !v->labels))
    return set_error(MG_E_ARG, "csr view has null arrays");
  if (v->m_out > 0 && !v->out_edges) return set_error(MG_E_ARG, "null out_edges");
  if (v->m_in > 0 && !v->in_edges) return set_error(MG_E_ARG, "null in_edges");
  if (v->n == 0) return MG_OK;
  if (v->out_off[0] != 0 || v->out_off[v->n] != v->m_out)
    return set_error(MG_E_FORMAT, "out_off does not span [0, m_out=%u]", v->m_out);
  if (v->in_off[0] != 0 || v->in_off[v->n] != v->m_in)
    return set_error(MG_E_FORMAT, "in_off does not span [0, m_in=%u]", v->m_in);
  for (uint32_t i = 0; i < v->n; ++i) {
    if (v->out_off[i + 1] < v->out_off[i] || v->in_off[i + 1] < v->in_off[i])
      return set_error(MG_E_FORMAT, "offsets decrease at vertex %u", i);
  }
  return MG_OK;
}

int validate_csr_view(const mg_csr_view* v) { return validate_view(v); }

static int read_dir(const std::string& dir, HostCSR* g) {
  std::string meta_path = dir + "meta.yaml";
  std::ifstream mf(meta_path);
  if (!mf) return set_error(MG_E_IO, "cannot open %s", meta_path.c_str());
  std::stringstream buf;
  buf << mf.rdbuf();
  Meta meta;
  if (parse_meta(buf.str(), &meta) != 0)
    return set_error(MG_E_FORMAT, "unparseable %s", meta_path.c_str());
  uint32_t nsub = 0;
  if (!meta.top.count("num_subgraphs") || !parse_u32(meta.top["num_subgraphs"], &nsub))
    return set_error(MG_E_FORMAT, "%s: GraphMetadata.num_subgraphs missing", meta_path.c_str());
  if (nsub != 1 || meta.subs.size() != 1)
    return set_error(MG_E_FORMAT, "%s: exactly one subgraph expected (num_subgraphs=%u, %zu listed)",
                     meta_path.c_str(), nsub, meta.subs.size());
  auto& s = meta.subs[0];
  const char* keys[6] = {"gid", "num_vertices", "num_incoming_edges",
                         "num_outgoing_edges", "max_vid", "min_vid"};
  uint32_t vals[6];
  if (s.size() != 6)
    return set_error(MG_E_FORMAT, "%s: subgraph entry has %zu keys, 6 expected",
                     meta_path.c_str(), s.size());
  for (int i = 0; i < 6; ++i) {
    if (!s.count(keys[i]) || !parse_u32(s[keys[i]], &vals[i]))
      return set_error(MG_E_FORMAT, "%s: subgraphs[0].%s missing or not a uint32",
                       meta_path.c_str(), keys[i]);
  }
  // The top-level fields must decode as uint32 too (yaml_config.h:96-103).
  const char* tkeys[4] = {"num_vertices", "num_edges", "max_vid", "min_vid"};
  for (auto* k : tkeys) {
    uint32_t tmp;
    if (!meta.top.count(k) || !parse_u32(meta.top[k], &tmp))
      return set_error(MG_E_FORMAT, "%s: GraphMetadata.%s missing or not a uint32",
                       meta_path.c_str(), k);
  }
  g->n = vals[1];
  g->m_in = vals[2];
  g->m_out = vals[3];
  g->max_vid = vals[4];
  g->min_vid = vals[5];
  const uint64_t n = g->n;
  const uint64_t nv = uint64_t(g->max_vid) + 1;
  std::string bin = dir + "graphs/0.bin", lab = dir + "label/0.bin";
  uint64_t bsz = 0, lsz = 0;
  if (!file_size(bin, &bsz)) return set_error(MG_E_IO, "cannot stat %s", bin.c_str());
  if (!file_size(lab, &lsz)) return set_error(MG_E_IO, "cannot stat %s", lab.c_str());
  const uint64_t core_words = 3 * n + 2 * (n + 1) + g->m_in + g->m_out;
  const uint64_t full_words = core_words + 2 * nv;
  if (bsz < core_words * 4 || bsz % 4 != 0)
    return set_error(MG_E_FORMAT, "%s: %llu bytes, at least %llu expected", bin.c_str(),
                     (unsigned long long)bsz, (unsigned long long)(core_words * 4));
  if (lsz < n * 4)
    return set_error(MG_E_FORMAT, "%s: %llu bytes, %llu expected", lab.c_str(),
                     (unsigned long long)lsz, (unsigned long long)(n * 4));
  std::ifstream bf(bin, std::ios::binary);
  if (!bf) return set_error(MG_E_IO, "cannot open %s", bin.c_str());
  auto rd = [&](std::vector<uint32_t>& v, uint64_t words) {
    v.resize(words);
    return read_exact(bf, v.data(), words * 4);
  };
  bool ok = rd(g->globalid, n) && rd(g->indeg, n) && rd(g->outdeg, n) &&
            rd(g->in_off, n + 1) && rd(g->out_off, n + 1) &&
            rd(g->in_edges, g->m_in) && rd(g->out_edges, g->m_out);
  if (ok && bsz >= full_words * 4) ok = rd(g->eg_by_l, nv) && rd(g->l_by_g, nv);
  if (!ok) return set_error(MG_E_IO, "short read of %s", bin.c_str());
  std::ifstream lf(lab, std::ios::binary);
  if (!lf) return set_error(MG_E_IO, "cannot open %s", lab.c_str());
  g->labels.resize(n);
  if (!read_exact(lf, g->labels.data(), n * 4))
    return set_error(MG_E_IO, "short read of %s", lab.c_str());
  mg_csr_view v;
  g->fill_view(&v);
  return validate_view(&v);
}

static bool mkdir_p(const std::string& d) {
  if (d.empty()) return true;
  struct stat st;
  if (stat(d.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
  return mkdir(d.c_str(), 0755) == 0 || errno == EEXIST;
}

static int write_dir(const std::string& dir, const mg_csr_view* v) {
  int rc = validate_view(v);
  if (rc) return rc;
  if (!mkdir_p(dir) || !mkdir_p(dir + "graphs") || !mkdir_p(dir + "label"))
    return set_error(MG_E_IO, "cannot create directories under %s", dir.c_str());
  std::ofstream bf(dir + "graphs/0.bin", std::ios::binary | std::ios::trunc);
  if (!bf) return set_error(MG_E_IO, "cannot write %sgraphs/0.bin", dir.c_str());
  const uint64_t n = v->n, nv = uint64_t(v->max_vid) + 1;
  std::vector<uint32_t> ident;
  auto ident_arr = [&]() -> const uint32_t* {
    if (ident.size() != nv) {
      ident.resize(nv);
      for (uint64_t i = 0; i < nv; ++i) ident[i] = uint32_t(i);
    }
    return ident.data();
  };
  // Degrees as stored (or recomputed from offsets when absent).
  std::vector<uint32_t> indeg, outdeg;
  const uint32_t* ind = v->indeg;
  const uint32_t* outd = v->outdeg;
  if (!ind) {
    indeg.resize(n);
    for (uint64_t i = 0; i < n; ++i) indeg[i] = v->in_off[i + 1] - v->in_off[i];
    ind = indeg.data();
  }
  if (!outd) {
    outdeg.resize(n);
    for (uint64_t i = 0; i < n; ++i) outdeg[i] = v->out_off[i + 1] - v->out_off[i];
    outd = outdeg.data();
  }
  bool ok = write_all(bf, v->globalid, n * 4) && write_all(bf, ind, n * 4) &&
            write_all(bf, outd, n * 4) && write_all(bf, v->in_off, (n + 1) * 4) &&
            write_all(bf, v->out_off, (n + 1) * 4) &&
            write_all(bf, v->in_edges, uint64_t(v->m_in) * 4) &&
            write_all(bf, v->out_edges, uint64_t(v->m_out) * 4) &&
            write_all(bf, v->edges_globalid_by_localid ? v->edges_globalid_by_localid : ident_arr(), nv * 4) &&
            write_all(bf, v->localid_by_globalid ? v->localid_by_globalid : ident_arr(), nv * 4);
  if (!ok) return set_error(MG_E_IO, "write failed: %sgraphs/0.bin", dir.c_str());
  bf.close();
  std::ofstream lf(dir + "label/0.bin", std::ios::binary | std::ios::trunc);
  if (!lf || !write_all(lf, v->labels, n * 4))
    return set_error(MG_E_IO, "write failed: %slabel/0.bin", dir.c_str());
  lf.close();
  std::ofstream mf(dir + "meta.yaml", std::ios::trunc);
  if (!mf) return set_error(MG_E_IO, "cannot write %smeta.yaml", dir.c_str());
  // num_edges is the uint32 sum of the reference (immutable_csr.cu:156-157).
  const uint32_t num_edges = uint32_t(v->m_in + v->m_out);
  mf << "GraphMetadata:\n"
     << "  num_vertices: " << v->n << "\n"
     << "  num_edges: " << num_edges << "\n"
     << "  max_vid: " << v->max_vid << "\n"
     << "  min_vid: " << v->min_vid << "\n"
     << "  count_border_vertices: 0\n"
     << "  num_subgraphs: 1\n"
     << "  subgraphs:\n"
     << "    - gid: 0\n"
     << "      num_vertices: " << v->n << "\n"
     << "      num_incoming_edges: " << v->m_in << "\n"
     << "      num_outgoing_edges: " << v->m_out << "\n"
     << "      max_vid: " << v->max_vid << "\n"
     << "      min_vid: " << v->min_vid << "\n";
  if (!mf) return set_error(MG_E_IO, "write failed: %smeta.yaml", dir.c_str());
  return MG_OK;
}

// ---- builder from directed pairs ---------------------------------------------
static unsigned hw_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t == 0 ? 1 : std::min(t, 64u);
}

template <class F>
static void parallel_for(uint64_t n, F f, unsigned threads = 0) {
  if (threads == 0) threads = hw_threads();
  if (n < 65536 || threads == 1) {
    f(0, n, 0u);
    return;
  }
  std::vector<std::thread> ts;
  uint64_t chunk = (n + threads - 1) / threads;
  for (unsigned t = 0; t < threads; ++t) {
    uint64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    ts.emplace_back([=, &f]() { f(a, b, t); });
  }
  for (auto& t : ts) t.join();
}

// Vertex ranges of about equal weight (list entries plus one per vertex,
// from the prefix offsets off64), handed out dynamically: hub-heavy id
// ranges (R-MAT ids are not permuted) no longer land on one thread.
template <class F>
static void parallel_for_volume(const std::vector<uint64_t>& off64, uint32_t n, F f) {
  const unsigned threads = hw_threads();
  const uint64_t total = off64[n] + n;
  if (total < 65536 || threads == 1) {
    f(0, n);
    return;
  }
  const uint32_t chunks = threads * 16;
  std::vector<uint32_t> bound(chunks + 1, n);
  bound[0] = 0;
  for (uint32_t c = 1; c < chunks; ++c) {
    const uint64_t target = total * c / chunks;
    uint32_t lo = bound[c - 1], hi = n;  // first v with off64[v] + v >= target
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (off64[mid] + mid < target)
        lo = mid + 1;
      else
        hi = mid;
    }
    bound[c] = lo;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> ts;
  for (unsigned t = 0; t < threads; ++t)
    ts.emplace_back([&]() {
      for (uint32_t c; (c = next.fetch_add(1)) < chunks;)
        if (bound[c] < bound[c + 1]) f(bound[c], bound[c + 1]);
    });
  for (auto& t : ts) t.join();
}

// One direction: CSR of (key -> val) pairs, sorted lists, optional dedup.
static int build_dir(uint32_t n, const uint32_t* key, const uint32_t* val,
                     uint64_t m, bool sym, uint32_t flags,
                     std::vector<uint32_t>& off, std::vector<uint32_t>& adj) {
  const bool no_self = flags & MG_BUILD_NO_SELF;
  const bool dedup = flags & MG_BUILD_DEDUP;
  std::vector<std::atomic<uint32_t>> cnt(n);
  for (auto& c : cnt) c.store(0, std::memory_order_relaxed);
  parallel_for(m, [&](uint64_t a, uint64_t b, unsigned) {
    for (uint64_t e = a; e < b; ++e) {
      uint32_t s = key[e], d = val[e];
      if (no_self && s == d) continue;
      cnt[s].fetch_add(1, std::memory_order_relaxed);
      if (sym && s != d) cnt[d].fetch_add(1, std::memory_order_relaxed);
    }
  });
  std::vector<uint64_t> off64(uint64_t(n) + 1, 0);
  for (uint32_t i = 0; i < n; ++i) off64[i + 1] = off64[i] + cnt[i].load();
  const uint64_t total = off64[n];
  if (total > 0xFFFFFFFFull)
    return set_error(MG_E_LIMIT, "adjacency of %llu entries exceeds uint32 offsets",
                     (unsigned long long)total);
  std::vector<uint32_t> tmp(total);
  for (uint32_t i = 0; i < n; ++i) cnt[i].store(uint32_t(off64[i]), std::memory_order_relaxed);
  parallel_for(m, [&](uint64_t a, uint64_t b, unsigned) {
    for (uint64_t e = a; e < b; ++e) {
      uint32_t s = key[e], d = val[e];
      if (no_self && s == d) continue;
      tmp[cnt[s].fetch_add(1, std::memory_order_relaxed)] = d;
      if (sym && s != d) tmp[cnt[d].fetch_add(1, std::memory_order_relaxed)] = s;
    }
  });
  // Sort (and optionally dedupe) each list; vertices split by edge volume.
  std::vector<uint32_t> newdeg(n);
  parallel_for_volume(off64, n, [&](uint64_t a, uint64_t b) {
    for (uint64_t v = a; v < b; ++v) {
      uint32_t* p = tmp.data() + off64[v];
      uint32_t* q = tmp.data() + off64[v + 1];
      std::sort(p, q);
      newdeg[v] = uint32_t(dedup ? (std::unique(p, q) - p) : (q - p));
    }
  });
  off.assign(uint64_t(n) + 1, 0);
  uint64_t acc = 0;
  for (uint32_t i = 0; i < n; ++i) {
    off[i] = uint32_t(acc);
    acc += newdeg[i];
  }
  off[n] = uint32_t(acc);
  if (acc == total) {
    adj.swap(tmp);
    return MG_OK;
  }
  adj.resize(acc);
  parallel_for_volume(off64, n, [&](uint64_t a, uint64_t b) {
    for (uint64_t v = a; v < b; ++v)
      std::memcpy(adj.data() + off[v], tmp.data() + off64[v], uint64_t(newdeg[v]) * 4);
  });
  return MG_OK;
}

int build_csr_from_pairs(uint32_t n, const uint32_t* src, const uint32_t* dst,
                         uint64_t m, const uint32_t* labels, uint32_t flags,
                         HostCSR* g) {
  std::atomic<uint64_t> bad{m};  // first edge with an endpoint out of range
  parallel_for(m, [&](uint64_t a, uint64_t b, unsigned) {
    for (uint64_t e = a; e < b; ++e)
      if (src[e] >= n || dst[e] >= n) {
        uint64_t cur = bad.load();
        while (e < cur && !bad.compare_exchange_weak(cur, e)) {
        }
        return;
      }
  });
  if (bad.load() < m) {
    const uint64_t e = bad.load();
    return set_error(MG_E_ARG, "edge %llu (%u,%u) out of range n=%u", (unsigned long long)e,
                     src[e], dst[e], n);
  }
  const bool sym = flags & MG_BUILD_SYMMETRIZE;
  int rc = build_dir(n, src, dst, m, sym, flags, g->out_off, g->out_edges);
  if (rc) return rc;
  g->n = n;
  g->m_out = g->out_off[n];
  if (sym) {
    g->in_is_out = true;
    g->m_in = g->m_out;
    g->in_off.clear();
    g->in_edges.clear();
  } else {
    rc = build_dir(n, dst, src, m, false, flags, g->in_off, g->in_edges);
    if (rc) return rc;
    g->in_is_out = false;
    g->m_in = g->in_off[n];
  }
  g->globalid.resize(n);
  g->outdeg.resize(n);
  g->indeg.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    g->globalid[i] = i;
    g->outdeg[i] = g->out_off[i + 1] - g->out_off[i];
    g->indeg[i] = sym ? g->outdeg[i] : g->in_off[i + 1] - g->in_off[i];
  }
  g->max_vid = n ? n - 1 : 0;
  g->min_vid = 0;
  g->eg_by_l.resize(uint64_t(g->max_vid) + 1);
  for (uint64_t i = 0; i < g->eg_by_l.size(); ++i) g->eg_by_l[i] = uint32_t(i);
  g->l_by_g = g->eg_by_l;
  g->labels.assign(n, 0);
  if (labels) std::memcpy(g->labels.data(), labels, uint64_t(n) * 4);
  return MG_OK;
}

// CSV "src,dst" -> first-appearance compaction (edgelist.cu:262-290), labels
// vid % label_range (edgelist.cu:425).  Keeps duplicates and self-loops, as the
// reference converter does.
static int csr_from_csv(const char* path, uint32_t label_range, HostCSR* g) {
  std::ifstream f(path);
  if (!f) return set_error(MG_E_IO, "cannot open %s", path);
  std::vector<uint32_t> raw;
  std::string line;
  while (std::getline(f, line)) {
    std::string t = trim(line);
    if (t.empty() || t[0] == '#') continue;
    for (char& c : t)
      if (c == ',' || c == '\t') c = ' ';
    std::stringstream ss(t);
    uint64_t a, b;
    if (!(ss >> a >> b) || a > 0xFFFFFFFFull || b > 0xFFFFFFFFull)
      return set_error(MG_E_FORMAT, "%s: bad edge line '%s'", path, line.c_str());
    raw.push_back(uint32_t(a));
    raw.push_back(uint32_t(b));
  }
  std::unordered_map<uint32_t, uint32_t> map;
  uint32_t next = 0;
  for (uint32_t x : raw)
    if (!map.count(x)) map[x] = next++;
  const uint64_t m = raw.size() / 2;
  std::vector<uint32_t> s(m), d(m);
  for (uint64_t e = 0; e < m; ++e) {
    s[e] = map[raw[2 * e]];
    d[e] = map[raw[2 * e + 1]];
  }
  std::vector<uint32_t> lab(next);
  if (label_range == 0) label_range = 1;
  for (uint32_t v = 0; v < next; ++v) lab[v] = v % label_range;
  return build_csr_from_pairs(next, s.data(), d.data(), m, lab.data(), 0, g);
}

}  // namespace mg

// ---- C-ABI -------------------------------------------------------------------
extern "C" {

int mg_csr_dir_open(const char* dir, mg_csr_view* out, void** owner) {
  mg::clear_error();
  if (!dir || !out || !owner) return mg::set_error(MG_E_ARG, "null argument");
  auto* g = new (std::nothrow) mg::HostCSR();
  if (!g) return mg::set_error(MG_E_OOM, "host allocation failed");
  int rc;
  try {
    rc = mg::read_dir(dir, g);
  } catch (const std::bad_alloc&) {
    rc = mg::set_error(MG_E_OOM, "host allocation failed reading %s", dir);
  }
  if (rc) {
    delete g;
    return rc;
  }
  g->fill_view(out);
  *owner = g;
  return MG_OK;
}

void mg_csr_dir_close(void* owner) { delete static_cast<mg::HostCSR*>(owner); }

int mg_csr_dir_write(const char* dir, const mg_csr_view* g) {
  mg::clear_error();
  if (!dir || !g) return mg::set_error(MG_E_ARG, "null argument");
  try {
    return mg::write_dir(dir, g);
  } catch (const std::bad_alloc&) {
    return mg::set_error(MG_E_OOM, "host allocation failed");
  }
}

int mg_csr_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst,
                      uint64_t m, const uint32_t* labels, uint32_t flags,
                      mg_csr_view* out, void** owner) {
  mg::clear_error();
  if ((m && (!src || !dst)) || !out || !owner) return mg::set_error(MG_E_ARG, "null argument");
  auto* g = new (std::nothrow) mg::HostCSR();
  if (!g) return mg::set_error(MG_E_OOM, "host allocation failed");
  int rc;
  try {
    rc = mg::build_csr_from_pairs(n, src, dst, m, labels, flags, g);
  } catch (const std::bad_alloc&) {
    rc = mg::set_error(MG_E_OOM, "host allocation failed");
  }
  if (rc) {
    delete g;
    return rc;
  }
  g->fill_view(out);
  *owner = g;
  return MG_OK;
}

int mg_csr_from_csv(const char* csv_path, uint32_t label_range, mg_csr_view* out,
                    void** owner) {
  mg::clear_error();
  if (!csv_path || !out || !owner) return mg::set_error(MG_E_ARG, "null argument");
  auto* g = new (std::nothrow) mg::HostCSR();
  if (!g) return mg::set_error(MG_E_OOM, "host allocation failed");
  int rc = mg::csr_from_csv(csv_path, label_range, g);
  if (rc) {
    delete g;
    return rc;
  }
  g->fill_view(out);
  *owner = g;
  return MG_OK;
}

}  // extern "C"
