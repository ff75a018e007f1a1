/*
 * oracle.c — CPU restatement of exact labelled subgraph matching.
 *
 * TEST INFRASTRUCTURE ONLY.  Used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py as the checker and as the
 * timed CPU port.  Nothing in the product links or calls it.
 *
 * What it restates (hsiaoko/MatrixGraph, paths relative to the project):
 *   - the binary CSR directory format: core/data_structures/immutable_csr.cu
 *     :168-247 (Read), metadata.h:39-66, core/common/yaml_config.h:85-110;
 *     adjacency entries are global ids (core/util/format_converter.cuh
 *     :166-184), mapped back to local ids through globalid[];
 *   - the matching rule of the only exact reference matcher,
 *     core/task/gpu_task/kernel/kernel_gar_match.cu:325-363: endpoint
 *     consistency of every pattern edge plus injectivity, non-induced;
 *   - the sound candidate predicates: label and degree
 *     (kernel_woj_subsio.cu:123-138) and neighbour labels, taken as a subset
 *     test of the neighbour-label set (the reference's popcount form at
 *     kernel_woj_subsio.cu:385-446 is weaker);
 *   - the reference heuristic order: pattern edges in CSR order
 *     (core/data_structures/woj_exec_plan.cuh:36-45), vertex introduction as
 *     in the join chain (kernel_woj_subsio.cu:942-1049), with disconnected
 *     edges rescanned instead of skipped (:1006-1008).
 *
 * Backtracking, depth first, one root (level-0 candidate) per task over
 * pthreads.  It also computes the per-prefix counts P_i and the algorithmic
 * byte count B_alg of the enumeration for a given order:
 *   B_alg = |L0| (4 + 8 + 4W)
 *         + sum_{i=1..k-1} sum_{m in P_i} sum_{(w,d) in B(u_i)} (8 + 4 |N^d_l(u_i)(m(w))|)
 * and B_alg_count, equal except that a last position with exactly one
 * backward neighbour and no self-loop is charged 8 bytes per prefix.
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_MAXK 16
#define ORC_OK 0
#define ORC_E_IO -1
#define ORC_E_FORMAT -2
#define ORC_E_OOM -3
#define ORC_E_ARG -7

typedef struct orc_graph {
  uint32_t n, L, W;
  int symmetric;
  uint32_t* label;        /* compact label per local vertex */
  uint32_t* label_values; /* compact -> raw, ascending */
  uint32_t* globalid;
  uint32_t* adj[2];       /* per direction: lists ordered by (label, id) */
  uint32_t* loff[2];      /* n*L + 1 slice starts (the format's uint32 offsets) */
  uint32_t* deg[2];
  uint32_t* nlb[2];       /* n*W */
  uint32_t* bucket_off;   /* L + 1 */
  uint32_t* bucket_vid;   /* ascending id per label */
  uint8_t* self;
} orc_graph;

typedef struct orc_query {
  uint32_t k;
  uint32_t label_raw[ORC_MAXK];
  uint32_t out_mask[ORC_MAXK];
  uint32_t n_edges;
  uint32_t esrc[ORC_MAXK * ORC_MAXK], edst[ORC_MAXK * ORC_MAXK]; /* CSR order */
} orc_query;

typedef struct orc_result {
  uint64_t count;
  uint64_t level_rows[ORC_MAXK + 1];
  uint64_t balg, balg_count;
} orc_result;

/* ---------------------------------------------------------------- graph -- */
static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : x > y;
}

static const uint32_t* g_sort_labels;
static int cmp_lab_id(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  uint32_t lx = g_sort_labels[x], ly = g_sort_labels[y];
  if (lx != ly) return lx < ly ? -1 : 1;
  return x < y ? -1 : x > y;
}

void orc_graph_free(orc_graph* g) {
  if (!g) return;
  free(g->label);
  free(g->label_values);
  free(g->globalid);
  for (int d = 0; d < 2; ++d) {
    free(g->adj[d]);
    free(g->loff[d]);
    free(g->deg[d]);
    free(g->nlb[d]);
    if (g->symmetric) break;
  }
  free(g->bucket_off);
  free(g->bucket_vid);
  free(g->self);
  free(g);
}

/* Vertex-parallel loop: fn(ctx, v) for v in [0, n) over the host's cores,
 * in interleaved blocks of 256 vertices. */
typedef struct par_job {
  uint32_t n, t, nt;
  void (*fn)(void*, uint32_t);
  void* ctx;
} par_job;

static void* par_run(void* arg) {
  par_job* J = (par_job*)arg;
  for (uint64_t b = (uint64_t)J->t * 256; b < J->n; b += (uint64_t)J->nt * 256) {
    uint64_t e = b + 256 < J->n ? b + 256 : J->n;
    for (uint64_t v = b; v < e; ++v) J->fn(J->ctx, (uint32_t)v);
  }
  return NULL;
}

static void par_for(uint32_t n, void (*fn)(void*, uint32_t), void* ctx) {
  long h = sysconf(_SC_NPROCESSORS_ONLN);
  uint32_t nt = h < 1 ? 1 : (uint32_t)(h > 256 ? 256 : h);
  if (n < 4096) nt = 1;
  par_job jobs[256];
  pthread_t th[256];
  for (uint32_t t = 0; t < nt; ++t) {
    jobs[t].n = n;
    jobs[t].t = t;
    jobs[t].nt = nt;
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
  }
  if (nt == 1) {
    par_run(&jobs[0]);
    return;
  }
  for (uint32_t t = 0; t < nt; ++t) pthread_create(&th[t], NULL, par_run, &jobs[t]);
  for (uint32_t t = 0; t < nt; ++t) pthread_join(th[t], NULL);
}

typedef struct norm_ctx {
  const uint32_t *off, *edges, *g2l;
  uint32_t max_vid;
  uint32_t* a;
  uint64_t* uniq;
  atomic_int bad;
} norm_ctx;

static void norm_vertex(void* p, uint32_t v) {
  norm_ctx* c = (norm_ctx*)p;
  const uint64_t s = c->off[v], e = c->off[v + 1];
  for (uint64_t j = s; j < e; ++j) {
    const uint32_t gid = c->edges[j];
    if (gid > c->max_vid || c->g2l[gid] == UINT32_MAX) {
      atomic_store(&c->bad, 1);
      c->uniq[v] = 0;
      return;
    }
    c->a[j] = c->g2l[gid];
  }
  qsort(c->a + s, e - s, 4, cmp_u32);
  uint64_t u = s;
  for (uint64_t j = s; j < e; ++j)
    if (j == s || c->a[j] != c->a[j - 1]) c->a[u++] = c->a[j];
  c->uniq[v] = u - s;
}

/* Local adjacency of one direction: map ids, sort, drop repeats. */
static int normalise_dir(uint32_t n, const uint32_t* off, const uint32_t* edges,
                         const uint32_t* g2l, uint32_t max_vid, uint64_t** noff,
                         uint32_t** nadj) {
  uint64_t m = off[n];
  uint64_t* o = (uint64_t*)calloc((size_t)n + 1, 8);
  uint32_t* a = (uint32_t*)malloc((m ? m : 1) * 4);
  if (!o || !a) return ORC_E_OOM;
  norm_ctx c = {off, edges, g2l, max_vid, a, o, 0};
  par_for(n, norm_vertex, &c); /* o[v] = distinct entries of v */
  if (atomic_load(&c.bad)) {
    free(o);
    free(a);
    return ORC_E_FORMAT;
  }
  uint64_t w = 0;
  for (uint32_t v = 0; v < n; ++v) {
    const uint64_t u = o[v];
    if (w != off[v]) memmove(a + w, a + off[v], u * 4);
    o[v] = w;
    w += u;
  }
  o[n] = w;
  *noff = o;
  *nadj = a;
  return ORC_OK;
}

typedef struct slice_ctx {
  orc_graph* g;
  int d;
  const uint64_t* off;
  uint32_t* adj;
} slice_ctx;

/* One vertex's list ordered by (label, id), its label-slice starts, degree,
 * neighbour-label bits and self-loop flag. */
static void slice_vertex(void* p, uint32_t v) {
  slice_ctx* c = (slice_ctx*)p;
  orc_graph* g = c->g;
  const int d = c->d;
  const uint32_t L = g->L, W = g->W;
  const uint64_t s = c->off[v], e = c->off[v + 1];
  g->deg[d][v] = (uint32_t)(e - s);
  for (uint64_t j = s; j < e; ++j)
    if (c->adj[j] == v) g->self[v] = 1;
  qsort(c->adj + s, e - s, 4, cmp_lab_id);
  uint64_t q = s;
  for (uint32_t l = 0; l < L; ++l) {
    g->loff[d][(uint64_t)v * L + l] = (uint32_t)q;
    while (q < e && g->label[c->adj[q]] == l) ++q;
    if (g->loff[d][(uint64_t)v * L + l] < q) g->nlb[d][(uint64_t)v * W + l / 32] |= 1u << (l % 32);
  }
}

orc_graph* orc_graph_from_arrays(uint32_t n, uint32_t max_vid, const uint32_t* globalid,
                                 const uint32_t* out_off, const uint32_t* out_edges,
                                 const uint32_t* in_off, const uint32_t* in_edges,
                                 const uint32_t* labels, int* err) {
  *err = ORC_OK;
  orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
  uint32_t* g2l = (uint32_t*)malloc(((size_t)max_vid + 1) * 4);
  if (!g || !g2l || n == 0) {
    *err = n == 0 ? ORC_E_ARG : ORC_E_OOM;
    free(g);
    free(g2l);
    return NULL;
  }
  memset(g2l, 0xFF, ((size_t)max_vid + 1) * 4);
  g->n = n;
  g->globalid = (uint32_t*)malloc((size_t)n * 4);
  memcpy(g->globalid, globalid, (size_t)n * 4);
  for (uint32_t i = 0; i < n; ++i) {
    if (globalid[i] > max_vid) {
      *err = ORC_E_FORMAT;
      goto fail;
    }
    g2l[globalid[i]] = i;
  }
  /* label compaction: sorted distinct raw labels */
  {
    uint32_t* tmp = (uint32_t*)malloc((size_t)n * 4);
    memcpy(tmp, labels, (size_t)n * 4);
    qsort(tmp, n, 4, cmp_u32);
    uint32_t L = 0;
    for (uint32_t i = 0; i < n; ++i)
      if (i == 0 || tmp[i] != tmp[i - 1]) tmp[L++] = tmp[i];
    g->L = L;
    g->W = (L + 31) / 32;
    g->label_values = tmp;
    g->label = (uint32_t*)malloc((size_t)n * 4);
    for (uint32_t v = 0; v < n; ++v) {
      uint32_t lo = 0, hi = L;
      while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (tmp[mid] < labels[v]) lo = mid + 1;
        else hi = mid;
      }
      g->label[v] = lo;
    }
  }
  uint64_t* off[2];
  uint32_t* adj[2];
  int rc = normalise_dir(n, out_off, out_edges, g2l, max_vid, &off[0], &adj[0]);
  const int same_arrays = in_off == out_off && in_edges == out_edges;
  if (rc == ORC_OK && !same_arrays)
    rc = normalise_dir(n, in_off, in_edges, g2l, max_vid, &off[1], &adj[1]);
  if (rc) {
    *err = rc;
    goto fail;
  }
  if (same_arrays) {
    g->symmetric = 1;
    off[1] = NULL;
    adj[1] = NULL;
  } else {
    g->symmetric = off[0][n] == off[1][n] && memcmp(off[0], off[1], ((size_t)n + 1) * 8) == 0 &&
                   memcmp(adj[0], adj[1], off[0][n] * 4) == 0;
  }
  g->self = (uint8_t*)calloc(n, 1);
  for (int d = 0; d < 2; ++d) {
    if (d == 1 && g->symmetric) {
      free(off[1]);
      free(adj[1]);
      g->adj[1] = g->adj[0];
      g->loff[1] = g->loff[0];
      g->deg[1] = g->deg[0];
      g->nlb[1] = g->nlb[0];
      break;
    }
    uint32_t L = g->L, W = g->W;
    g->loff[d] = (uint32_t*)malloc(((size_t)n * L + 1) * 4);
    g->deg[d] = (uint32_t*)malloc((size_t)n * 4);
    g->nlb[d] = (uint32_t*)calloc((size_t)n * W, 4);
    g_sort_labels = g->label;
    slice_ctx sc = {g, d, off[d], adj[d]};
    par_for(n, slice_vertex, &sc);
    g->loff[d][(uint64_t)n * L] = (uint32_t)off[d][n];
    g->adj[d] = adj[d];
    free(off[d]);
  }
  g->bucket_off = (uint32_t*)calloc(g->L + 1, 4);
  g->bucket_vid = (uint32_t*)malloc((size_t)n * 4);
  for (uint32_t v = 0; v < n; ++v) g->bucket_off[g->label[v] + 1]++;
  for (uint32_t l = 0; l < g->L; ++l) g->bucket_off[l + 1] += g->bucket_off[l];
  {
    uint32_t* cur = (uint32_t*)malloc((size_t)(g->L + 1) * 4);
    memcpy(cur, g->bucket_off, (size_t)(g->L + 1) * 4);
    for (uint32_t v = 0; v < n; ++v) g->bucket_vid[cur[g->label[v]]++] = v;
    free(cur);
  }
  free(g2l);
  return g;
fail:
  free(g2l);
  orc_graph_free(g);
  return NULL;
}

void orc_graph_info(const orc_graph* g, uint32_t* n, uint32_t* L, int* symmetric,
                    uint64_t* m_out) {
  *n = g->n;
  *L = g->L;
  *symmetric = g->symmetric;
  *m_out = g->loff[0][(uint64_t)g->n * g->L];
}

/* ---- own reader of the CSR directory (immutable_csr.cu:168-247) -------- */
static int meta_value(const char* text, const char* section, const char* key, uint32_t* out) {
  const char* p = section ? strstr(text, section) : text;
  if (!p) return -1;
  size_t kl = strlen(key);
  for (const char* s = p; (s = strstr(s, key)) != NULL; s += kl) {
    const char* before = s == text ? s : s - 1;
    if (s != text && !(*before == ' ' || *before == '\n' || *before == '-' || *before == '{' ||
                       *before == ','))
      continue;
    const char* c = s + kl;
    while (*c == ' ') ++c;
    if (*c != ':') continue;
    ++c;
    unsigned long long v = strtoull(c, NULL, 10);
    if (v > 0xFFFFFFFFull) return -1;
    *out = (uint32_t)v;
    return 0;
  }
  return -1;
}

static uint32_t* read_words(FILE* f, uint64_t words) {
  uint32_t* p = (uint32_t*)malloc((words ? words : 1) * 4);
  if (p && words && fread(p, 4, words, f) != words) {
    free(p);
    return NULL;
  }
  return p;
}

orc_graph* orc_read_dir(const char* dir, int* err) {
  char path[4096];
  snprintf(path, sizeof(path), "%smeta.yaml", dir);
  FILE* f = fopen(path, "rb");
  if (!f) {
    *err = ORC_E_IO;
    return NULL;
  }
  char text[8192];
  size_t len = fread(text, 1, sizeof(text) - 1, f);
  text[len] = 0;
  fclose(f);
  uint32_t n, m_in, m_out, max_vid;
  if (meta_value(text, "subgraphs", "num_vertices", &n) ||
      meta_value(text, "subgraphs", "num_incoming_edges", &m_in) ||
      meta_value(text, "subgraphs", "num_outgoing_edges", &m_out) ||
      meta_value(text, "subgraphs", "max_vid", &max_vid)) {
    *err = ORC_E_FORMAT;
    return NULL;
  }
  snprintf(path, sizeof(path), "%sgraphs/0.bin", dir);
  f = fopen(path, "rb");
  if (!f) {
    *err = ORC_E_IO;
    return NULL;
  }
  uint32_t* gid = read_words(f, n);
  uint32_t* ind = read_words(f, n);
  uint32_t* outd = read_words(f, n);
  uint32_t* in_off = read_words(f, (uint64_t)n + 1);
  uint32_t* out_off = read_words(f, (uint64_t)n + 1);
  uint32_t* in_e = read_words(f, m_in);
  uint32_t* out_e = read_words(f, m_out);
  fclose(f);
  snprintf(path, sizeof(path), "%slabel/0.bin", dir);
  f = fopen(path, "rb");
  uint32_t* lab = f ? read_words(f, n) : NULL;
  if (f) fclose(f);
  orc_graph* g = NULL;
  if (!gid || !ind || !outd || !in_off || !out_off || !in_e || !out_e || !lab) {
    *err = ORC_E_IO;
  } else {
    g = orc_graph_from_arrays(n, max_vid, gid, out_off, out_e, in_off, in_e, lab, err);
  }
  free(gid);
  free(ind);
  free(outd);
  free(in_off);
  free(out_off);
  free(in_e);
  free(out_e);
  free(lab);
  return g;
}

/* ---------------------------------------------------------------- query -- */
int orc_query_from_arrays(uint32_t k, const uint32_t* globalid, const uint32_t* out_off,
                          const uint32_t* out_edges, const uint32_t* labels, orc_query* q) {
  if (k == 0 || k > ORC_MAXK) return ORC_E_ARG;
  memset(q, 0, sizeof(*q));
  q->k = k;
  for (uint32_t u = 0; u < k; ++u) q->label_raw[u] = labels[u];
  for (uint32_t u = 0; u < k; ++u)
    for (uint32_t e = out_off[u]; e < out_off[u + 1]; ++e) {
      uint32_t w = UINT32_MAX;
      for (uint32_t x = 0; x < k; ++x)
        if (globalid[x] == out_edges[e]) w = x;
      if (w == UINT32_MAX) return ORC_E_FORMAT;
      if (!(q->out_mask[u] >> w & 1u)) {
        q->esrc[q->n_edges] = u;
        q->edst[q->n_edges] = w;
        q->n_edges++;
      }
      q->out_mask[u] |= 1u << w;
    }
  return ORC_OK;
}

void orc_order_reference(const orc_query* q, uint32_t* order) {
  uint32_t placed = 0, n = 0;
#define PLACE(v)                    \
  do {                              \
    if (!(placed >> (v) & 1u)) {    \
      placed |= 1u << (v);          \
      order[n++] = (v);             \
    }                               \
  } while (0)
  if (q->n_edges) {
    PLACE(q->esrc[0]);
    PLACE(q->edst[0]);
  }
  while (n < q->k) {
    int changed = 1;
    while (changed) {
      changed = 0;
      for (uint32_t e = 0; e < q->n_edges; ++e) {
        int a = placed >> q->esrc[e] & 1u, b = placed >> q->edst[e] & 1u;
        if (a && !b) {
          PLACE(q->edst[e]);
          changed = 1;
        } else if (b && !a) {
          PLACE(q->esrc[e]);
          changed = 1;
        }
      }
    }
    for (uint32_t v = 0; v < q->k && n < q->k; ++v)
      if (!(placed >> v & 1u)) {
        PLACE(v);
        break;
      }
  }
#undef PLACE
}

/* --------------------------------------------------------------- search -- */
typedef struct plan {
  uint32_t k, zero, last_o1;
  uint32_t label[ORC_MAXK];
  uint32_t nc[ORC_MAXK];
  uint32_t cpos[ORC_MAXK][2 * ORC_MAXK], cdir[ORC_MAXK][2 * ORC_MAXK];
  uint32_t self[ORC_MAXK];
  uint32_t req[2][ORC_MAXK];
  uint32_t nlbq[2][ORC_MAXK][8];
  uint32_t perm[ORC_MAXK];
} plan;

static int make_plan(const orc_graph* g, const orc_query* q, const uint32_t* order, plan* P) {
  memset(P, 0, sizeof(*P));
  uint32_t k = q->k;
  P->k = k;
  int clab[ORC_MAXK];
  uint32_t in_mask[ORC_MAXK] = {0};
  for (uint32_t u = 0; u < k; ++u)
    for (uint32_t w = 0; w < k; ++w)
      if (q->out_mask[u] >> w & 1u) in_mask[w] |= 1u << u;
  for (uint32_t u = 0; u < k; ++u) {
    int c = -1;
    for (uint32_t l = 0; l < g->L; ++l)
      if (g->label_values[l] == q->label_raw[u]) c = (int)l;
    clab[u] = c;
    if (c < 0) P->zero = 1;
  }
  uint32_t seen = 0;
  for (uint32_t i = 0; i < k; ++i) {
    if (order[i] >= k || (seen >> order[i] & 1u)) return ORC_E_ARG;
    seen |= 1u << order[i];
  }
  for (uint32_t i = 0; i < k; ++i) {
    uint32_t u = order[i];
    P->perm[i] = u;
    P->label[i] = clab[u] < 0 ? 0 : (uint32_t)clab[u];
    for (uint32_t j = 0; j < i; ++j) {
      uint32_t w = order[j];
      int w_to_u = q->out_mask[w] >> u & 1u, u_to_w = q->out_mask[u] >> w & 1u;
      if (g->symmetric) {
        if (w_to_u || u_to_w) {
          P->cpos[i][P->nc[i]] = j;
          P->cdir[i][P->nc[i]++] = 0;
        }
      } else {
        if (w_to_u) {
          P->cpos[i][P->nc[i]] = j;
          P->cdir[i][P->nc[i]++] = 0;
        }
        if (u_to_w) {
          P->cpos[i][P->nc[i]] = j;
          P->cdir[i][P->nc[i]++] = 1;
        }
      }
    }
    P->self[i] = q->out_mask[u] >> u & 1u;
    uint32_t nb0 = g->symmetric ? (q->out_mask[u] | in_mask[u]) : q->out_mask[u];
    uint32_t nb1 = in_mask[u];
    P->req[0][i] = (uint32_t)__builtin_popcount(nb0);
    P->req[1][i] = g->symmetric ? 0 : (uint32_t)__builtin_popcount(nb1);
    for (uint32_t w = 0; w < k; ++w) {
      if (clab[w] < 0) continue;
      if (nb0 >> w & 1u) P->nlbq[0][i][clab[w] / 32] |= 1u << (clab[w] % 32);
      if (!g->symmetric && (nb1 >> w & 1u)) P->nlbq[1][i][clab[w] / 32] |= 1u << (clab[w] % 32);
    }
  }
  P->last_o1 = k >= 2 && P->nc[k - 1] == 1 && !P->self[k - 1];
  return ORC_OK;
}

typedef struct shared_ctx {
  const orc_graph* g;
  const plan* P;
  uint32_t filters;
  uint32_t* emit_rows;
  uint64_t emit_cap;
  uint64_t emit_n;
  atomic_ullong next_root; /* index j of the next root position begin + j*step */
  uint64_t root_begin, root_end, root_step;
} shared_ctx;

typedef struct thread_ctx {
  shared_ctx* S;
  uint64_t count, balg, balgc;
  uint64_t rows[ORC_MAXK + 1];
  uint32_t m[ORC_MAXK];
} thread_ctx;

static int contains(const uint32_t* a, uint64_t s, uint64_t e, uint32_t x) {
  uint64_t lo = s, hi = e;
  while (lo < hi) {
    uint64_t mid = (lo + hi) / 2;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo < e && a[lo] == x;
}

static int passes(const thread_ctx* T, uint32_t i, uint32_t x) {
  const orc_graph* g = T->S->g;
  const plan* P = T->S->P;
  for (uint32_t j = 0; j < i; ++j)
    if (T->m[j] == x) return 0;
  for (uint32_t c = 0; c < P->nc[i]; ++c) {
    uint32_t y = T->m[P->cpos[i][c]], d = P->cdir[i][c];
    const uint32_t* lo = g->loff[d] + (uint64_t)y * g->L + P->label[i];
    if (!contains(g->adj[d], lo[0], lo[1], x)) return 0;
  }
  if (P->self[i] && !g->self[x]) return 0;
  /* Filters prune positions that are extended further, except the position
   * before a last position with a single backward neighbour (its candidates
   * are closed in O(1) by the slice length). */
  if (i + 1 < P->k && !(i + 2 == P->k && P->last_o1)) {
    uint32_t f = T->S->filters;
    if (f & 1u) {
      if (g->deg[0][x] < P->req[0][i]) return 0;
      if (!g->symmetric && g->deg[1][x] < P->req[1][i]) return 0;
    }
    if (f & 2u) {
      for (uint32_t w = 0; w < g->W; ++w) {
        if (P->nlbq[0][i][w] & ~g->nlb[0][(uint64_t)x * g->W + w]) return 0;
        if (!g->symmetric && (P->nlbq[1][i][w] & ~g->nlb[1][(uint64_t)x * g->W + w])) return 0;
      }
    }
  }
  return 1;
}

static pthread_mutex_t emit_mu = PTHREAD_MUTEX_INITIALIZER;

static void record(thread_ctx* T) {
  shared_ctx* S = T->S;
  T->count++;
  if (!S->emit_rows) return;
  pthread_mutex_lock(&emit_mu);
  if (S->emit_n < S->emit_cap) {
    uint32_t* row = S->emit_rows + S->emit_n * S->P->k;
    for (uint32_t i = 0; i < S->P->k; ++i) row[S->P->perm[i]] = S->g->globalid[T->m[i]];
  }
  S->emit_n++;
  pthread_mutex_unlock(&emit_mu);
}

/* Extends the prefix m[0..i-1] at position i. */
static void extend(thread_ctx* T, uint32_t i) {
  const orc_graph* g = T->S->g;
  const plan* P = T->S->P;
  const uint32_t lab = P->label[i];
  const uint32_t* list;
  uint64_t s, e;
  uint64_t charge = 0;
  if (P->nc[i] == 0) {
    list = g->bucket_vid;
    s = g->bucket_off[lab];
    e = g->bucket_off[lab + 1];
    charge = (e - s) * (12ull + 4ull * g->W);
    T->balg += charge;
    T->balgc += charge;
  } else {
    uint64_t best = UINT64_MAX;
    list = NULL;
    s = e = 0;
    for (uint32_t c = 0; c < P->nc[i]; ++c) {
      uint32_t y = T->m[P->cpos[i][c]], d = P->cdir[i][c];
      const uint32_t* lo = g->loff[d] + (uint64_t)y * g->L + lab;
      uint64_t len = lo[1] - lo[0];
      charge += 8 + 4 * len;
      if (len < best) {
        best = len;
        list = g->adj[d];
        s = lo[0];
        e = lo[1];
      }
    }
    T->balg += charge;
    T->balgc += (i + 1 == P->k && P->last_o1) ? 8 : charge;
  }
  for (uint64_t p = s; p < e; ++p) {
    uint32_t x = list[p];
    if (!passes(T, i, x)) continue;
    T->rows[i + 1]++;
    T->m[i] = x;
    if (i + 1 == P->k) record(T);
    else extend(T, i + 1);
  }
}

static void* worker(void* arg) {
  thread_ctx* T = (thread_ctx*)arg;
  shared_ctx* S = T->S;
  const orc_graph* g = S->g;
  const plan* P = S->P;
  const uint32_t lab = P->label[0];
  const uint32_t b0 = g->bucket_off[lab];
  for (;;) {
    const uint64_t j = atomic_fetch_add(&S->next_root, 1);
    if (j >= (S->root_end - S->root_begin + S->root_step - 1) / S->root_step) break;
    const uint64_t r = S->root_begin + j * S->root_step;
    uint32_t x = g->bucket_vid[b0 + r];
    if (!passes(T, 0, x)) continue;
    T->rows[1]++;
    T->m[0] = x;
    if (P->k == 1) record(T);
    else extend(T, 1);
  }
  return NULL;
}

static int run(const orc_graph* g, const orc_query* q, const uint32_t* order, uint32_t filters,
               int threads, uint64_t root_begin, uint64_t root_end, uint64_t root_step,
               uint32_t* emit_rows, uint64_t emit_cap, orc_result* res, uint64_t* emitted) {
  plan P;
  int rc = make_plan(g, q, order, &P);
  if (rc) return rc;
  memset(res, 0, sizeof(*res));
  if (P.zero) return ORC_OK;
  const uint32_t lab = P.label[0];
  const uint64_t nb = g->bucket_off[lab + 1] - g->bucket_off[lab];
  if (root_end > nb) root_end = nb;
  if (root_begin > root_end) root_begin = root_end;
  shared_ctx S;
  memset(&S, 0, sizeof(S));
  S.g = g;
  S.P = &P;
  S.filters = filters;
  S.emit_rows = emit_rows;
  S.emit_cap = emit_cap;
  S.root_begin = root_begin;
  S.root_end = root_end;
  S.root_step = root_step < 1 ? 1 : root_step;
  atomic_init(&S.next_root, 0);
  if (threads < 1) threads = 1;
  if (emit_rows) threads = 1;
  thread_ctx* T = (thread_ctx*)calloc((size_t)threads, sizeof(thread_ctx));
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  for (int t = 0; t < threads; ++t) {
    T[t].S = &S;
    if (threads > 1) pthread_create(&th[t], NULL, worker, &T[t]);
  }
  if (threads == 1) worker(&T[0]);
  else
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  /* level-0 charge: one candidate test per root position taken */
  res->balg = res->balg_count =
      ((root_end - root_begin + S.root_step - 1) / S.root_step) * (12ull + 4ull * g->W);
  for (int t = 0; t < threads; ++t) {
    res->count += T[t].count;
    res->balg += T[t].balg;
    res->balg_count += T[t].balgc;
    for (uint32_t i = 0; i <= P.k; ++i) res->level_rows[i] += T[t].rows[i];
  }
  if (emitted) *emitted = S.emit_n;
  free(T);
  free(th);
  return ORC_OK;
}

/* Count over the level-0 candidates at bucket positions root_begin,
 * root_begin + root_step, ... below root_end (root_step 0 or 1: all). */
int orc_count(const orc_graph* g, const orc_query* q, const uint32_t* order, uint32_t filters,
              int threads, uint64_t root_begin, uint64_t root_end, uint64_t root_step,
              orc_result* res) {
  return run(g, q, order, filters, threads, root_begin, root_end, root_step, NULL, 0, res, NULL);
}

static uint32_t g_row_k;
static int cmp_rows(const void* a, const void* b) {
  const uint32_t* x = (const uint32_t*)a;
  const uint32_t* y = (const uint32_t*)b;
  for (uint32_t i = 0; i < g_row_k; ++i)
    if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
  return 0;
}

/* All matches as rows in query-vertex order, lexicographically sorted, over
 * the level-0 candidates at bucket positions root_begin, root_begin +
 * root_step, ... below root_end. */
int orc_emit(const orc_graph* g, const orc_query* q, const uint32_t* order, uint32_t filters,
             uint64_t root_begin, uint64_t root_end, uint64_t root_step, uint32_t* rows,
             uint64_t cap, uint64_t* n_rows) {
  orc_result res;
  int rc = run(g, q, order, filters, 1, root_begin, root_end, root_step, rows, cap, &res, n_rows);
  if (rc) return rc;
  g_row_k = q->k;
  qsort(rows, *n_rows < cap ? *n_rows : cap, (size_t)q->k * 4, cmp_rows);
  return ORC_OK;
}

uint32_t orc_bucket_size(const orc_graph* g, const orc_query* q, const uint32_t* order) {
  for (uint32_t l = 0; l < g->L; ++l)
    if (g->label_values[l] == q->label_raw[order[0]]) return g->bucket_off[l + 1] - g->bucket_off[l];
  return 0;
}
