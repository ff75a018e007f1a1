/*
 * gen.c — seeded synthetic inputs for the checker side: R-MAT data graphs,
 * uniform / Zipf vertex labels and random-walk query labels.
 *
 * TEST INFRASTRUCTURE ONLY.  Used by tests/ (to pin the product generators
 * bit for bit) and by bench.py's reference arm, which must build its
 * workload without loading the product library.  Nothing in the product
 * links or calls it.
 *
 * Every draw is a pure function of (seed, index) through Philox4x32-10
 * (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2,
 * 3", SC'11): ten rounds of two 32x32->64-bit multiplies with the round
 * keys bumped by the Weyl constants.  The stream assignment (which counter
 * and stream word feed which draw) is the workload specification of this
 * project:
 *   R-MAT edge e, levels 4j..4j+3:  philox(seed, e, 0x524D00 + j), word l&3;
 *                                   quadrant by integer thresholds floor(p*2^32)
 *   label of vertex v:              philox(seed, v, 0x4C4200); uniform: w0*L>>32;
 *                                   Zipf: u53(w0, w1) against the normalised CDF
 *   walk of a query (seed):         sequential words of stream 0x57414C4B,
 *                                   below(n) = w*n >> 32
 *   random query (seed):            sequential words of stream 0x51525900
 *   Chung-Lu pair (i, j):           philox(seed, i*n + j, 0x434C00), u53(w0, w1)
 * The data graph is symmetrised with self-loops and repeated pairs removed and
 * sorted adjacency, as the reference's converter writes lists
 * (core/util/format_converter.cuh:236-249).
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint32_t v[4];
} ph4;

static ph4 philox(uint64_t key, uint64_t ctr_lo, uint64_t ctr_hi) {
  uint32_t x0 = (uint32_t)ctr_lo, x1 = (uint32_t)(ctr_lo >> 32);
  uint32_t x2 = (uint32_t)ctr_hi, x3 = (uint32_t)(ctr_hi >> 32);
  uint32_t ka = (uint32_t)key, kb = (uint32_t)(key >> 32);
  for (int round = 0; round < 10; ++round) {
    const uint64_t pa = (uint64_t)0xD2511F53u * x0;
    const uint64_t pb = (uint64_t)0xCD9E8D57u * x2;
    const uint32_t y0 = (uint32_t)(pb >> 32) ^ x1 ^ ka;
    const uint32_t y1 = (uint32_t)pb;
    const uint32_t y2 = (uint32_t)(pa >> 32) ^ x3 ^ kb;
    const uint32_t y3 = (uint32_t)pa;
    x0 = y0;
    x1 = y1;
    x2 = y2;
    x3 = y3;
    ka += 0x9E3779B9u;
    kb += 0xBB67AE85u;
  }
  ph4 r = {{x0, x1, x2, x3}};
  return r;
}

/* 53-bit uniform double in [0, 1) from two words. */
static double u53(uint32_t a, uint32_t b) {
  uint64_t x = ((uint64_t)a << 21) ^ ((uint64_t)b >> 11);
  x &= ((uint64_t)1 << 53) - 1;
  return (double)x * (1.0 / 9007199254740992.0);
}

typedef struct {
  uint64_t seed, stream, ctr;
  ph4 buf;
  int used;
} wstream;

static void ws_init(wstream* w, uint64_t seed, uint64_t stream) {
  w->seed = seed;
  w->stream = stream;
  w->ctr = 0;
  w->used = 4;
}

static uint32_t ws_next(wstream* w) {
  if (w->used == 4) {
    w->buf = philox(w->seed, w->ctr++, w->stream);
    w->used = 0;
  }
  return w->buf.v[w->used++];
}

static uint32_t ws_below(wstream* w, uint32_t n) {
  return (uint32_t)(((uint64_t)ws_next(w) * n) >> 32);
}

static double ws_uniform(wstream* w) {
  uint32_t a = ws_next(w);
  uint32_t b = ws_next(w);
  return u53(a, b);
}

/* ------------------------------------------------------------ R-MAT ------- */
typedef struct {
  int t, nt;
  uint32_t scale;
  uint64_t m, ta, tab, tabc, seed;
  uint32_t *src, *dst;
} rmat_job;

static void* rmat_edges(void* arg) {
  rmat_job* J = (rmat_job*)arg;
  const uint64_t chunk = (J->m + (uint64_t)J->nt - 1) / (uint64_t)J->nt;
  const uint64_t lo = (uint64_t)J->t * chunk;
  const uint64_t hi = lo + chunk < J->m ? lo + chunk : J->m;
  for (uint64_t e = lo; e < hi; ++e) {
    uint32_t s = 0, d = 0;
    ph4 r = {{0, 0, 0, 0}};
    for (uint32_t l = 0; l < J->scale; ++l) {
      if ((l & 3u) == 0) r = philox(J->seed, e, 0x524D00ull + (l >> 2));
      const uint64_t u = r.v[l & 3u];
      const uint32_t bit = 1u << (J->scale - 1 - l);
      if (u >= J->tabc) {
        s |= bit;
        d |= bit;
      } else if (u >= J->tab) {
        s |= bit;
      } else if (u >= J->ta) {
        d |= bit;
      }
    }
    J->src[e] = s;
    J->dst[e] = d;
  }
  return NULL;
}

/* Symmetrised CSR from directed pairs: self-loops dropped, lists sorted and
 * deduplicated.  Threads split the pairs for counting and placement and the
 * vertices for sorting. */
typedef struct {
  int t, nt, phase;
  uint32_t n;
  uint64_t m;
  const uint32_t *src, *dst;
  _Atomic uint32_t* cnt;
  uint64_t* off;
  uint32_t* adj;
  uint32_t* uniq;
} csr_job;

static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : x > y;
}

static void* csr_work(void* arg) {
  csr_job* J = (csr_job*)arg;
  if (J->phase < 2) {
    const uint64_t chunk = (J->m + (uint64_t)J->nt - 1) / (uint64_t)J->nt;
    const uint64_t lo = (uint64_t)J->t * chunk;
    const uint64_t hi = lo + chunk < J->m ? lo + chunk : J->m;
    for (uint64_t e = lo; e < hi; ++e) {
      const uint32_t s = J->src[e], d = J->dst[e];
      if (s == d) continue;
      if (J->phase == 0) {
        atomic_fetch_add_explicit(&J->cnt[s], 1u, memory_order_relaxed);
        atomic_fetch_add_explicit(&J->cnt[d], 1u, memory_order_relaxed);
      } else {
        uint32_t ps = atomic_fetch_add_explicit(&J->cnt[s], 1u, memory_order_relaxed);
        uint32_t pd = atomic_fetch_add_explicit(&J->cnt[d], 1u, memory_order_relaxed);
        J->adj[J->off[s] + ps] = d;
        J->adj[J->off[d] + pd] = s;
      }
    }
  } else {
    for (uint64_t v = (uint64_t)J->t; v < J->n; v += (uint64_t)J->nt) {
      uint32_t* a = J->adj + J->off[v];
      const uint64_t len = J->off[v + 1] - J->off[v];
      qsort(a, len, 4, cmp_u32);
      uint32_t u = 0;
      for (uint64_t i = 0; i < len; ++i)
        if (i == 0 || a[i] != a[i - 1]) a[u++] = a[i];
      J->uniq[v] = u;
    }
  }
  return NULL;
}

static int run_threads(int nt, void* jobs, size_t job_size, void* (*fn)(void*)) {
  pthread_t* th = (pthread_t*)calloc((size_t)nt, sizeof(pthread_t));
  if (!th) return -3;
  for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, fn, (char*)jobs + job_size * (size_t)t);
  for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
  free(th);
  return 0;
}

/* Builds the symmetrised CSR of n vertices from m directed pairs.  *off
 * (n+1 entries) and *adj are malloc'ed; the caller frees them. */
int orc_csr_symmetric(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m,
                      int threads, uint32_t** off_out, uint32_t** adj_out, uint64_t* m_out) {
  int nt = threads < 1 ? 1 : threads;
  _Atomic uint32_t* cnt = (_Atomic uint32_t*)calloc((size_t)n + 1, sizeof(_Atomic uint32_t));
  uint64_t* off = (uint64_t*)malloc(((size_t)n + 1) * 8);
  uint32_t* uniq = (uint32_t*)malloc(((size_t)n + 1) * 4);
  csr_job* jobs = (csr_job*)calloc((size_t)nt, sizeof(csr_job));
  if (!cnt || !off || !uniq || !jobs) return -3;
  for (int t = 0; t < nt; ++t) {
    jobs[t].t = t;
    jobs[t].nt = nt;
    jobs[t].n = n;
    jobs[t].m = m;
    jobs[t].src = src;
    jobs[t].dst = dst;
    jobs[t].cnt = cnt;
    jobs[t].off = off;
    jobs[t].uniq = uniq;
  }
  run_threads(nt, jobs, sizeof(csr_job), csr_work);
  off[0] = 0;
  for (uint32_t v = 0; v < n; ++v) {
    off[v + 1] = off[v] + atomic_load(&cnt[v]);
    atomic_store(&cnt[v], 0u);
  }
  uint32_t* adj = (uint32_t*)malloc((off[n] ? off[n] : 1) * 4);
  if (!adj) return -3;
  for (int t = 0; t < nt; ++t) {
    jobs[t].phase = 1;
    jobs[t].adj = adj;
  }
  run_threads(nt, jobs, sizeof(csr_job), csr_work);
  for (int t = 0; t < nt; ++t) jobs[t].phase = 2;
  run_threads(nt, jobs, sizeof(csr_job), csr_work);
  /* compact the deduplicated lists */
  uint32_t* o32 = (uint32_t*)malloc(((size_t)n + 1) * 4);
  if (!o32) return -3;
  uint64_t w = 0;
  for (uint32_t v = 0; v < n; ++v) {
    o32[v] = (uint32_t)w;
    if (w != off[v]) memmove(adj + w, adj + off[v], (size_t)uniq[v] * 4);
    w += uniq[v];
  }
  o32[n] = (uint32_t)w;
  *off_out = o32;
  *adj_out = adj;
  *m_out = w;
  free(cnt);
  free(off);
  free(uniq);
  free(jobs);
  return 0;
}

/* R-MAT data graph, symmetrised CSR (ids not permuted). */
int orc_gen_rmat_csr(uint32_t scale, uint32_t ef, double a, double b, double c, uint64_t seed,
                     int threads, uint32_t** off, uint32_t** adj, uint64_t* m_out) {
  if (scale == 0 || scale > 31 || ef == 0) return -7;
  const uint64_t m = (uint64_t)ef << scale;
  const double two32 = 4294967296.0;
  uint32_t* src = (uint32_t*)malloc(m * 4);
  uint32_t* dst = (uint32_t*)malloc(m * 4);
  int nt = threads < 1 ? 1 : threads;
  rmat_job* jobs = (rmat_job*)calloc((size_t)nt, sizeof(rmat_job));
  if (!src || !dst || !jobs) return -3;
  for (int t = 0; t < nt; ++t) {
    jobs[t].t = t;
    jobs[t].nt = nt;
    jobs[t].scale = scale;
    jobs[t].m = m;
    jobs[t].ta = (uint64_t)floor(a * two32);
    jobs[t].tab = (uint64_t)floor((a + b) * two32);
    jobs[t].tabc = (uint64_t)floor((a + b + c) * two32);
    jobs[t].seed = seed;
    jobs[t].src = src;
    jobs[t].dst = dst;
  }
  run_threads(nt, jobs, sizeof(rmat_job), rmat_edges);
  free(jobs);
  int rc = orc_csr_symmetric(1u << scale, src, dst, m, threads, off, adj, m_out);
  free(src);
  free(dst);
  return rc;
}

/* ----------------------------------------------------------- labels ------- */
int orc_gen_labels(uint32_t n, uint32_t kind, uint32_t L, double s, uint64_t seed,
                   uint32_t* labels) {
  if (L == 0) return -7;
  double* cdf = NULL;
  if (kind == 1) {
    cdf = (double*)malloc((size_t)L * sizeof(double));
    if (!cdf) return -3;
    double acc = 0;
    for (uint32_t k = 0; k < L; ++k) {
      acc += pow((double)(k + 1), -s);
      cdf[k] = acc;
    }
    for (uint32_t k = 0; k < L; ++k) cdf[k] /= acc;
    cdf[L - 1] = 1.0;
  }
  for (uint64_t v = 0; v < n; ++v) {
    const ph4 r = philox(seed, v, 0x4C4200ull);
    if (kind == 0) {
      labels[v] = (uint32_t)(((uint64_t)r.v[0] * L) >> 32);
    } else {
      const double u = u53(r.v[0], r.v[1]);
      uint32_t lo = 0, hi = L; /* first k with cdf[k] > u */
      while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
      }
      labels[v] = lo < L ? lo : L - 1;
    }
  }
  free(cdf);
  return 0;
}

/* ------------------------------------------------------ query labels ------ */
/* Labels of a k-vertex query (adjacency bit masks adjm[k]) copied from a
 * random walk on the data graph (identity ids, sorted CSR off/adj) along the
 * query's BFS spanning tree from vertex 0: the image of a child is a uniform
 * neighbour of its parent's image (the parent's own image on a dead end). */
int orc_walk_labels(uint32_t n, const uint32_t* off, const uint32_t* adj, const uint32_t* labels,
                    uint32_t k, const uint32_t* adjm, uint64_t seed, uint64_t stream,
                    uint32_t* qlab) {
  if (n == 0 || k == 0 || k > 16) return -7;
  wstream w;
  ws_init(&w, seed, stream);
  uint32_t start = 0;
  int found = 0;
  for (int tries = 0; tries < (1 << 20); ++tries) {
    uint32_t v = ws_below(&w, n);
    if (off[v + 1] > off[v]) {
      start = v;
      found = 1;
      break;
    }
  }
  if (!found) return -7;
  uint32_t img[16], queue[16], qn = 0;
  for (uint32_t u = 0; u < k; ++u) img[u] = UINT32_MAX;
  img[0] = start;
  queue[qn++] = 0;
  for (uint32_t h = 0; h < qn; ++h) {
    const uint32_t p = queue[h];
    for (uint32_t c = 0; c < k; ++c) {
      if (!(adjm[p] >> c & 1u) || img[c] != UINT32_MAX) continue;
      const uint32_t x = img[p];
      const uint32_t deg = off[x + 1] - off[x];
      img[c] = deg == 0 ? x : adj[off[x] + ws_below(&w, deg)];
      queue[qn++] = c;
    }
  }
  for (uint32_t u = 0; u < k; ++u) qlab[u] = labels[img[u] == UINT32_MAX ? start : img[u]];
  return 0;
}

/* Random connected query of k vertices: vertex j joins a uniform earlier
 * vertex, then every other pair is added with probability p_extra.  Writes
 * the adjacency masks; the walk labels use seed ^ 0x9E3779B97F4A7C15. */
int orc_random_query_shape(uint32_t k, double p_extra, uint64_t seed, uint32_t* adjm) {
  if (k == 0 || k > 16) return -7;
  wstream w;
  ws_init(&w, seed, 0x51525900ull);
  for (uint32_t u = 0; u < k; ++u) adjm[u] = 0;
  for (uint32_t j = 1; j < k; ++j) {
    const uint32_t p = ws_below(&w, j);
    adjm[p] |= 1u << j;
    adjm[j] |= 1u << p;
  }
  for (uint32_t i = 0; i < k; ++i)
    for (uint32_t j = i + 1; j < k; ++j) {
      if (adjm[i] >> j & 1u) continue;
      if (ws_uniform(&w) < p_extra) {
        adjm[i] |= 1u << j;
        adjm[j] |= 1u << i;
      }
    }
  return 0;
}
