/*
 * mg_subiso.h — C-ABI of the B200 subgraph-isomorphism engine (libmg_subiso.so).
 *
 * Plain C: host pointers, sizes and integer status codes only; no CUDA or
 * torch types cross this boundary.  Every entry point returns MG_OK (0) or a
 * negative MG_E_* code and never calls exit()/abort(); the message of the
 * last failure on the calling thread is returned by mg_last_error().
 *
 * Each entry point names the reference interface it replaces
 * (hsiaoko/MatrixGraph, paths relative to the project root).
 *
 * Semantics of a "match" (all entry points): an injective map f from query
 * vertices to data vertices with label(f(u)) == label(u) for every query
 * vertex u and (f(u), f(w)) an edge of the data graph for every directed
 * query edge (u, w).  Non-induced; automorphic images are counted
 * separately.  Edge multiplicity is ignored (set semantics).  This is the
 * matching rule of the reference's only exact GPU matcher,
 * core/task/gpu_task/kernel/kernel_gar_match.cu:305-363.
 */
#ifndef MG_SUBISO_H_
#define MG_SUBISO_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MG_OK          0
#define MG_E_IO       -1   /* file missing / unreadable / unwritable          */
#define MG_E_FORMAT   -2   /* malformed meta.yaml or inconsistent CSR arrays  */
#define MG_E_OOM      -3   /* device or host allocation failed / over budget  */
#define MG_E_CAPACITY -4   /* emit output truncated at cap_rows               */
#define MG_E_TIMEOUT  -5   /* a bounded device wait expired                   */
#define MG_E_CUDA     -6   /* CUDA runtime error                              */
#define MG_E_ARG      -7   /* invalid argument                                */
#define MG_E_LIMIT    -8   /* input beyond a documented engine limit          */

#define MG_MAX_QUERY_VERTICES 16   /* k <= 16                                */
#define MG_MAX_LABELS        256   /* distinct vertex labels in a data graph  */

/* ---- CSR view: the reference's binary CSR directory, in memory ---------- *
 * Layout of graphs/0.bin (uint32 arrays, in this order) — replaces the
 * buffers parsed by ImmutableCSR::Read / ParseBasePtr
 * (core/data_structures/immutable_csr.cu:79-101, :168-247):
 *   globalid[n] indeg[n] outdeg[n] in_off[n+1] out_off[n+1]
 *   in_edges[m_in] out_edges[m_out]
 *   edges_globalid_by_localid[max_vid+1] localid_by_globalid[max_vid+1]
 * label/0.bin holds labels[n].  Adjacency entries are GLOBAL vertex ids
 * (core/util/format_converter.cuh:166-184).  All pointers are host memory
 * owned by the caller (or by the owner handle of mg_csr_dir_open).
 * edges_globalid_by_localid / localid_by_globalid may be NULL.          */
typedef struct mg_csr_view {
  uint32_t n;          /* num_vertices                                      */
  uint32_t max_vid;
  uint32_t min_vid;
  uint32_t m_in;       /* num_incoming_edges                                */
  uint32_t m_out;      /* num_outgoing_edges                                */
  uint32_t _pad;
  const uint32_t* globalid;
  const uint32_t* indeg;
  const uint32_t* outdeg;
  const uint32_t* in_off;
  const uint32_t* out_off;
  const uint32_t* in_edges;
  const uint32_t* out_edges;
  const uint32_t* edges_globalid_by_localid;
  const uint32_t* localid_by_globalid;
  const uint32_t* labels;
} mg_csr_view;

/* Matching order selection. */
#define MG_ORDER_REFERENCE 0  /* vertex-introduction order of the reference WOJ
                                 edge chain (core/data_structures/
                                 woj_exec_plan.cuh:36-45), rescanning skipped
                                 edges so every vertex is placed            */
#define MG_ORDER_STRONG    1  /* fewest candidates first, then most backward
                                 neighbours                                  */
#define MG_ORDER_LEARNED   2  /* order chosen by a loaded order model        */
#define MG_ORDER_GIVEN     3  /* opts->given_order[k] (query local ids)      */

/* Candidate-filter bits (all sound: they never remove a true match). */
#define MG_FILTER_DEGREE 1u   /* deg(v) >= deg_q(u): kernel_woj_subsio.cu:123-138 */
#define MG_FILTER_NLB    2u   /* neighbour-label bit subset: the sound form of
                                 NeighborLabelCounterFilter :385-446          */
#define MG_FILTER_ALL    3u

typedef struct mg_opts {
  int32_t  order;            /* MG_ORDER_*                                   */
  uint32_t filters;          /* MG_FILTER_* bits; default MG_FILTER_ALL      */
  const uint32_t* given_order; /* k query-local ids when order == GIVEN      */
  void*    model;            /* order model for MG_ORDER_LEARNED (may be NULL:
                                then the reference order is used)            */
  uint64_t chunk_rows;       /* partial-match rows per level chunk; 0 = auto */
  uint32_t grab;             /* expand tiles (256 candidates each) a block
                                takes from the device work queue at a time;
                                0 = auto                                     */
  uint32_t root_step;        /* level-0 candidates are the bucket positions
                                root_begin, root_begin + root_step, ... below
                                root_end (0 or 1: every position).  A stride
                                equal to the rank count with root_begin =
                                rank spreads the hub roots evenly over ranks */
  uint32_t probe_min;        /* a probe into the label slice of a hub uses the
                                hub's bitmap when the slice has at least this
                                many entries, binary search otherwise
                                (0 or 1: always the bitmap)                  */
  uint32_t kernel_events;    /* 1: time every expand-kernel launch with a CUDA
                                event pair (mg_stats.expand_ms); each launch
                                then waits for the previous one on the host,
                                so use it for measurement passes only        */
  uint64_t mem_budget_bytes; /* cap on enumeration scratch; 0 = auto        */
  uint64_t root_begin;       /* level-0 candidates [root_begin, root_end) of  */
  uint64_t root_end;         /* the first position's label bucket; 0,0 = all  */
  uint32_t no_tail;          /* closed-form count of a two-position ending
                                (count mode): a pendant path or two leaves of
                                one anchor; 0 or 2 = whenever the plan ends
                                in one, 1 = never                            */
  uint32_t lanes;            /* batch counts: queries run as fixed launch
                                sequences on this many concurrent streams,
                                every size read on the device, one host sync
                                per batch (0 = 8); MG_LANES_SHARED = one
                                level-synchronous run over shared tables     */
  uint64_t max_elements;     /* work budget in candidate elements (0 = none):
                                a single-query call above it returns
                                MG_E_LIMIT; in a batch it applies per query
                                and a query above it reports UINT64_MAX      */
  void*    matrix_filter;    /* lossy learned candidate filter
                                (mg_matrix_filter_load), single-query count
                                and emit only; NULL = off (exact)            */
} mg_opts;

#define MG_LANES_SHARED 0xFFFFFFFFu

/* Per-call statistics (optional out-parameter of the *_ex entry points). */
typedef struct mg_stats {
  uint32_t k;
  uint32_t order[MG_MAX_QUERY_VERTICES];        /* chosen order (query ids) */
  uint64_t level_rows[MG_MAX_QUERY_VERTICES + 1]; /* P_i: surviving prefixes of
                                                   length i (i = 1..k)       */
  uint64_t balg_bytes;       /* algorithmic bytes, full-slice definition     */
  uint64_t balg_count_bytes; /* algorithmic bytes, count-mode definition     */
  double   device_ms;        /* device time from first launch to result      */
  uint64_t launches;         /* kernels launched by this call                */
  uint64_t chunks;           /* level chunks processed                       */
  uint64_t elements;         /* candidate elements expanded                  */
  double   expand_ms;        /* summed durations of the expand-kernel launches
                                (opts->kernel_events = 1, else 0)            */
  uint64_t expand_launches;  /* expand-kernel launches                       */
} mg_stats;

typedef struct mg_graph_info {
  uint32_t n;
  uint32_t n_labels;         /* distinct labels after compaction             */
  uint64_t m_out;            /* distinct directed adjacency entries (out)    */
  uint64_t m_in;
  uint32_t symmetric;        /* 1 if in-CSR == out-CSR                       */
  uint32_t device;
  uint64_t device_bytes;     /* resident bytes of graph + derived indices    */
  uint32_t max_degree;
  uint32_t nlb_words;        /* W = ceil(n_labels / 32)                       */
  uint32_t hubs;             /* vertices with a dense neighbour bitmap        */
  uint32_t hub_min_degree;   /* smallest degree among them                    */
  uint64_t hub_bytes;        /* device bytes of the hub bitmaps               */
} mg_graph_info;

/* Options of mg_graph_upload_ex.  Hub bitmaps: the highest-degree vertices
 * get one bit per data vertex over their whole adjacency, so testing whether
 * a candidate lies in a hub's label slice is one load instead of a binary
 * search.  Vertices are taken in decreasing degree while the budget lasts
 * (ties at the cut are all taken or all left out).                        */
#define MG_HUB_AUTO (~(uint64_t)0)
typedef struct mg_upload_opts {
  uint64_t hub_bytes;        /* MG_HUB_AUTO: min(4 GiB, free device memory/8);
                                0: no hub bitmaps                            */
  uint32_t hub_min_degree;   /* smallest degree of a hub; 0 = 128             */
  uint32_t _reserved;        /* must be 0                                    */
} mg_upload_opts;

/* ---- library ------------------------------------------------------------ */
const char* mg_last_error(void);
const char* mg_version(void);
void mg_opts_default(mg_opts* o);

/* ---- reference CSR directory format ------------------------------------- */
/* Replaces ImmutableCSR::Read (core/data_structures/immutable_csr.cu:168-247)
 * and the meta.yaml decoder (core/common/yaml_config.h:85-110).  `dir` is a
 * directory prefix that ends in '/', exactly as the reference concatenates
 * it.  *owner receives the host memory holding the arrays.               */
int  mg_csr_dir_open(const char* dir, mg_csr_view* out, void** owner);
void mg_csr_dir_close(void* owner);
/* Replaces ImmutableCSR::Write (core/data_structures/immutable_csr.cu:103-166);
 * num_edges = m_in + m_out wraps modulo 2^32 as the reference's uint32 sum. */
int  mg_csr_dir_write(const char* dir, const mg_csr_view* g);

/* Build a reference-layout CSR from a directed edge list (host).  Replaces
 * Edgelist2ImmutableCSR (core/util/format_converter.cuh:91-284): vertex ids
 * 0..n-1, per-vertex sorted adjacency, labels given.  flags bit0: add the
 * reverse of every edge; bit1: drop self-loops; bit2: drop duplicates.     */
#define MG_BUILD_SYMMETRIZE 1u
#define MG_BUILD_NO_SELF    2u
#define MG_BUILD_DEDUP      4u
int  mg_csr_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst,
                       uint64_t m, const uint32_t* labels, uint32_t flags,
                       mg_csr_view* out, void** owner);
/* Edge list CSV ("src,dst" per line) -> CSR with first-appearance id
 * compaction and labels vid % label_range.  Replaces
 * ConvertEdgelistCSV2ImmutableCSR (tools/graph_converter/
 * to_immutable_csr.cuh:21-73) with Edges::ReadFromCSV
 * (core/data_structures/edgelist.cu:200-290) and GenerateVLabel
 * (core/data_structures/edgelist.cu:425).                                 */
int  mg_csr_from_csv(const char* csv_path, uint32_t label_range,
                     mg_csr_view* out, void** owner);

/* ---- synthetic inputs (seeded, counter-based Philox4x32-10) ------------- */
/* Chung-Lu power-law graph: weights c*(i+1)^(-1/(beta-1)) scaled so that
 * sum(w) = n*avg_deg; every pair i<j included with p = min(1, wi*wj/sum w);
 * symmetrised, no self-loops, sorted adjacency.                            */
int  mg_gen_chung_lu(uint32_t n, double beta, double avg_deg, uint64_t seed,
                     uint32_t threads, uint32_t** src, uint32_t** dst,
                     uint64_t* m);
/* R-MAT: 2^scale vertices, edge_factor*2^scale directed draws with
 * quadrant probabilities (a, b, c, 1-a-b-c), `scale` levels per edge.     */
int  mg_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                 double c, uint64_t seed, uint32_t threads, uint32_t** src,
                 uint32_t** dst, uint64_t* m);
void mg_free_buffer(void* p);
/* Vertex labels: kind 0 uniform over L, kind 1 Zipf P(k) ~ (k+1)^-s.     */
int  mg_gen_labels(uint32_t n, uint32_t kind, uint32_t L, double s,
                   uint64_t seed, uint32_t* labels);
/* Labelled query from a shape given as an undirected edge list over k
 * vertices; labels copied from a random walk on the data graph along the
 * query's BFS spanning tree from vertex 0.  The query is symmetrised.     */
int  mg_gen_query_walk(const mg_csr_view* g, uint32_t k, const uint32_t* eu,
                       const uint32_t* ev, uint32_t ne, uint64_t seed,
                       mg_csr_view* out, void** owner);
/* Random connected query: recursive spanning tree (vertex j joins a uniform
 * earlier vertex) plus every other pair with probability p_extra, labels by
 * random walk.                                                             */
int  mg_gen_query_random(const mg_csr_view* g, uint32_t k, double p_extra,
                         uint64_t seed, mg_csr_view* out, void** owner);
/* Query with explicit labels from an undirected edge list (symmetrised). */
int  mg_query_from_edges(uint32_t k, const uint32_t* eu, const uint32_t* ev,
                         uint32_t ne, const uint32_t* labels, int directed,
                         mg_csr_view* out, void** owner);

/* ---- matching plan ------------------------------------------------------ */
/* Replaces WOJExecutionPlan::GenerateWOJExecutionPlan
 * (core/data_structures/woj_exec_plan.cuh:33-50): writes the matching
 * order (k query-local ids) for the given graph, query and options.
 * dgraph may be NULL for MG_ORDER_REFERENCE and MG_ORDER_GIVEN.           */
int  mg_plan_order(void* dgraph, const mg_csr_view* q, const mg_opts* opts,
                   uint32_t* order, uint32_t* k);
/* Orders of nq queries at once (orders[q*MG_MAX_QUERY_VERTICES + i]); with
 * MG_ORDER_LEARNED one inference launch scores every candidate prefix of the
 * whole set.  Same plan as nq calls of WOJExecutionPlan::
 * GenerateWOJExecutionPlan (core/data_structures/woj_exec_plan.cuh:33-50). */
int  mg_plan_orders(void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                    const mg_opts* opts, uint32_t* orders);

/* ---- device graph ------------------------------------------------------- */
/* Uploads a data graph to `device` and builds the derived indices
 * (label-sliced adjacency, neighbour-label bits, label buckets).  Replaces
 * the UnifiedOwnedBuffer::Init uploads of WOJSubIsoKernelWrapper::Filter
 * (core/task/gpu_task/kernel/kernel_woj_subsio.cu:753-815).               */
int  mg_graph_upload(const mg_csr_view* g, int device, void** dgraph);
/* The same with explicit options (NULL = defaults, as mg_graph_upload).     */
int  mg_graph_upload_ex(const mg_csr_view* g, int device, const mg_upload_opts* opts,
                        void** dgraph);
void mg_graph_free(void* dgraph);
int  mg_graph_get_info(void* dgraph, mg_graph_info* info);

/* ---- matching ----------------------------------------------------------- */
/* Exact match count.  Replaces WOJSubIsoKernelWrapper::Filter + ::Join
 * (core/task/gpu_task/kernel/kernel_woj_subiso.cuh:45-51,
 * kernel_woj_subsio.cu:723-1079) as called by SubIso::WOJMatching
 * (core/task/gpu_task/subiso.cu:201-234).                                  */
int  mg_subiso_count(void* dgraph, const mg_csr_view* q, const mg_opts* opts,
                     uint64_t* count);
int  mg_subiso_count_ex(void* dgraph, const mg_csr_view* q,
                        const mg_opts* opts, uint64_t* count, mg_stats* st);
/* All matches as rows of k GLOBAL data-vertex ids in query-local-id order,
 * sorted lexicographically.  *n_rows receives the full count; when it
 * exceeds cap_rows, the first cap_rows rows in sorted order are written and
 * MG_E_CAPACITY is returned.  Replaces the join output tables
 * (core/data_structures/woj_matches.cuh:15-98) printed by
 * WOJMatches::Print (core/data_structures/woj_matches.cu:140).           */
int  mg_subiso_emit(void* dgraph, const mg_csr_view* q, const mg_opts* opts,
                    uint32_t* rows, uint64_t cap_rows, uint64_t* n_rows);
int  mg_subiso_emit_ex(void* dgraph, const mg_csr_view* q,
                       const mg_opts* opts, uint32_t* rows, uint64_t cap_rows,
                       uint64_t* n_rows, mg_stats* st);
/* Counts for nq queries in one batch against one resident data graph.
 * Replaces nq calls of SubIso::Run (core/task/gpu_task/subiso.cu:236-260). */
int  mg_subiso_batch_count(void* dgraph, const mg_csr_view* const* qs,
                           uint32_t nq, const mg_opts* opts, uint64_t* counts);
int  mg_subiso_batch_count_ex(void* dgraph, const mg_csr_view* const* qs,
                              uint32_t nq, const mg_opts* opts,
                              uint64_t* counts, mg_stats* st);

/* Batch count with one matching order per query (orders[q*16 + i], query
 * local ids; NULL = opts->order for all) and, optionally, the surviving
 * prefixes of every query: level_rows[q*(MG_MAX_QUERY_VERTICES+1) + i] = P_i
 * (i = 1..k; P_k = count).  These per-prefix counts are what the order model
 * learns from.  Replaces nq calls of SubIso::Run with a chosen order
 * (core/task/gpu_task/subiso.cu:236-260).                                  */
int  mg_subiso_batch_count_orders(void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                                  const uint32_t* orders, const mg_opts* opts,
                                  uint64_t* counts, uint64_t* level_rows, mg_stats* st);

/* ---- learned matching order ---------------------------------------------- *
 * A message-passing network over the query graph (2 layers, 64 hidden units)
 * predicts log(1 + P(S)) for connected vertex sets S of a query from the data
 * graph's label statistics; MG_ORDER_LEARNED picks the order with the least
 * predicted work.  Orders change work only, never counts.  Training uses
 * FP32 forward/backward CUDA kernels and Adam; inference uses BF16 weights.
 * Files reuse the reference's matrix container (<dir>/meta.yaml with x, y and
 * <dir>/embedding.bin, core/data_structures/matrix.cu:12-35).  The
 * reference's learned component, MatrixFilter (core/task/cpu_task/
 * cpu_subiso.cu:237-277), is a lossy candidate filter; this one is an order. */
int  mg_order_model_create(int device, uint64_t seed, void** model);
int  mg_order_model_load(const char* dir, int device, void** model);
int  mg_order_model_save(void* model, const char* dir);
void mg_order_model_free(void* model);
int  mg_order_model_num_params(void);
int  mg_order_model_get_params(void* model, float* out);
int  mg_order_model_set_params(void* model, const float* params);
/* Samples are (query index into qs, vertex-set mask over query local ids,
 * target log(1 + P)).  The loss is the mean squared error over the samples. */
int  mg_order_model_train(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                          const uint32_t* s_query, const uint32_t* s_mask, const float* s_target,
                          uint32_t ns, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                          float* final_loss);
int  mg_order_model_grad(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                         const uint32_t* s_query, const uint32_t* s_mask, const float* s_target,
                         uint32_t ns, float* grad_out, float* loss_out, float* pred_out);
int  mg_order_model_predict(void* model, void* dgraph, const mg_csr_view* const* qs, uint32_t nq,
                            const uint32_t* s_query, const uint32_t* s_mask, uint32_t ns,
                            float* out);
/* Network inputs of one query: x[16][8] (feature 5 = degree inside S is
 * computed per sample and left 0), e[16][16], adjacency masks adj[16].      */
int  mg_order_model_features(void* dgraph, const mg_csr_view* q, float* x, float* e,
                             uint32_t* adj);

/* Self-test of the bounded device waits (no counterpart in the reference;
 * the reference has no device-side wait).  The batch lane pipeline's
 * work/scan kernel waits, tile by tile, for the sums of earlier tiles; every
 * such wait gives up after a fixed number of polls and the call then returns
 * MG_E_TIMEOUT instead of spinning.  This entry point runs that kernel once
 * with the first tile never handed out, so the wait for it must run out:
 * *status receives MG_E_TIMEOUT when the bound worked (MG_OK otherwise).
 * `q` needs a second vertex joined to its first; spin_limit >= 1 polls.    */
int  mg_selftest_wait_timeout(void* dgraph, const mg_csr_view* q, uint32_t spin_limit,
                              int* status);

/* ---- lossy learned candidate filter (MatrixFilter) ---------------------
 * Replaces the reference's MatrixFilter (core/task/cpu_task/cpu_subiso.cu:
 * 237-277) with its CPU MLP helpers (core/task/gpu_task/kernel/
 * kernel_matrix_ops.cu:431-509).  dirs[0..5] are six matrices in the
 * reference's container (<dir>meta.yaml with x and y, <dir>embedding.bin
 * float32 row-major; core/data_structures/matrix.cu:12-35), in the order of
 * the reference's -m1..-m6: query-vertex embeddings (k rows x dim),
 * data-vertex embeddings (n rows x dim, row = local vertex id), W1 (hidden
 * rows x dim), b1 (hidden values), W2 (hidden x 1), b2 (1 value); hidden is
 * at most 64 and dim at most 1024.  A candidate v of query vertex u is
 * rejected when sigmoid(W2 . relu(W1 . (e_u - e_v)^2 + b1) + b2) < 0.1, with
 * every product and sum rounded to float32 in the reference's order.  With
 * mg_opts.matrix_filter set, the level-0 candidates (the first vertex of the
 * matching order) are filtered; counts then lose the matches of rejected
 * roots.  Off by default, as in the reference's CLI. */
int  mg_matrix_filter_load(const char* const dirs[6], int device, void** filter);
void mg_matrix_filter_free(void* filter);
/* keep[i] = 1 when the filter keeps (u, v[i]); host arrays; u < k rows of
 * dirs[0], every v[i] < n rows of dirs[1]. */
int  mg_matrix_filter_keep(void* filter, uint32_t u, const uint32_t* v, uint64_t nv,
                           uint8_t* keep);

/* Exact count that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory when they ask for a count:
 * processes whose HBM is owned by another allocator (a framework's caching
 * allocator or a fixed arena that has reserved nearly all of it), and
 * latency-critical paths that must not pay for cudaMalloc/cudaFree or the
 * device-wide synchronisation cudaFree implies.  The enumeration scratch
 * (level tables, scan space, counters, plan) lives in one file-scope device
 * array of MG_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until the process exits; the level tables are sized to fit it, so any
 * match count is reachable (more, smaller chunks).  A caller-set chunk_rows
 * whose tables do not fit is rejected with MG_E_LIMIT.  The data graph must
 * already be resident (mg_graph_upload); orders: reference, strong, given.
 * The closed-form two-position endings are not used (the pendant tail's
 * aggregate tables would need scratch of their own), so no_tail is ignored;
 * counts are the same.
 * The first call on a device looks up the array's device address with that
 * device current; make that first call before any stream capture.  Every
 * call shares the array and leaves its contents behind (counters are
 * cleared at the start of each call); calls are serialised by a process-wide
 * lock, since calls that overlapped on the GPU would race on the array.    */
#define MG_NOALLOC_SCRATCH_BYTES (16u << 20)
int  mg_subiso_count_noalloc(void* dgraph, const mg_csr_view* q, const mg_opts* opts,
                             uint64_t* count);

#ifdef __cplusplus
}
#endif
#endif /* MG_SUBISO_H_ */
