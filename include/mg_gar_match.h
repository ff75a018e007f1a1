/* GAR (graph association rule) pattern match over edge lists — C-ABI of
 * libmg_subiso.so.
 *
 * matrixgraph_gar_match replaces the entry point of the same name and
 * signature in the reference's Go/cgo library libmatrixgraph_goapi.so
 * (core/go_api/matrixgraph_go_api.h:30-55, implemented by
 * core/go_api/matrixgraph_go_api.cu:209-227 -> GARMatch::Run,
 * core/task/gpu_task/gar_match.cu:193-240 ->
 * GARMatchKernelWrapper::GARMatch,
 * core/task/gpu_task/kernel/kernel_gar_match.cu:365-709).
 *
 * Inputs (host memory, caller-owned):
 *   data graph: n vertices by local index 0..n-1 with instance ids g_v_id
 *     (NULL: the local index is the id) and labels g_v_label_idx; directed
 *     edges (g_e_src[i] -> g_e_dst[i]) by local index with labels
 *     g_e_label_idx (NULL: edge labels are not compared); g_e_id is unused.
 *   pattern: p_n_nodes nodes with labels p_node_label_idx; directed edges
 *     (p_edge_src[j] -> p_edge_dst[j]) with labels p_edge_label_idx (NULL:
 *     every pattern edge has label 0).
 * A match is an injective map f of the pattern nodes onto data vertices with
 * equal labels such that every pattern edge (s, d, l) has a data edge
 * (f(s), f(d)) labelled l.  Pattern node 0 is the pivot.
 *
 * Output (GARMatchArrays, core/data_structures/gar_match_arrays.h:14-51):
 * for every pivot vertex (ascending local index) that has a match, one row
 * per pattern position pos = 0..p_n_nodes-1: row_pivot_id = pivot instance
 * id, row_cond_j = row_pos = pos, and the sorted distinct instance ids that
 * position takes over the pivot's matches, stored at
 * out_matched_v_ids[row_offset .. row_offset + row_count).  Rows stop at
 * out_row_capacity and ids at out_match_capacity exactly as in the
 * reference (the row that meets the id capacity is written with the ids
 * that fit, then output stops).  *out_num_conditions = p_n_nodes when at
 * least one match exists, else 1 (with zero rows), as in the reference.
 * Any output pointer may be NULL; its writes are skipped.
 *
 * Differences from the reference, all deliberate:
 *   - every match is found: the reference keeps at most
 *     out_match_capacity / p_n_nodes partial matches per join step and
 *     drops the rest in arrival order, and its k-min-wise vertex filter
 *     (heap of 7 label hashes) can reject a vertex that a match uses; where
 *     neither happens the outputs are identical;
 *   - a CUDA or allocation failure returns a non-zero MG_E_* code with the
 *     message in mg_last_error() instead of ending the process;
 *   - MATRIXGRAPH_CUDA_DEVICE selects the device as in the reference, but the
 *     calling thread's current device is left unchanged.
 * Patterns are limited to p_n_nodes + (distinct pattern edges when they use
 * two or more edge labels) <= 16 (MG_E_LIMIT beyond).
 * Returns 0 on success, non-zero on error.                                   */
#ifndef MG_GAR_MATCH_H_
#define MG_GAR_MATCH_H_

#include <stdint.h>

#include "mg_subiso.h"

#ifdef __cplusplus
extern "C" {
#endif

int matrixgraph_gar_match(
    const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
    const uint32_t* g_e_src, const uint32_t* g_e_dst, const uint32_t* g_e_id,
    const int32_t* g_e_label_idx, int g_n_edges,
    const int32_t* p_node_label_idx, int p_n_nodes,
    const int32_t* p_edge_src, const int32_t* p_edge_dst,
    const int32_t* p_edge_label_idx, int p_n_edges,
    int* out_num_conditions, uint32_t* out_row_pivot_id, int32_t* out_row_cond_j,
    int32_t* out_row_pos, int32_t* out_row_offset, int32_t* out_row_count,
    int out_row_capacity, int* out_row_size,
    uint32_t* out_matched_v_ids, int out_match_capacity, int* out_match_size);

/* Same as matrixgraph_gar_match, with enumeration options (order, filters,
 * budgets; root_begin/root_end are ignored) and the number of distinct
 * matches written to *n_matches (may be NULL).  No counterpart in the
 * reference.                                                                 */
int mg_gar_match_ex(
    const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
    const uint32_t* g_e_src, const uint32_t* g_e_dst, const uint32_t* g_e_id,
    const int32_t* g_e_label_idx, int g_n_edges,
    const int32_t* p_node_label_idx, int p_n_nodes,
    const int32_t* p_edge_src, const int32_t* p_edge_dst,
    const int32_t* p_edge_label_idx, int p_n_edges,
    int* out_num_conditions, uint32_t* out_row_pivot_id, int32_t* out_row_cond_j,
    int32_t* out_row_pos, int32_t* out_row_offset, int32_t* out_row_count,
    int out_row_capacity, int* out_row_size,
    uint32_t* out_matched_v_ids, int out_match_capacity, int* out_match_size,
    const mg_opts* opts, uint64_t* n_matches);

/* The two host halves of mg_gar_match_ex, for callers that match the
 * instance themselves and for host-only tests.  No counterpart in the
 * reference.
 *
 * mg_gar_instance: the matching instance of a (graph, pattern) pair, as a
 * reference-layout data CSR (vertices 0..n-1 are the graph's local indices,
 * followed by one vertex per usable labelled edge when the pattern uses two
 * or more edge labels) and a directed query whose vertices 0..p_n_nodes-1
 * are the pattern nodes.  When the answer is empty without matching, both
 * owners are set to NULL and MG_OK is returned.  Free the owners with
 * mg_csr_dir_close.
 *
 * mg_gar_flatten: the GARMatchArrays output from match rows of row_width
 * ids whose first n_nodes entries are the pattern nodes' local indices (any
 * row order, repeats allowed).                                             */
int mg_gar_instance(
    const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
    const uint32_t* g_e_src, const uint32_t* g_e_dst, const int32_t* g_e_label_idx,
    int g_n_edges, const int32_t* p_node_label_idx, int p_n_nodes,
    const int32_t* p_edge_src, const int32_t* p_edge_dst,
    const int32_t* p_edge_label_idx, int p_n_edges,
    mg_csr_view* data, void** data_owner, mg_csr_view* query, void** query_owner);

int mg_gar_flatten(
    const uint32_t* rows, uint64_t n_rows, uint32_t row_width, uint32_t n_nodes,
    const uint32_t* g_v_id, int g_n_vertices,
    int* out_num_conditions, uint32_t* out_row_pivot_id, int32_t* out_row_cond_j,
    int32_t* out_row_pos, int32_t* out_row_offset, int32_t* out_row_count,
    int out_row_capacity, int* out_row_size,
    uint32_t* out_matched_v_ids, int out_match_capacity, int* out_match_size);

#ifdef __cplusplus
}
#endif

#endif /* MG_GAR_MATCH_H_ */
