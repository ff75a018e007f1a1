// Host-side mirror of the reference's subiso task and runtime dispatch,
// written over the C-ABI of libmg_subiso.so.
//
//   SubIso(pattern_path, data_graph_path, data_graph_edgelist_path,
//          output_path).Run()         core/task/gpu_task/subiso.cuh:43-51
//   MatrixGraph(scheduler).Run(kSubIso, task)
//                                     core/matrixgraph.cuh:36-42, matrixgraph.cu:30-46
//   GARMatch(g, p, out).Run(), GARMatch::Run(arrays...)
//                                     core/task/gpu_task/gar_match.cuh:33-70
//
// Differences from the reference: the count is exact; errors raise
// std::runtime_error with the library's message instead of exiting.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "mg_gar_match.h"
#include "mg_subiso.h"

namespace matrixgraph {

enum TaskType { kGEMM, kMatrixAnalysis, kPPRQuery, kSubIso, kGARMatch, kCPUSubIso,
                kWCC, kSSSP, kBFS, kPageRank, kGEMV };
enum SchedulerType { kCHBL, kEvenSplit, kRoundRobin };

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

void Check(int rc);

class SubIso {
 public:
  // matrix_paths: the six directories of the reference CPUSubIso's
  // matrix_path1..6 (core/task/cpu_task/cpu_subiso.cuh:32-39); all six set
  // turn on the lossy MatrixFilter on the level-0 candidates.
  SubIso(const std::string& pattern_path, const std::string& data_graph_path,
         const std::string& data_graph_edgelist_path, const std::string& output_path,
         const std::string& mode = "count", int order = MG_ORDER_REFERENCE, int device = 0,
         const std::string& model_path = "",
         const std::vector<std::string>& matrix_paths = {});
  ~SubIso();
  void Run();

  uint64_t count() const { return count_; }
  const std::vector<uint32_t>& rows() const { return rows_; }
  double match_ms() const { return match_ms_; }

 private:
  void LoadData();
  void Write() const;

  std::string pattern_path_, data_graph_path_, data_graph_edgelist_path_, output_path_;
  std::string mode_, model_path_;
  std::vector<std::string> matrix_paths_;
  int order_, device_;
  mg_csr_view p_{}, g_{};
  void* p_owner_ = nullptr;
  void* g_owner_ = nullptr;
  uint64_t count_ = 0;
  uint32_t k_ = 0;
  std::vector<uint32_t> rows_;
  double match_ms_ = 0;
};

// Many patterns against one resident data graph in one batched call
// (mg_subiso_batch_count_ex, learned orders planned in one inference
// launch).  No counterpart in the reference, whose CLI takes one pattern.
class BatchSubIso {
 public:
  // tune_path: an autotuner table (matrixgraph_b200/autotune.py): rows
  // "signature k_lo k_hi lanes probe_min grab seconds"; the rows of this
  // graph's signature set the launch options of each query-size bucket.
  BatchSubIso(const std::vector<std::string>& pattern_paths, const std::string& data_graph_path,
              const std::string& output_path, int order = MG_ORDER_REFERENCE,
              const std::string& model_path = "", int device = 0,
              const std::string& tune_path = "");
  ~BatchSubIso();
  void Run();

  const std::vector<uint64_t>& counts() const { return counts_; }

 private:
  std::vector<std::string> pattern_paths_;
  std::string data_graph_path_, output_path_, model_path_, tune_path_;
  int order_, device_;
  std::vector<mg_csr_view> p_;
  std::vector<void*> p_owner_;
  mg_csr_view g_{};
  void* g_owner_ = nullptr;
  std::vector<uint64_t> counts_;
};

// GAR match over serialized arrays: the reference's GARGraphArrays,
// GARPatternArrays and GARMatchArrays (core/data_structures/
// gar_graph_arrays.h, gar_pattern_arrays.h, gar_match_arrays.h:56-70) and
// the array-based GARMatch task (core/task/gpu_task/gar_match.cuh:33-70).
// The config-file constructor of the reference (an ArangoDB loader) has no
// counterpart here.
struct GARGraphArrays {
  const uint32_t* v_id = nullptr;
  const int32_t* v_label_idx = nullptr;
  int n_vertices = 0;
  const uint32_t* e_src = nullptr;
  const uint32_t* e_dst = nullptr;
  const uint32_t* e_id = nullptr;
  const int32_t* e_label_idx = nullptr;
  int n_edges = 0;
};

struct GARPatternArrays {
  const int32_t* node_label_idx = nullptr;
  int n_nodes = 0;
  const int32_t* edge_src = nullptr;
  const int32_t* edge_dst = nullptr;
  const int32_t* edge_label_idx = nullptr;
  int n_edges = 0;
};

struct GARMatchArrays {
  int* num_conditions = nullptr;
  uint32_t* row_pivot_id = nullptr;
  int32_t* row_cond_j = nullptr;
  int32_t* row_pos = nullptr;
  int32_t* row_offset = nullptr;
  int32_t* row_count = nullptr;
  int row_capacity = 0;
  int* row_size = nullptr;
  uint32_t* matched_v_ids = nullptr;
  int match_capacity = 0;
  int* match_size = nullptr;
};

class GARMatch {
 public:
  GARMatch(const GARGraphArrays& g, const GARPatternArrays& p, GARMatchArrays* out)
      : g_(g), p_(p), out_(out) {}

  // C-style entry (the reference's static GARMatch::Run): 0 on success.
  static int Run(const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
                 const uint32_t* g_e_src, const uint32_t* g_e_dst, const uint32_t* g_e_id,
                 const int32_t* g_e_label_idx, int g_n_edges, const int32_t* p_node_label_idx,
                 int p_n_nodes, const int32_t* p_edge_src, const int32_t* p_edge_dst,
                 const int32_t* p_edge_label_idx, int p_n_edges, int* out_num_conditions,
                 uint32_t* out_row_pivot_id, int32_t* out_row_cond_j, int32_t* out_row_pos,
                 int32_t* out_row_offset, int32_t* out_row_count, int out_row_capacity,
                 int* out_row_size, uint32_t* out_matched_v_ids, int out_match_capacity,
                 int* out_match_size);

  // Matches the arrays given at construction; the status is kept in
  // Status() (0 on success, an MG_E_* code otherwise) instead of ending the
  // process on a CUDA error.
  void Run();
  int Status() const { return status_; }

 private:
  GARGraphArrays g_;
  GARPatternArrays p_;
  GARMatchArrays* out_;
  int status_ = 1;
};

class MatrixGraph {
 public:
  explicit MatrixGraph(SchedulerType scheduler = kCHBL) : scheduler_(scheduler) {}
  void Run(TaskType type, SubIso* task);
  void Run(TaskType type, BatchSubIso* task);
  void Run(TaskType type, GARMatch* task);

 private:
  SchedulerType scheduler_;  // accepted and ignored by subiso, as in the reference
};

}  // namespace matrixgraph
