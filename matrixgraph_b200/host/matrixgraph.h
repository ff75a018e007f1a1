// Host-side mirror of the reference's subiso task and runtime dispatch,
// written over the C-ABI of libmg_subiso.so.
//
//   SubIso(pattern_path, data_graph_path, data_graph_edgelist_path,
//          output_path).Run()         core/task/gpu_task/subiso.cuh:43-51
//   MatrixGraph(scheduler).Run(kSubIso, task)
//                                     core/matrixgraph.cuh:36-42, matrixgraph.cu:30-46
//
// Differences from the reference: the count is exact; errors raise
// std::runtime_error with the library's message instead of exiting.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

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
  SubIso(const std::string& pattern_path, const std::string& data_graph_path,
         const std::string& data_graph_edgelist_path, const std::string& output_path,
         const std::string& mode = "count", int order = MG_ORDER_REFERENCE, int device = 0);
  ~SubIso();
  void Run();

  uint64_t count() const { return count_; }
  const std::vector<uint32_t>& rows() const { return rows_; }
  double match_ms() const { return match_ms_; }

 private:
  void LoadData();
  void Write() const;

  std::string pattern_path_, data_graph_path_, data_graph_edgelist_path_, output_path_;
  std::string mode_;
  int order_, device_;
  mg_csr_view p_{}, g_{};
  void* p_owner_ = nullptr;
  void* g_owner_ = nullptr;
  uint64_t count_ = 0;
  uint32_t k_ = 0;
  std::vector<uint32_t> rows_;
  double match_ms_ = 0;
};

class MatrixGraph {
 public:
  explicit MatrixGraph(SchedulerType scheduler = kCHBL) : scheduler_(scheduler) {}
  void Run(TaskType type, SubIso* task);

 private:
  SchedulerType scheduler_;  // accepted and ignored by subiso, as in the reference
};

}  // namespace matrixgraph
