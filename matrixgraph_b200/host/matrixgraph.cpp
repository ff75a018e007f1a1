#include "matrixgraph.h"

#include <chrono>
#include <fstream>
#include <iostream>

namespace matrixgraph {

void Check(int rc) {
  if (rc != MG_OK) throw Error(rc, mg_last_error());
}

SubIso::SubIso(const std::string& pattern_path, const std::string& data_graph_path,
               const std::string& data_graph_edgelist_path, const std::string& output_path,
               const std::string& mode, int order, int device)
    : pattern_path_(pattern_path),
      data_graph_path_(data_graph_path),
      data_graph_edgelist_path_(data_graph_edgelist_path),
      output_path_(output_path),
      mode_(mode),
      order_(order),
      device_(device) {}

SubIso::~SubIso() {
  if (p_owner_) mg_csr_dir_close(p_owner_);
  if (g_owner_) mg_csr_dir_close(g_owner_);
}

void SubIso::LoadData() {
  std::cout << "[SubIso] LoadData() ..." << std::endl;
  Check(mg_csr_dir_open(pattern_path_.c_str(), &p_, &p_owner_));
  Check(mg_csr_dir_open(data_graph_path_.c_str(), &g_, &g_owner_));
}

void SubIso::Run() {
  auto t0 = std::chrono::steady_clock::now();
  LoadData();
  auto t1 = std::chrono::steady_clock::now();
  void* dg = nullptr;
  Check(mg_graph_upload(&g_, device_, &dg));
  mg_opts o;
  mg_opts_default(&o);
  o.order = order_;
  mg_stats st;
  int rc = mg_subiso_count_ex(dg, &p_, &o, &count_, &st);
  if (rc == MG_OK && mode_ == "emit") {
    k_ = p_.n;
    rows_.assign(count_ * k_, 0);
    uint64_t n = 0;
    rc = mg_subiso_emit(dg, &p_, &o, rows_.data(), count_, &n);
  }
  auto t2 = std::chrono::steady_clock::now();
  mg_graph_free(dg);
  Check(rc);
  match_ms_ = st.device_ms;
  std::cout << "[SubIso] LoadData() elapsed: "
            << std::chrono::duration<double>(t1 - t0).count() << " s" << std::endl;
  std::cout << "[SubIso] Matching() elapsed: "
            << std::chrono::duration<double>(t2 - t1).count() << " s (device "
            << st.device_ms << " ms)" << std::endl;
  std::cout << "[SubIso] exact matches: " << count_ << std::endl;
  if (!output_path_.empty()) Write();
}

void SubIso::Write() const {
  std::ofstream f(output_path_);
  if (!f) throw Error(MG_E_IO, "cannot write " + output_path_);
  f << count_ << "\n";
  for (uint64_t r = 0; k_ && r < rows_.size() / k_; ++r) {
    for (uint32_t c = 0; c < k_; ++c) f << (c ? "," : "") << rows_[r * k_ + c];
    f << "\n";
  }
}

void MatrixGraph::Run(TaskType type, SubIso* task) {
  (void)scheduler_;
  if (type != kSubIso) throw Error(MG_E_ARG, "only kSubIso is served");
  task->Run();
}

}  // namespace matrixgraph
