#include "matrixgraph.h"

#include <chrono>
#include <fstream>
#include <sstream>
#include <iostream>

namespace matrixgraph {

void Check(int rc) {
  if (rc != MG_OK) throw Error(rc, mg_last_error());
}

SubIso::SubIso(const std::string& pattern_path, const std::string& data_graph_path,
               const std::string& data_graph_edgelist_path, const std::string& output_path,
               const std::string& mode, int order, int device, const std::string& model_path,
               const std::vector<std::string>& matrix_paths)
    : pattern_path_(pattern_path),
      data_graph_path_(data_graph_path),
      data_graph_edgelist_path_(data_graph_edgelist_path),
      output_path_(output_path),
      mode_(mode),
      model_path_(model_path),
      matrix_paths_(matrix_paths),
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
  void* model = nullptr;
  if (order_ == MG_ORDER_LEARNED && !model_path_.empty())
    Check(mg_order_model_load(model_path_.c_str(), device_, &model));
  void* filter = nullptr;
  if (matrix_paths_.size() == 6) {
    const char* dirs[6];
    for (int i = 0; i < 6; ++i) dirs[i] = matrix_paths_[i].c_str();
    int frc = mg_matrix_filter_load(dirs, device_, &filter);
    if (frc != MG_OK) {
      const std::string msg = mg_last_error();
      if (model) mg_order_model_free(model);
      throw Error(frc, msg);
    }
  }
  void* dg = nullptr;
  int rc = mg_graph_upload(&g_, device_, &dg);
  if (rc != MG_OK) {
    const std::string msg = mg_last_error();
    if (model) mg_order_model_free(model);
    if (filter) mg_matrix_filter_free(filter);
    throw Error(rc, msg);
  }
  mg_opts o;
  mg_opts_default(&o);
  o.order = order_;
  o.model = model;
  o.matrix_filter = filter;
  mg_stats st;
  rc = mg_subiso_count_ex(dg, &p_, &o, &count_, &st);
  if (rc == MG_OK && mode_ == "emit") {
    k_ = p_.n;
    rows_.assign(count_ * k_, 0);
    uint64_t n = 0;
    rc = mg_subiso_emit(dg, &p_, &o, rows_.data(), count_, &n);
  }
  auto t2 = std::chrono::steady_clock::now();
  const std::string msg = rc == MG_OK ? "" : mg_last_error();
  mg_graph_free(dg);
  if (model) mg_order_model_free(model);
  if (filter) mg_matrix_filter_free(filter);
  if (rc != MG_OK) throw Error(rc, msg);
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

BatchSubIso::BatchSubIso(const std::vector<std::string>& pattern_paths,
                         const std::string& data_graph_path, const std::string& output_path,
                         int order, const std::string& model_path, int device,
                         const std::string& tune_path)
    : pattern_paths_(pattern_paths),
      data_graph_path_(data_graph_path),
      output_path_(output_path),
      model_path_(model_path),
      tune_path_(tune_path),
      order_(order),
      device_(device) {}

namespace {
struct TuneRow {
  uint32_t k_lo, k_hi, lanes, probe_min, grab;
};

// Rows of an autotuner table whose signature is this graph's.
std::vector<TuneRow> ReadTuneTable(const std::string& path, const mg_graph_info& gi) {
  std::ifstream f(path);
  if (!f) throw Error(MG_E_IO, "cannot read the tune table " + path);
  const std::string sig = "n" + std::to_string(gi.n) + ".m" + std::to_string(gi.m_out) + ".L" +
                          std::to_string(gi.n_labels) + ".d" + std::to_string(gi.max_degree);
  std::vector<TuneRow> rows;
  for (std::string line; std::getline(f, line);) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream in(line);
    std::string s;
    TuneRow r{};
    if ((in >> s >> r.k_lo >> r.k_hi >> r.lanes >> r.probe_min >> r.grab) && s == sig)
      rows.push_back(r);
  }
  return rows;
}
}  // namespace

BatchSubIso::~BatchSubIso() {
  for (void* o : p_owner_)
    if (o) mg_csr_dir_close(o);
  if (g_owner_) mg_csr_dir_close(g_owner_);
}

void BatchSubIso::Run() {
  if (pattern_paths_.empty()) throw Error(MG_E_ARG, "no pattern paths in the batch");
  p_.assign(pattern_paths_.size(), mg_csr_view{});
  p_owner_.assign(pattern_paths_.size(), nullptr);
  for (size_t i = 0; i < pattern_paths_.size(); ++i)
    Check(mg_csr_dir_open(pattern_paths_[i].c_str(), &p_[i], &p_owner_[i]));
  Check(mg_csr_dir_open(data_graph_path_.c_str(), &g_, &g_owner_));
  void* model = nullptr;
  if (order_ == MG_ORDER_LEARNED && !model_path_.empty())
    Check(mg_order_model_load(model_path_.c_str(), device_, &model));
  void* dg = nullptr;
  int rc = mg_graph_upload(&g_, device_, &dg);
  if (rc == MG_OK) {
    mg_opts o;
    mg_opts_default(&o);
    o.order = order_;
    o.model = model;
    std::vector<const mg_csr_view*> qs;
    for (auto& v : p_) qs.push_back(&v);
    counts_.assign(qs.size(), 0);
    mg_stats st;
    std::vector<TuneRow> tune;
    if (!tune_path_.empty()) {
      mg_graph_info gi;
      Check(mg_graph_get_info(dg, &gi));
      tune = ReadTuneTable(tune_path_, gi);
    }
    if (tune.empty()) {
      rc = mg_subiso_batch_count_ex(dg, qs.data(), uint32_t(qs.size()), &o, counts_.data(),
                                    &st);
      if (rc == MG_OK)
        std::cout << "[BatchSubIso] " << qs.size() << " patterns, device " << st.device_ms
                  << " ms, " << st.launches << " launches" << std::endl;
    } else {
      // one batched call per tuned size bucket, then the leftover sizes
      std::vector<char> done(qs.size(), 0);
      for (size_t b = 0; b <= tune.size() && rc == MG_OK; ++b) {
        std::vector<const mg_csr_view*> part;
        std::vector<size_t> idx;
        for (size_t i = 0; i < qs.size(); ++i) {
          const uint32_t k = qs[i]->n;
          const bool in = b < tune.size() ? (k >= tune[b].k_lo && k <= tune[b].k_hi) : !done[i];
          if (in && !done[i]) {
            part.push_back(qs[i]);
            idx.push_back(i);
            done[i] = 1;
          }
        }
        if (part.empty()) continue;
        mg_opts ob = o;
        if (b < tune.size()) {
          ob.lanes = tune[b].lanes;
          ob.probe_min = tune[b].probe_min;
          ob.grab = tune[b].grab;
        }
        std::vector<uint64_t> c(part.size(), 0);
        rc = mg_subiso_batch_count(dg, part.data(), uint32_t(part.size()), &ob, c.data());
        for (size_t j = 0; j < idx.size() && rc == MG_OK; ++j) counts_[idx[j]] = c[j];
      }
      if (rc == MG_OK)
        std::cout << "[BatchSubIso] " << qs.size() << " patterns, tuned by " << tune_path_
                  << std::endl;
    }
  }
  const std::string msg = rc == MG_OK ? "" : mg_last_error();
  if (dg) mg_graph_free(dg);
  if (model) mg_order_model_free(model);
  if (rc != MG_OK) throw Error(rc, msg);
  std::ostream* os = &std::cout;
  std::ofstream f;
  if (!output_path_.empty()) {
    f.open(output_path_);
    if (!f) throw Error(MG_E_IO, "cannot write " + output_path_);
    os = &f;
  }
  for (size_t i = 0; i < counts_.size(); ++i)
    *os << pattern_paths_[i] << " " << counts_[i] << "\n";
}

int GARMatch::Run(const uint32_t* g_v_id, const int32_t* g_v_label_idx, int g_n_vertices,
                  const uint32_t* g_e_src, const uint32_t* g_e_dst, const uint32_t* g_e_id,
                  const int32_t* g_e_label_idx, int g_n_edges, const int32_t* p_node_label_idx,
                  int p_n_nodes, const int32_t* p_edge_src, const int32_t* p_edge_dst,
                  const int32_t* p_edge_label_idx, int p_n_edges, int* out_num_conditions,
                  uint32_t* out_row_pivot_id, int32_t* out_row_cond_j, int32_t* out_row_pos,
                  int32_t* out_row_offset, int32_t* out_row_count, int out_row_capacity,
                  int* out_row_size, uint32_t* out_matched_v_ids, int out_match_capacity,
                  int* out_match_size) {
  return matrixgraph_gar_match(g_v_id, g_v_label_idx, g_n_vertices, g_e_src, g_e_dst, g_e_id,
                               g_e_label_idx, g_n_edges, p_node_label_idx, p_n_nodes,
                               p_edge_src, p_edge_dst, p_edge_label_idx, p_n_edges,
                               out_num_conditions, out_row_pivot_id, out_row_cond_j,
                               out_row_pos, out_row_offset, out_row_count, out_row_capacity,
                               out_row_size, out_matched_v_ids, out_match_capacity,
                               out_match_size);
}

void GARMatch::Run() {
  if (!out_) {  // the reference's wrapper returns 1 without an output object
    status_ = 1;
    return;
  }
  status_ = Run(g_.v_id, g_.v_label_idx, g_.n_vertices, g_.e_src, g_.e_dst, g_.e_id,
                g_.e_label_idx, g_.n_edges, p_.node_label_idx, p_.n_nodes, p_.edge_src,
                p_.edge_dst, p_.edge_label_idx, p_.n_edges, out_->num_conditions,
                out_->row_pivot_id, out_->row_cond_j, out_->row_pos, out_->row_offset,
                out_->row_count, out_->row_capacity, out_->row_size, out_->matched_v_ids,
                out_->match_capacity, out_->match_size);
  if (status_ != MG_OK) std::cerr << "[GARMatch] " << mg_last_error() << std::endl;
}

void MatrixGraph::Run(TaskType type, SubIso* task) {
  (void)scheduler_;
  if (type != kSubIso) throw Error(MG_E_ARG, "a SubIso task needs kSubIso");
  task->Run();
}

void MatrixGraph::Run(TaskType type, BatchSubIso* task) {
  (void)scheduler_;
  if (type != kSubIso) throw Error(MG_E_ARG, "a BatchSubIso task needs kSubIso");
  task->Run();
}

void MatrixGraph::Run(TaskType type, GARMatch* task) {
  (void)scheduler_;
  if (type != kGARMatch) throw Error(MG_E_ARG, "a GARMatch task needs kGARMatch");
  task->Run();
}

}  // namespace matrixgraph
