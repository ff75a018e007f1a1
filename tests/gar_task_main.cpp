// Drives the C++ GARMatch task mirror (matrixgraph_b200/host/matrixgraph.h)
// on the example of the reference's GARMatchArrays documentation
// (core/data_structures/gar_match_arrays.h:33-51) and prints the outputs.
// argv[1]: "example" (a match exists) or "no_edges" (empty pattern edge set).
#include <cstdio>
#include <cstring>
#include <vector>

#include "matrixgraph.h"

int main(int argc, char** argv) {
  const bool no_edges = argc > 1 && std::strcmp(argv[1], "no_edges") == 0;
  const std::vector<uint32_t> v_id = {126, 138, 183, 115407, 192};
  const std::vector<int32_t> v_label = {0, 0, 1, 1, 1};
  const std::vector<uint32_t> e_src = {0, 0, 1}, e_dst = {2, 3, 4}, e_id = {0, 1, 2};
  const std::vector<int32_t> e_label = {5, 5, 5};
  const std::vector<int32_t> p_label = {0, 1}, p_src = {0}, p_dst = {1}, p_elabel = {5};

  matrixgraph::GARGraphArrays g;
  g.v_id = v_id.data();
  g.v_label_idx = v_label.data();
  g.n_vertices = 5;
  g.e_src = e_src.data();
  g.e_dst = e_dst.data();
  g.e_id = e_id.data();
  g.e_label_idx = e_label.data();
  g.n_edges = 3;
  matrixgraph::GARPatternArrays p;
  p.node_label_idx = p_label.data();
  p.n_nodes = 2;
  p.edge_src = p_src.data();
  p.edge_dst = p_dst.data();
  p.edge_label_idx = p_elabel.data();
  p.n_edges = no_edges ? 0 : 1;

  int nc = -9, rs = -9, ms = -9;
  std::vector<uint32_t> pivot(16), ids(16);
  std::vector<int32_t> cond(16), pos(16), off(16), cnt(16);
  matrixgraph::GARMatchArrays out;
  out.num_conditions = &nc;
  out.row_pivot_id = pivot.data();
  out.row_cond_j = cond.data();
  out.row_pos = pos.data();
  out.row_offset = off.data();
  out.row_count = cnt.data();
  out.row_capacity = 16;
  out.row_size = &rs;
  out.matched_v_ids = ids.data();
  out.match_capacity = 16;
  out.match_size = &ms;

  matrixgraph::GARMatch task(g, p, &out);
  matrixgraph::MatrixGraph system;
  system.Run(matrixgraph::kGARMatch, &task);
  std::printf("status=%d num_conditions=%d row_size=%d match_size=%d\n", task.Status(), nc, rs,
              ms);
  for (int i = 0; i < rs; ++i)
    std::printf("row %u %d %d %d %d\n", pivot[i], cond[i], pos[i], off[i], cnt[i]);
  std::printf("ids");
  for (int i = 0; i < ms; ++i) std::printf(" %u", ids[i]);
  std::printf("\n");
  return 0;
}
