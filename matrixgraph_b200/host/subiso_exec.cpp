// subiso_exec: the reference's subiso CLI (apps/subiso.cu:16-97) over the
// C-ABI.  Flags: -p <pattern dir/> -g <graph dir/> [-e <edge list, unused>]
// [-o <output>] [-scheduler CHBL|EvenSplit|RoundRobin] plus
// [-mode count|emit] [-order reference|heuristic|strong|learned]
// [-model <order model dir/>] [-batch <file of pattern dirs, one per line>]
// [-device N] [-tune <autotuner table>] [-m1 .. -m6 <matrix dir/>].  With
// -batch, -p is not needed and every pattern is counted in batched calls (one
// per tuned query-size bucket with -tune); -o receives "pattern count" lines.
// -m1..-m6 are the six matrices of the reference CPU subiso's MatrixFilter
// (apps/cpu_subiso.cpp, core/task/cpu_task/cpu_subiso.cuh:32-39): all six
// turn on the lossy learned filter of the level-0 candidates (single
// pattern only).
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "matrixgraph.h"

using matrixgraph::MatrixGraph;
using matrixgraph::SchedulerType;
using matrixgraph::SubIso;

static SchedulerType Scheduler2Enum(const std::string& s) {
  if (s == "EvenSplit") return matrixgraph::kEvenSplit;
  if (s == "RoundRobin") return matrixgraph::kRoundRobin;
  return matrixgraph::kCHBL;
}

int main(int argc, char** argv) {
  std::map<std::string, std::string> flags = {
      {"p", ""}, {"g", ""}, {"e", ""}, {"o", ""}, {"scheduler", "CHBL"},
      {"mode", "count"}, {"order", "reference"}, {"device", "0"}, {"batch", ""},
      {"model", ""}, {"tune", ""}, {"m1", ""}, {"m2", ""}, {"m3", ""}, {"m4", ""},
      {"m5", ""}, {"m6", ""}};
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    while (!a.empty() && a[0] == '-') a = a.substr(1);
    std::string v;
    size_t eq = a.find('=');
    if (eq != std::string::npos) {
      v = a.substr(eq + 1);
      a = a.substr(0, eq);
    } else if (i + 1 < argc) {
      v = argv[++i];
    }
    if (!flags.count(a)) {
      std::cerr << "Error: unknown flag -" << a << std::endl;
      return EXIT_FAILURE;
    }
    flags[a] = v;
  }
  bool ok = true;
  static const std::map<std::string, int> kOrders = {{"reference", MG_ORDER_REFERENCE},
                                                     {"heuristic", MG_ORDER_REFERENCE},
                                                     {"strong", MG_ORDER_STRONG},
                                                     {"learned", MG_ORDER_LEARNED}};
  if (!kOrders.count(flags["order"])) {
    std::cerr << "Error: unknown order " << flags["order"] << std::endl;
    ok = false;
  }
  if (flags["order"] == "learned" && flags["model"].empty()) {
    std::cerr << "Error: -order learned needs -model <order model dir/>" << std::endl;
    ok = false;
  }
  std::vector<std::string> batch;
  if (!flags["batch"].empty()) {
    std::ifstream f(flags["batch"]);
    if (!f) {
      std::cerr << "Error: cannot read the batch list " << flags["batch"] << std::endl;
      return EXIT_FAILURE;
    }
    for (std::string line; std::getline(f, line);) {
      while (!line.empty() && (line.back() == '\r' || line.back() == ' ')) line.pop_back();
      if (!line.empty() && line[0] != '#') batch.push_back(line);
    }
    if (batch.empty()) {
      std::cerr << "Error: the batch list " << flags["batch"] << " names no pattern" << std::endl;
      ok = false;
    }
  }
  if (flags["p"].empty() && batch.empty()) {
    std::cerr << "Error: Pattern graph path (-p) is required" << std::endl;
    ok = false;
  }
  if (flags["g"].empty()) {
    std::cerr << "Error: Data graph path (-g) is required" << std::endl;
    ok = false;
  }
  std::vector<std::string> matrix_paths;
  for (const char* m : {"m1", "m2", "m3", "m4", "m5", "m6"})
    if (!flags[m].empty()) matrix_paths.push_back(flags[m]);
  if (!matrix_paths.empty() && matrix_paths.size() != 6) {
    std::cerr << "Error: the matrix filter needs all of -m1 .. -m6" << std::endl;
    ok = false;
  }
  if (!matrix_paths.empty() && !batch.empty()) {
    std::cerr << "Error: -m1 .. -m6 apply to a single pattern (-p), not to -batch" << std::endl;
    ok = false;
  }
  if (!ok) {
    std::cerr << "Usage: " << argv[0] << " -p <pattern_path/> -g <graph_path/> [-e <edge_list>]"
              << " [-o <output_path>] [-scheduler CHBL] [-mode count|emit]"
              << " [-order reference|strong|learned] [-model <dir/>] [-batch <list>]"
              << " [-device N] [-tune <table>] [-m1 .. -m6 <matrix dir/>]" << std::endl;
    return EXIT_FAILURE;
  }
  std::cout << "\n=== SubIso Configuration ===\nPattern Graph: " << flags["p"]
            << "\nData Graph: " << flags["g"] << "\nEdge List: " << flags["e"]
            << "\nOutput Path: " << flags["o"] << "\nScheduler: " << flags["scheduler"]
            << "\n==========================\n" << std::endl;
  try {
    MatrixGraph system(Scheduler2Enum(flags["scheduler"]));
    const int order = kOrders.at(flags["order"]);
    const int device = std::atoi(flags["device"].c_str());
    if (!batch.empty()) {
      matrixgraph::BatchSubIso task(batch, flags["g"], flags["o"], order, flags["model"],
                                    device, flags["tune"]);
      system.Run(matrixgraph::kSubIso, &task);
    } else {
      SubIso task(flags["p"], flags["g"], flags["e"], flags["o"], flags["mode"], order, device,
                  flags["model"], matrix_paths);
      system.Run(matrixgraph::kSubIso, &task);
    }
  } catch (const std::exception& e) {
    std::cerr << "Error: " << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
