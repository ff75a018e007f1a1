// subiso_exec: the reference's subiso CLI (apps/subiso.cu:16-97) over the
// C-ABI.  Flags: -p <pattern dir/> -g <graph dir/> [-e <edge list, unused>]
// [-o <output>] [-scheduler CHBL|EvenSplit|RoundRobin] plus
// [-mode count|emit] [-order reference|strong] [-device N].
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <string>

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
      {"mode", "count"}, {"order", "reference"}, {"device", "0"}};
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
  if (flags["p"].empty()) {
    std::cerr << "Error: Pattern graph path (-p) is required" << std::endl;
    ok = false;
  }
  if (flags["g"].empty()) {
    std::cerr << "Error: Data graph path (-g) is required" << std::endl;
    ok = false;
  }
  if (!ok) {
    std::cerr << "Usage: " << argv[0] << " -p <pattern_path/> -g <graph_path/> [-e <edge_list>]"
              << " [-o <output_path>] [-scheduler CHBL] [-mode count|emit]"
              << " [-order reference|strong] [-device N]" << std::endl;
    return EXIT_FAILURE;
  }
  std::cout << "\n=== SubIso Configuration ===\nPattern Graph: " << flags["p"]
            << "\nData Graph: " << flags["g"] << "\nEdge List: " << flags["e"]
            << "\nOutput Path: " << flags["o"] << "\nScheduler: " << flags["scheduler"]
            << "\n==========================\n" << std::endl;
  try {
    MatrixGraph system(Scheduler2Enum(flags["scheduler"]));
    int order = flags["order"] == "strong" ? MG_ORDER_STRONG : MG_ORDER_REFERENCE;
    SubIso task(flags["p"], flags["g"], flags["e"], flags["o"], flags["mode"], order,
                std::atoi(flags["device"].c_str()));
    system.Run(matrixgraph::kSubIso, &task);
  } catch (const std::exception& e) {
    std::cerr << "Error: " << e.what() << std::endl;
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}
