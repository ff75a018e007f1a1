"""Chooses the root samples of tests/golden/c5_samples.json (run on a GPU).

C5 counts are concentrated on hub roots, and most low-degree roots have no
match, so a root sample that the CPU oracle can count and that still holds
matches is hard to find blind.  This script counts single roots on the GPU
only to choose them: for each of the first 16 C5 queries it counts the roots
at 1,024 evenly spaced positions of the query's level-0 bucket, each under a
budget of 2^22 candidate elements, and writes the positions whose count is
between 1 and 10^6 (with their element totals) to
tests/golden/c5_roots.json (or OUT).  The expected values of the fixture
are then computed by the oracle on the CPU (make_c5_golden.py), never taken
from this scan.

    python tests/golden/scan_c5_roots.py [n_queries [OUT]]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import matrixgraph_b200 as mg  # noqa: E402
from matrixgraph_b200 import _lib as L  # noqa: E402
from matrixgraph_b200 import workloads as W  # noqa: E402


def main():
    nq = int(sys.argv[1]) if len(sys.argv) > 1 else 16
    path = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "c5_roots.json")
    t0 = time.time()
    g = W.c5_graph()
    dg = mg.DeviceGraph(g, 0)
    print(f"graph generated and uploaded in {time.time() - t0:.0f} s", flush=True)
    sizes = np.bincount(g.array("labels"), minlength=W.C5_LABELS)
    out = {"positions_per_query": 1024, "budget_elements": 1 << 22, "queries": []}
    for q, x in enumerate(W.c5_queries(g, nq)):
        nb = int(sizes[int(x.array("labels")[mg.plan_order(x)[0]])])
        found = []
        for j in range(1024):
            p = (nb * j) // 1024
            try:
                c, st = dg.count(x, stats=True, root_range=(p, p + 1), max_elements=1 << 22)
            except L.MGError as e:
                if e.code != L.MG_E_LIMIT:
                    raise
                continue
            if 1 <= c <= 10 ** 6:
                found.append({"pos": p, "count": int(c), "elements": int(st["elements"])})
        out["queries"].append({"q": q, "bucket": nb, "roots": found})
        print(f"q {q}: bucket {nb}, {len(found)} roots with 1..10^6 matches", flush=True)
    dg.free()
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
