"""Generates the committed golden fixtures under tests/golden/.

Run from the repository root in a container where the reference project is
checked out (read here, never at test time), given as the argument or as
MG_REFERENCE_DIR:

    python tests/golden/make_golden.py <reference checkout>

Fixtures:
  toy_graph/            the reference's only data fixture
                        (data/toy_graph/test_graph.csv, 16 vertices, 25 directed
                        edges with self-loops) as a CSR directory written by
                        this project's converter (first-appearance id
                        compaction, labels vid % 1, duplicates and self-loops
                        kept, as tools/graph_converter does);
  docs_example/         the 5-vertex labelled example graph printed in
                        docs/tools/GenerateRandomGraph.md (undirected,
                        symmetrised);
  expected.json         for both graphs: the exact CSR arrays computed here by
                        an independent numpy restatement of the layout
                        (immutable_csr.cu:103-166), and brute-force match
                        counts (enumeration of all injective maps, no pruning)
                        for a set of small queries under several labellings.
"""
from __future__ import annotations

import itertools
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# The reference checkout to read fixtures from: first argument or
# MG_REFERENCE_DIR (required; there is no default location).
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MG_REFERENCE_DIR", "")
if __name__ == "__main__" and not os.path.isdir(os.path.join(REF, "core")):
    sys.exit("usage: make_golden.py <reference checkout> (or set MG_REFERENCE_DIR)")
sys.path.insert(0, ROOT)


def read_toy_csv():
    pairs = []
    with open(os.path.join(REF, "data/toy_graph/test_graph.csv")) as f:
        for line in f:
            line = line.strip()
            if line:
                a, b = line.split(",")
                pairs.append((int(a), int(b)))
    return pairs


def read_docs_example():
    text = open(os.path.join(REF, "docs/tools/GenerateRandomGraph.md")).read()
    block = text.split("```")[1]  # first fenced block holds the example
    labels, edges = {}, []
    for line in block.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            labels[int(t[1])] = int(t[2])
        elif t[0] == "e":
            edges.append((int(t[1]), int(t[2])))
    n = max(labels) + 1
    return n, [labels[i] for i in range(n)], edges


def csr_arrays(n, pairs):
    """Independent restatement of the CSR layout: sorted lists, duplicates kept."""
    out = [[] for _ in range(n)]
    inn = [[] for _ in range(n)]
    for a, b in pairs:
        out[a].append(b)
        inn[b].append(a)
    out = [sorted(x) for x in out]
    inn = [sorted(x) for x in inn]
    out_off = np.cumsum([0] + [len(x) for x in out]).tolist()
    in_off = np.cumsum([0] + [len(x) for x in inn]).tolist()
    return {"globalid": list(range(n)), "indeg": [len(x) for x in inn],
            "outdeg": [len(x) for x in out], "in_off": in_off, "out_off": out_off,
            "in_edges": [v for x in inn for v in x], "out_edges": [v for x in out for v in x]}


def brute_count(n, edges, labels, k, qedges, qlabels):
    eset = set(edges)
    cands = [[v for v in range(n) if labels[v] == qlabels[u]] for u in range(k)]
    c = 0
    for f in itertools.product(*cands):
        if len(set(f)) != k:
            continue
        if all((f[a], f[b]) in eset for a, b in qedges):
            c += 1
    return c


QUERIES = {
    "edge": (2, [(0, 1)]),
    "wedge": (3, [(0, 1), (1, 2)]),
    "triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "4-cycle": (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
    "4-path": (4, [(0, 1), (1, 2), (2, 3)]),
    "star3": (4, [(0, 1), (0, 2), (0, 3)]),
    "tailed-triangle": (4, [(0, 1), (1, 2), (2, 0), (2, 3)]),
    "self-loop": (1, [(0, 0)]),
    "loop-edge": (2, [(0, 0), (0, 1)]),
}


def main():
    import matrixgraph_b200 as mg

    exp = {}
    # -- toy graph: directed, duplicates / self-loops kept ---------------------
    pairs = read_toy_csv()
    ids = []
    for a, b in pairs:
        for x in (a, b):
            if x not in ids:
                ids.append(x)
    remap = {x: i for i, x in enumerate(ids)}
    cp = [(remap[a], remap[b]) for a, b in pairs]
    n = len(ids)
    g = mg.CSRGraph.from_csv(os.path.join(REF, "data/toy_graph/test_graph.csv"), 1)
    g.Write(os.path.join(HERE, "toy_graph") + "/")
    toy = {"n": n, "pairs": cp, "arrays": csr_arrays(n, cp), "labelings": {}}
    labelings = {"all0": [0] * n, "mod2": [v % 2 for v in range(n)],
                 "mod3": [v % 3 for v in range(n)]}
    for name, lab in labelings.items():
        res = {}
        for qn, (k, qe) in QUERIES.items():
            for ql in sorted(set(itertools.product(sorted(set(lab)), repeat=k)))[:6]:
                key = f"{qn}|{','.join(map(str, ql))}|directed"
                res[key] = brute_count(n, cp, lab, k, qe, list(ql))
                und = [(a, b) for a, b in qe] + [(b, a) for a, b in qe if a != b]
                key = f"{qn}|{','.join(map(str, ql))}|symmetric"
                res[key] = brute_count(n, cp, lab, k, und, list(ql))
        toy["labelings"][name] = {"labels": lab, "counts": res}
    exp["toy_graph"] = toy
    # -- docs example: undirected labelled 5-vertex graph ------------------------
    n5, lab5, e5 = read_docs_example()
    sym = e5 + [(b, a) for a, b in e5]
    src = [a for a, _ in e5]
    dst = [b for _, b in e5]
    g5 = mg.CSRGraph.from_edges(n5, src, dst, lab5, symmetrize=True)
    g5.Write(os.path.join(HERE, "docs_example") + "/")
    d5 = {"n": n5, "labels": lab5, "edges": e5, "arrays": csr_arrays(n5, sym), "counts": {}}
    for qn, (k, qe) in QUERIES.items():
        if any(a == b for a, b in qe):
            continue
        und = [(a, b) for a, b in qe] + [(b, a) for a, b in qe]
        for ql in itertools.product(sorted(set(lab5)), repeat=k):
            key = f"{qn}|{','.join(map(str, ql))}|symmetric"
            d5["counts"][key] = brute_count(n5, sym, lab5, k, und, list(ql))
    # the docs graph matched against itself (as a query pattern)
    und5 = sym
    d5["self_match"] = brute_count(n5, sym, lab5, n5, und5, lab5)
    exp["docs_example"] = d5
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(exp, f, indent=0, sort_keys=True)
    print("wrote", os.path.join(HERE, "expected.json"))


if __name__ == "__main__":
    main()
