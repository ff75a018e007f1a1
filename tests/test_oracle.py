"""The oracle pinned against closed forms, brute force and the golden fixtures."""
import itertools
import json
import math
import os

import numpy as np
import pytest

import matrixgraph_b200 as mg
import oracle as O
from helpers import (bipartite, brute_count, brute_rows, complete, cycle, graph, oracle_count,
                     oracle_rows, random_graph, random_query, star, undirected)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def q(k, edges, labels=None, directed=False):
    return mg.CSRGraph.query(k, edges, labels if labels is not None else [0] * k, directed)


TRI = [(0, 1), (1, 2), (2, 0)]
C4 = [(0, 1), (1, 2), (2, 3), (3, 0)]
K4 = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def path(k):
    return [(i, i + 1) for i in range(k - 1)]


def falling(n, k):
    return math.perm(n, k)


@pytest.mark.parametrize("n", [3, 4, 5, 7, 9])
def test_complete_graph_closed_forms(n):
    g = complete(n)
    assert oracle_count(g, q(3, TRI))["count"] == falling(n, 3)
    if n >= 4:
        assert oracle_count(g, q(4, C4))["count"] == falling(n, 4)
        assert oracle_count(g, q(4, K4))["count"] == falling(n, 4)
    for k in range(1, min(n, 6) + 1):
        assert oracle_count(g, q(k, path(k)))["count"] == falling(n, k)


@pytest.mark.parametrize("n", [4, 5, 6, 9])
def test_cycle_graph_closed_forms(n):
    g = cycle(n)
    assert oracle_count(g, q(3, TRI))["count"] == 0
    assert oracle_count(g, q(4, C4))["count"] == (8 if n == 4 else 0)
    for k in range(2, n):
        assert oracle_count(g, q(k, path(k)))["count"] == 2 * n


@pytest.mark.parametrize("d", [1, 2, 5, 8])
def test_star_closed_forms(d):
    g = star(d)
    assert oracle_count(g, q(2, [(0, 1)]))["count"] == 2 * d
    assert oracle_count(g, q(3, [(0, 1), (1, 2)]))["count"] == d * (d - 1)
    assert oracle_count(g, q(3, TRI))["count"] == 0


@pytest.mark.parametrize("a,b", [(2, 3), (3, 3), (4, 2)])
def test_bipartite_labelled_closed_forms(a, b):
    g = bipartite(a, b)
    assert oracle_count(g, q(2, [(0, 1)], [0, 1]))["count"] == a * b
    assert oracle_count(g, q(2, [(0, 1)], [0, 0]))["count"] == 0
    assert oracle_count(g, q(4, C4, [0, 1, 0, 1]))["count"] == a * (a - 1) * b * (b - 1)
    assert oracle_count(g, q(3, TRI, [0, 1, 0]))["count"] == 0


def test_partitioned_labels_complete():
    n0, n1 = 4, 3
    g = complete(n0 + n1, [0] * n0 + [1] * n1)
    assert oracle_count(g, q(3, TRI, [0, 0, 1]))["count"] == n0 * (n0 - 1) * n1
    assert oracle_count(g, q(3, TRI, [1, 1, 1]))["count"] == falling(n1, 3)
    assert oracle_count(g, q(3, TRI, [2, 0, 0]))["count"] == 0  # absent label


@pytest.mark.parametrize("seed", range(12))
def test_bruteforce_undirected(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(6, 12))
    edges, labels = random_graph(rng, n, 0.45, int(rng.integers(1, 4)))
    g = graph(n, edges, labels)
    k = int(rng.integers(2, 6))
    qe, ql = random_query(rng, k, 0.4, max(labels) + 1)
    qq = q(k, qe, ql)
    want = brute_count(n, undirected(edges), labels, k, undirected(qe), ql)
    got = oracle_count(g, qq)
    assert got["count"] == want
    assert got["level_rows"][k] == want
    rows = oracle_rows(g, qq)
    assert np.array_equal(rows, brute_rows(n, undirected(edges), labels, k, undirected(qe), ql))


@pytest.mark.parametrize("seed", range(8))
def test_bruteforce_directed_with_self_loops(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(6, 11))
    edges, labels = random_graph(rng, n, 0.35, 2, directed=True, self_loops=True)
    g = graph(n, edges, labels, symmetric=False)
    k = int(rng.integers(2, 5))
    qe, ql = random_query(rng, k, 0.3, 2, directed=True)
    if seed % 3 == 0:
        qe = qe + [(0, 0)]
    qq = q(k, qe, ql, directed=True)
    want = brute_count(n, edges, labels, k, qe, ql)
    assert oracle_count(g, qq)["count"] == want


@pytest.mark.parametrize("seed", range(6))
def test_order_and_filter_invariance(seed):
    rng = np.random.default_rng(200 + seed)
    n = 11
    edges, labels = random_graph(rng, n, 0.5, 2)
    g = graph(n, edges, labels)
    k = 4
    qe, ql = random_query(rng, k, 0.5, 2)
    qq = q(k, qe, ql)
    base = oracle_count(g, qq)["count"]
    for perm in itertools.permutations(range(k)):
        for f in (0, 1, 2, 3):
            assert oracle_count(g, qq, order=perm, filters=f)["count"] == base


def test_relabelling_invariance():
    rng = np.random.default_rng(7)
    n = 12
    edges, labels = random_graph(rng, n, 0.4, 3)
    perm = rng.permutation(n)
    g1 = graph(n, edges, labels)
    g2 = graph(n, [(int(perm[a]), int(perm[b])) for a, b in edges],
               [labels[int(np.argsort(perm)[v])] for v in range(n)])
    qq = q(4, C4, [0, 1, 0, 2])
    assert oracle_count(g1, qq)["count"] == oracle_count(g2, qq)["count"]


def test_threads_and_root_ranges_sum():
    g = mg.chung_lu(2000, avg_deg=8, n_labels=4)
    qq = q(4, C4, [0, 1, 0, 1])
    full = oracle_count(g, qq, threads=4)
    one = oracle_count(g, qq, threads=1)
    assert full == one
    nb = O.bucket_size(O.Graph.from_csr(g), O.query_from_csr(qq), full["order"])
    parts = [oracle_count(g, qq, root_range=(a, b))["count"]
             for a, b in [(0, nb // 3), (nb // 3, 2 * nb // 3), (2 * nb // 3, nb)]]
    assert sum(parts) == full["count"]


def test_reference_order_restatement_matches_library():
    rng = np.random.default_rng(3)
    for _ in range(40):
        k = int(rng.integers(2, 9))
        qe, ql = random_query(rng, k, 0.3, 3, directed=bool(rng.integers(0, 2)))
        qq = q(k, qe, ql, directed=True)
        assert mg.plan_order(qq) == O.reference_order(O.query_from_csr(qq))


def _golden():
    with open(os.path.join(GOLDEN, "expected.json")) as f:
        return json.load(f)


QUERIES = {
    "edge": (2, [(0, 1)]), "wedge": (3, [(0, 1), (1, 2)]), "triangle": (3, TRI),
    "4-cycle": (4, C4), "4-path": (4, path(4)), "star3": (4, [(0, 1), (0, 2), (0, 3)]),
    "tailed-triangle": (4, [(0, 1), (1, 2), (2, 0), (2, 3)]), "self-loop": (1, [(0, 0)]),
    "loop-edge": (2, [(0, 0), (0, 1)]),
}


def golden_cases():
    exp = _golden()
    out = []
    for lname, d in exp["toy_graph"]["labelings"].items():
        for key, want in d["counts"].items():
            out.append(("toy_graph", lname, key, want))
    for key, want in exp["docs_example"]["counts"].items():
        out.append(("docs_example", None, key, want))
    return out


def golden_graph(name, labeling):
    exp = _golden()
    g = mg.CSRGraph.Read(os.path.join(GOLDEN, name) + "/")
    if labeling is None:
        return g
    d = exp[name]
    lab = d["labelings"][labeling]["labels"]
    a = {k: g.array(k) for k in ("out_off", "out_edges")}
    src = [u for u in range(g.n) for _ in range(a["out_off"][u], a["out_off"][u + 1])]
    return mg.CSRGraph.from_edges(g.n, src, a["out_edges"], lab)


def golden_query(key):
    qn, labs, mode = key.split("|")
    k, qe = QUERIES[qn]
    ql = [int(x) for x in labs.split(",")]
    if mode == "symmetric":
        return q(k, qe, ql, directed=False)
    return q(k, qe, ql, directed=True)


def test_golden_counts_oracle():
    cache = {}
    for name, lname, key, want in golden_cases():
        if (name, lname) not in cache:
            cache[(name, lname)] = golden_graph(name, lname)
        g = cache[(name, lname)]
        assert oracle_count(g, golden_query(key))["count"] == want, (name, lname, key)


def test_golden_docs_self_match():
    exp = _golden()["docs_example"]
    g = mg.CSRGraph.Read(os.path.join(GOLDEN, "docs_example") + "/")
    qq = q(exp["n"], exp["edges"], exp["labels"])
    assert oracle_count(g, qq)["count"] == exp["self_match"]


def test_oracle_reader_matches_library_reader():
    for name in ("toy_graph", "docs_example"):
        path_ = os.path.join(GOLDEN, name) + "/"
        a = O.Graph.read_dir(path_).info()
        b = O.Graph.from_csr(mg.CSRGraph.Read(path_)).info()
        assert a == b
