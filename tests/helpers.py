"""Shared helpers: small graph families, brute-force enumeration, oracle glue."""
from __future__ import annotations

import itertools

import numpy as np

import matrixgraph_b200 as mg
import oracle as O


def undirected(edges):
    return [(a, b) for a, b in edges] + [(b, a) for a, b in edges if a != b]


def graph(n, edges, labels=None, symmetric=True):
    """CSRGraph over 0..n-1; `edges` undirected when symmetric."""
    lab = labels if labels is not None else [0] * n
    s = [a for a, _ in edges]
    d = [b for _, b in edges]
    return mg.CSRGraph.from_edges(n, s, d, lab, symmetrize=symmetric, dedup=True)


def complete(n, labels=None):
    return graph(n, [(i, j) for i in range(n) for j in range(i + 1, n)], labels)


def cycle(n, labels=None):
    return graph(n, [(i, (i + 1) % n) for i in range(n)], labels)


def star(d, labels=None):
    return graph(d + 1, [(0, i) for i in range(1, d + 1)], labels)


def bipartite(a, b):
    edges = [(i, a + j) for i in range(a) for j in range(b)]
    return graph(a + b, edges, [0] * a + [1] * b)


def random_graph(rng, n, p, n_labels, directed=False, self_loops=False):
    edges = []
    for i in range(n):
        for j in range(n):
            if i == j and not self_loops:
                continue
            if not directed and j <= i and i != j:
                continue
            if rng.random() < p:
                edges.append((i, j))
    labels = rng.integers(0, n_labels, n).tolist()
    return edges, labels


def random_query(rng, k, p_extra, n_labels, directed=False):
    edges = set()
    for j in range(1, k):
        p = int(rng.integers(0, j))
        edges.add((p, j) if rng.random() < 0.5 or not directed else (j, p))
    for i in range(k):
        for j in range(i + 1, k):
            if (i, j) not in edges and (j, i) not in edges and rng.random() < p_extra:
                edges.add((i, j) if rng.random() < 0.5 or not directed else (j, i))
    labels = rng.integers(0, n_labels, k).tolist()
    return sorted(edges), labels


def brute_count(n, dir_edges, labels, k, q_dir_edges, qlabels):
    """All injective label-preserving maps preserving every directed query edge."""
    eset = set(dir_edges)
    cands = [[v for v in range(n) if labels[v] == qlabels[u]] for u in range(k)]
    c = 0
    for f in itertools.product(*cands):
        if len(set(f)) != k:
            continue
        if all((f[a], f[b]) in eset for a, b in q_dir_edges):
            c += 1
    return c


def brute_rows(n, dir_edges, labels, k, q_dir_edges, qlabels):
    eset = set(dir_edges)
    cands = [[v for v in range(n) if labels[v] == qlabels[u]] for u in range(k)]
    rows = []
    for f in itertools.product(*cands):
        if len(set(f)) == k and all((f[a], f[b]) in eset for a, b in q_dir_edges):
            rows.append(f)
    return np.array(sorted(rows), dtype=np.uint32).reshape(-1, k)


def oracle_count(g, q, order=None, filters=3, threads=1, root_range=None):
    og = O.Graph.from_csr(g)
    oq = O.query_from_csr(q)
    return O.count(og, oq, order=order, filters=filters, threads=threads, root_range=root_range)


def oracle_rows(g, q, order=None):
    return O.emit(O.Graph.from_csr(g), O.query_from_csr(q), order=order)
