"""Seeded GAR match instances shared by the oracle and library tests."""
from __future__ import annotations

import itertools

import numpy as np

from oracle.gar import GarGraph, GarPattern


def random_graph(rng, n, m, v_labels, e_labels, self_loops=0.05, id_base=1000,
                 with_ids=True, with_elabels=True):
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    loop = rng.random(m) < self_loops
    dst[loop] = src[loop]
    # instance ids: distinct, not in local order
    ids = (id_base + rng.permutation(n) * 7).astype(np.uint32) if with_ids else None
    vl = rng.integers(0, v_labels, n).astype(np.int32)
    el = rng.integers(0, e_labels, m).astype(np.int32) if with_elabels else None
    return GarGraph(v_id=None if ids is None else ids.tolist(), v_label=vl.tolist(),
                    e_src=src.tolist(), e_dst=dst.tolist(),
                    e_label=None if el is None else el.tolist(), n_vertices=n)


def random_pattern(rng, k, extra, v_labels, e_labels, self_loop=False, with_elabels=True):
    """Connected-ish random pattern: a random spanning tree in random
    directions plus `extra` random edges (possibly parallel)."""
    es, ed = [], []
    for j in range(1, k):
        a, b = int(rng.integers(0, j)), j
        if rng.random() < 0.5:
            a, b = b, a
        es.append(a)
        ed.append(b)
    for _ in range(extra):
        a, b = int(rng.integers(0, k)), int(rng.integers(0, k))
        if a == b and not self_loop:
            continue
        es.append(a)
        ed.append(b)
    if k == 1 or self_loop:
        u = int(rng.integers(0, k))
        es.append(u)
        ed.append(u)
    labels = rng.integers(0, v_labels, k).astype(np.int32).tolist()
    el = rng.integers(0, e_labels, len(es)).astype(np.int32).tolist() if with_elabels else None
    return GarPattern(node_label=labels, edge_src=es, edge_dst=ed, edge_label=el, n_nodes=k)


def brute_force(g: GarGraph, p: GarPattern):
    """All injective node maps by itertools (tiny graphs only)."""
    has = set()
    for i in range(len(g.e_src)):
        s, d = g.e_src[i], g.e_dst[i]
        if s < g.n_vertices and d < g.n_vertices:
            has.add((s, d, None if g.e_label is None else g.e_label[i]))
    out = []
    for f in itertools.permutations(range(g.n_vertices), p.n_nodes):
        if any(g.v_label[f[u]] != p.node_label[u] for u in range(p.n_nodes)):
            continue
        ok = True
        for j in range(len(p.edge_src)):
            lab = None if g.e_label is None else (
                p.edge_label[j] if p.edge_label is not None else 0)
            if (f[p.edge_src[j]], f[p.edge_dst[j]], lab) not in has:
                ok = False
                break
        if ok:
            out.append(f)
    return out


def doc_example():
    """The example of core/data_structures/gar_match_arrays.h:33-51: pivots
    126 and 138, pattern position 1 matched by {183, 115407} and {192}."""
    ids = [126, 138, 183, 115407, 192]
    g = GarGraph(v_id=ids, v_label=[0, 0, 1, 1, 1], e_src=[0, 0, 1], e_dst=[2, 3, 4],
                 e_label=[5, 5, 5], n_vertices=5)
    p = GarPattern(node_label=[0, 1], edge_src=[0], edge_dst=[1], edge_label=[5], n_nodes=2)
    expected = dict(num_conditions=2, row_pivot_id=[126, 126, 138, 138],
                    row_cond_j=[0, 1, 0, 1], row_pos=[0, 1, 0, 1], row_offset=[0, 1, 3, 4],
                    row_count=[1, 2, 1, 1], matched_v_ids=[126, 183, 115407, 138, 192])
    return g, p, expected


def two_label_case(rng, n=14, m=90, v_labels=2, k=None, extra=None):
    """Dense small graph with two edge labels and a pattern whose first two
    edges carry different labels (the subdivided matching path)."""
    g = random_graph(rng, n, m, v_labels=v_labels, e_labels=2, self_loops=0.08)
    k = int(rng.integers(2, 5)) if k is None else k
    extra = int(rng.integers(1, 3)) if extra is None else extra
    p = random_pattern(rng, k, extra, v_labels=v_labels, e_labels=2)
    if len(p.edge_label) >= 2:
        p.edge_label[0], p.edge_label[1] = 0, 1
    return g, p
