"""Seeded synthetic inputs: determinism, thread independence, shapes."""
import numpy as np

import matrixgraph_b200 as mg


def test_chung_lu_config1_shape():
    g = mg.chung_lu()  # n = 10,000, beta 2.5, mean degree 10, seed 0
    assert g.n == 10000
    assert 90_000 < g.m_out < 110_000  # ~50k undirected edges
    off, adj = g.array("out_off"), g.array("out_edges")
    for v in range(0, g.n, 97):
        lst = adj[off[v]:off[v + 1]]
        assert np.all(np.diff(lst.astype(np.int64)) > 0)  # sorted, no repeats
        assert v not in lst  # no self-loops
    assert np.array_equal(g.array("in_edges"), g.array("out_edges"))


def test_chung_lu_thread_independent():
    a = mg.chung_lu(3000, threads=1)
    b = mg.chung_lu(3000, threads=7)
    assert np.array_equal(a.array("out_edges"), b.array("out_edges"))


def test_rmat_deterministic_and_symmetric():
    a = mg.rmat(12, threads=1)
    b = mg.rmat(12, threads=5)
    assert np.array_equal(a.array("out_edges"), b.array("out_edges"))
    assert a.n == 4096
    c = mg.rmat(12, seed=1)
    assert not np.array_equal(a.array("out_edges"), c.array("out_edges"))
    # skew: R-MAT with a=0.57 concentrates edges on low ids
    deg = np.diff(a.array("out_off").astype(np.int64))
    assert deg[:64].mean() > 5 * deg[-1024:].mean()


def test_zipf_labels():
    lab = mg.gen_labels(200_000, 32, "zipf", 1.0, seed=1)
    freq = np.bincount(lab, minlength=32) / len(lab)
    h = sum(1.0 / (k + 1) for k in range(32))
    assert abs(freq[0] - 1.0 / h) < 0.01
    assert abs(freq[1] - 0.5 / h) < 0.01
    uni = mg.gen_labels(100_000, 8, "uniform", seed=1)
    assert np.all(np.abs(np.bincount(uni, minlength=8) / 1e5 - 0.125) < 0.01)


def test_query_generators():
    g = mg.chung_lu(2000, n_labels=8)
    lab = g.array("labels")
    for s in range(20):
        q = mg.query_random(g, 3 + s % 6, 0.3, seed=1000 + s)
        assert q.n == 3 + s % 6
        assert set(q.array("labels").tolist()) <= set(lab.tolist())
        # connected: a BFS from 0 over the symmetric query reaches everyone
        e = mg.query_edges(q)
        seen, front = {0}, [0]
        while front:
            u = front.pop()
            for a, b in e:
                if a == u and b not in seen:
                    seen.add(b)
                    front.append(b)
        assert len(seen) == q.n
    q1 = mg.query_walk(g, "4-cycle", seed=2)
    q2 = mg.query_walk(g, "4-cycle", seed=2)
    assert q1.array("labels").tolist() == q2.array("labels").tolist()
