"""The checker-side generators (oracle/gen.c) reproduce the product
generators bit for bit: R-MAT CSR, uniform and Zipf labels, random-walk query
labels and random connected query shapes.  The bench's reference arm builds
its workload with them, so this is what makes the two arms' inputs equal."""
import numpy as np
import pytest

import matrixgraph_b200 as mg
import oracle as O


@pytest.mark.parametrize("scale,labels", [(10, 4), (16, 32)])
def test_rmat_csr_and_labels_match_the_product(scale, labels):
    g = mg.rmat(scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=labels, label_kind="zipf",
                zipf_s=1.0, label_seed=1)
    p = O.rmat(scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=labels, label_kind="zipf",
               zipf_s=1.0, label_seed=1, threads=3)
    assert np.array_equal(g.array("out_off"), p.off)
    assert np.array_equal(g.array("out_edges"), p.adj)
    assert np.array_equal(g.array("labels"), p.labels)
    for i, s in enumerate(mg.SHAPES):
        k, e = mg.SHAPES[s]
        q = mg.query_walk(g, s, seed=2 + i)
        assert q.array("labels").tolist() == O.walk_labels(p, k, e, 2 + i), s


def test_other_parameters_and_uniform_labels():
    g = mg.rmat(11, 4, 0.45, 0.15, 0.15, seed=7, n_labels=8, label_kind="uniform", label_seed=3)
    p = O.rmat(11, 4, 0.45, 0.15, 0.15, seed=7, n_labels=8, label_kind="uniform", label_seed=3)
    assert np.array_equal(g.array("out_edges"), p.adj)
    assert np.array_equal(g.array("labels"), p.labels)
    assert np.array_equal(mg.gen_labels(1000, 64, "zipf", 1.2, seed=5),
                          O.gen_labels(1000, 64, "zipf", 1.2, seed=5))


def test_random_query_shapes_match_the_product():
    g = mg.rmat(12, n_labels=8)
    p = O.rmat(12, n_labels=8)
    for seed in range(1000, 1012):
        k = 3 + seed % 6
        q = mg.query_random(g, k, 0.3, seed=seed)
        e = O.random_query_edges(k, 0.3, seed)
        und = sorted({(min(u, w), max(u, w)) for u, w in mg.query_edges(q)})
        assert und == e, seed
        assert q.array("labels").tolist() == O.walk_labels(p, k, e, seed ^ 0x9E3779B97F4A7C15)
