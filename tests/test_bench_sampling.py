"""The CPU baseline's bounded sampling (bench.py): attempts in forked
children under a hard time limit, prefix then suffix root ranges."""
import numpy as np
import pytest

import bench
import matrixgraph_b200 as mg
import oracle as O


@pytest.fixture(scope="module")
def case():
    g = mg.rmat(14, 16, 0.57, 0.19, 0.19, seed=0, n_labels=4, label_kind="zipf", zipf_s=1.0,
                label_seed=1)
    q = mg.query_walk(g, "4-cycle", seed=3)
    og, oq = O.Graph.from_csr(g), O.query_from_csr(q)
    order = O.reference_order(oq)
    return og, oq, order, O.bucket_size(og, oq, order)


def test_timed_count_matches_direct_count(case):
    og, oq, order, nb = case
    rr = (0, min(nb, 64))
    got = bench._timed_count(og, oq, order, 2, rr, 60.0)
    assert got is not None
    assert got[0] == O.count(og, oq, order=order, threads=2, root_range=rr)["count"]
    assert got[1] >= 0.0


def test_timed_count_gives_up_at_the_limit(case):
    og, oq, order, nb = case
    # a limit far below the time of the whole bucket: the child is killed
    assert bench._timed_count(og, oq, order, 1, (0, nb), 1e-4) is None
    # and the process has no child left behind
    with pytest.raises(ChildProcessError):
        import os
        os.waitpid(-1, os.WNOHANG)


def test_choose_sample_range_and_count(case):
    og, oq, order, nb = case
    s = bench.choose_sample(og, oq, order, nb, 0.5, 2)
    assert s is not None
    b, e, c, dt = s
    assert 0 <= b < e <= nb
    assert b == 0 or e == nb
    assert c == O.count(og, oq, order=order, threads=2, root_range=(b, e))["count"]
