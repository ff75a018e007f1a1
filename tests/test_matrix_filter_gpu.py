"""The lossy MatrixFilter on the GPU against the restated reference filter
(oracle/matrix_filter.py) and the oracle: keep decisions, filtered counts
(the oracle's per-root counts summed over the kept roots), filtered emit
rows, the task mirror and subiso_exec -m1..-m6, and the entry points that
reject it."""
import os
import subprocess

import numpy as np
import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import _lib as L
from matrixgraph_b200.matrix_filter import MatrixFilter
from oracle import matrix_filter as OMF

import oracle as O
from test_matrix_filter import save, weights

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("mf")
    g = mg.chung_lu(600, avg_deg=6, n_labels=3)
    qs = [mg.query_random(g, 3 + i % 3, 0.4, seed=800 + i) for i in range(6)]
    rng = np.random.default_rng(9)
    mats = weights(rng, 8, g.n)
    dirs = save(tmp, mats)
    mf = MatrixFilter.load(dirs)
    dg = mg.DeviceGraph(g)
    yield g, qs, mats, dirs, mf, dg, tmp
    mf.free()
    dg.free()


def test_keep_matches_the_restated_filter(setup):
    g, qs, mats, dirs, mf, dg, _ = setup
    vs = np.arange(g.n, dtype=np.uint32)
    for u in range(8):
        got = mf.keep(u, vs).astype(bool)
        want, unsure = OMF.keep(*mats, u, vs)
        assert np.array_equal(got[~unsure], want[~unsure]), u
        assert 0.05 < got.mean() < 0.95


def _bucket(g, q, first):
    lab = g.array("labels")
    return np.flatnonzero(lab == q.array("labels")[first]).astype(np.uint32)


def test_filtered_counts_and_rows_equal_the_oracle(setup):
    g, qs, mats, dirs, mf, dg, _ = setup
    og = O.Graph.from_csr(g)
    some_dropped = False
    for q in qs:
        oq = O.query_from_csr(q)
        order = O.reference_order(oq)
        bucket = _bucket(g, q, order[0])
        keep = mf.keep(order[0], bucket).astype(bool)
        per_root = [O.count(og, oq, order=order, root_range=(p, p + 1))["count"]
                    for p in range(len(bucket))]
        want = sum(c for c, k in zip(per_root, keep) if k)
        full = dg.count(q)
        assert full == sum(per_root)
        got = dg.count(q, matrix_filter=mf)
        assert got == want, (q.n, got, want)
        some_dropped |= got < full
        rows = dg.emit(q, matrix_filter=mf)
        all_rows = O.emit(og, oq, order=order)
        kept_ids = set(bucket[keep].tolist())
        sel = np.array([r[order[0]] in kept_ids for r in all_rows], dtype=bool)
        want_rows = all_rows[sel] if len(all_rows) else all_rows
        assert np.array_equal(np.asarray(rows).reshape(-1, q.n), want_rows.reshape(-1, q.n))
    assert some_dropped


def test_entry_points_that_reject_the_filter(setup):
    g, qs, mats, dirs, mf, dg, _ = setup
    with pytest.raises(L.MGError) as e:
        dg.batch_count(qs[:2], matrix_filter=mf)
    assert e.value.code == L.MG_E_ARG
    from test_zz_no_alloc import count_noalloc
    with pytest.raises(L.MGError) as e:
        count_noalloc(dg, qs[0], matrix_filter=mf)
    assert e.value.code == L.MG_E_ARG


def test_task_mirror_and_cli(setup):
    g, qs, mats, dirs, mf, dg, tmp = setup
    q = qs[1]
    g.Write(str(tmp / "g") + "/")
    q.Write(str(tmp / "p") + "/")
    want = dg.count(q, matrix_filter=mf)
    task = mg.SubIso(str(tmp / "p") + "/", str(tmp / "g") + "/", "", "", matrix_paths=dirs)
    mg.MatrixGraph().Run(mg.TaskType.kSubIso, task)
    assert task.count == want
    exe = os.path.join(os.path.dirname(mg.__file__), "subiso_exec")
    args = [exe, "-p", str(tmp / "p") + "/", "-g", str(tmp / "g") + "/", "-o",
            str(tmp / "out.txt")]
    for i, d in enumerate(dirs):
        args += [f"-m{i + 1}", d]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert int((tmp / "out.txt").read_text().split()[0]) == want
