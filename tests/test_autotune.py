"""The autotuner's host logic on the CPU: bucket choice, the trial loop (a
fake device graph whose batch_count records the settings it was given and
times them by a fixed cost model), the table written and read back, tuned
batches grouped by bucket, and rows of other graphs kept on rewrite."""
import numpy as np

from matrixgraph_b200 import autotune as T


class Q:
    def __init__(self, n):
        self.n = n


class FakeGraph:
    def __init__(self, n=100, best=None):
        self.info = {"n": n, "m_out": 4 * n, "n_labels": 3, "max_degree": 9}
        self.calls = []
        self.best = best or {"lanes": 8, "probe_min": 16, "grab": 0}

    def batch_count(self, qs, **opts):
        self.calls.append(dict(opts))
        return np.array([q.n * 10 for q in qs], dtype=np.uint64)


def test_bucket_of():
    assert T.bucket_of(3) == (1, 3)
    assert T.bucket_of(4) == (4, 4)
    assert T.bucket_of(6) == (5, 6)
    assert T.bucket_of(12) == (7, 16)
    assert T.bucket_of(40) == T.BUCKETS[-1]


def test_tune_picks_the_fastest_setting(monkeypatch):
    g = FakeGraph()
    clock = {"t": 0.0}
    last = {}

    def fake_batch(qs, **opts):
        last.update(opts)
        g.calls.append(dict(opts))
        return np.array([q.n * 10 for q in qs], dtype=np.uint64)

    def perf():
        # every trial costs 1 s, except the preferred setting (0.1 s)
        clock["t"] += 0.05 if all(last.get(k) == v for k, v in g.best.items()) else 0.5
        return clock["t"]

    monkeypatch.setattr(g, "batch_count", fake_batch)
    monkeypatch.setattr(T.time, "perf_counter", perf)
    qs = [Q(3), Q(4), Q(4), Q(6)]
    best = T.tune(g, qs)
    assert set(best) == {(1, 3), (4, 4), (5, 6)}
    for b, (opts, t) in best.items():
        assert opts == g.best, b
    n_settings = np.prod([len(v) for v in T.CANDIDATES.values()])
    assert len(g.calls) == 3 * n_settings * 2  # warm-up + one timed run each


def test_tune_rejects_a_setting_that_changes_counts():
    g = FakeGraph()

    def bad(qs, **opts):
        return np.array([opts["lanes"]] * len(qs), dtype=np.uint64)

    g.batch_count = bad
    try:
        T.tune(g, [Q(3)])
    except AssertionError:
        return
    raise AssertionError("a count change went unnoticed")


def test_table_round_trip_and_other_graphs_kept(tmp_path):
    path = str(tmp_path / "tune.txt")
    a, b = FakeGraph(100), FakeGraph(200)
    T.save_table(path, a, {(1, 3): ({"lanes": 4, "probe_min": 1, "grab": 16}, 0.5)})
    T.save_table(path, b, {(4, 4): ({"lanes": 16, "probe_min": 256, "grab": 0}, 1.5)})
    T.save_table(path, a, {(5, 6): ({"lanes": 8, "probe_min": 16, "grab": 0}, 0.25)})
    assert T.load_table(path, a) == {(5, 6): {"lanes": 8, "probe_min": 16, "grab": 0}}
    assert T.load_table(path, b) == {(4, 4): {"lanes": 16, "probe_min": 256, "grab": 0}}
    lines = open(path).read().splitlines()
    assert lines[0].startswith("#")
    assert len(lines) == 3
    # the row layout subiso_exec -tune parses: signature k_lo k_hi lanes probe_min grab s
    sig, lo, hi, lanes, pm, grab, sec = lines[-1].split()
    assert sig == T.signature(a) == "n100.m400.L3.d9"
    assert (int(lo), int(hi), int(lanes), int(pm), int(grab)) == (5, 6, 8, 16, 0)
    assert float(sec) == 0.25


def test_tuned_batch_count_groups_by_bucket():
    g = FakeGraph()
    table = {(4, 4): {"lanes": 16, "probe_min": 1, "grab": 0}}
    qs = [Q(3), Q(4), Q(7), Q(4)]
    out = T.tuned_batch_count(g, qs, table)
    assert out.tolist() == [30, 40, 70, 40]
    assert {"lanes": 16, "probe_min": 1, "grab": 0} in g.calls
    assert {} in g.calls  # untuned buckets run with the defaults
    assert len(g.calls) == 3
