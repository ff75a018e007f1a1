"""GPU parity: the CUDA path (through the C-ABI) against the oracle and brute force."""
import itertools
import os

import numpy as np
import pytest

import matrixgraph_b200 as mg
import oracle as O
from matrixgraph_b200 import _lib as L
from helpers import (brute_count, brute_rows, complete, graph, oracle_count, oracle_rows,
                     random_graph, random_query, undirected)
from test_oracle import GOLDEN, QUERIES, golden_cases, golden_graph, golden_query

pytestmark = pytest.mark.gpu

C4 = [(0, 1), (1, 2), (2, 3), (3, 0)]


@pytest.fixture(scope="module")
def c1():
    """Chung-Lu n=10,000, beta 2.5, mean degree 10, 8 uniform labels; 4-cycle query."""
    g = mg.chung_lu()
    q = mg.CSRGraph.query(4, C4, mg.gen_labels(4, 8, "uniform", seed=2))
    dg = mg.DeviceGraph(g)
    yield g, q, dg
    dg.free()


def test_c1_count_rows_and_stats(c1):
    g, q, dg = c1
    want = oracle_count(g, q, threads=4)
    got, st = dg.count(q, stats=True)
    assert got == want["count"] > 0
    assert st["level_rows"] == want["level_rows"]
    assert st["balg_bytes"] == want["balg"]
    assert st["balg_count_bytes"] == want["balg_count"]
    rows = dg.emit(q)
    assert np.array_equal(rows, oracle_rows(g, q))


def test_c1_all_orders_and_chunks(c1):
    g, q, dg = c1
    want = oracle_count(g, q)["count"]
    for perm in itertools.permutations(range(4)):
        for chunk in (0, 97):
            r = oracle_count(g, q, order=perm)
            c, st = dg.count(q, given_order=perm, chunk_rows=chunk, stats=True)
            assert c == want
            assert st["level_rows"] == r["level_rows"]
            assert st["balg_bytes"] == r["balg"]
    for f in (0, 1, 2):
        assert dg.count(q, filters=f) == want


def test_graph_info(c1):
    g, q, dg = c1
    info = dg.info
    assert info["n"] == 10000 and info["n_labels"] == 8 and info["symmetric"] == 1
    assert info["m_out"] == g.m_out


@pytest.mark.parametrize("seed", range(16))
def test_random_undirected(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 40))
    edges, labels = random_graph(rng, n, 0.3, int(rng.integers(1, 4)))
    g = graph(n, edges, labels)
    dg = mg.DeviceGraph(g)
    for _ in range(4):
        k = int(rng.integers(1, 7))
        qe, ql = random_query(rng, k, 0.35, max(labels) + 1)
        q = mg.CSRGraph.query(k, qe, ql)
        want = oracle_count(g, q)
        c, st = dg.count(q, stats=True, chunk_rows=int(rng.choice([0, 1, 5, 64])))
        assert c == want["count"]
        assert st["level_rows"] == want["level_rows"]
        if n <= 14 and k <= 5:
            assert c == brute_count(n, undirected(edges), labels, k, undirected(qe), ql)
        rows = dg.emit(q)
        assert np.array_equal(rows, oracle_rows(g, q))
    dg.free()


@pytest.mark.parametrize("seed", range(8))
def test_random_directed_self_loops(seed):
    rng = np.random.default_rng(500 + seed)
    n = int(rng.integers(6, 24))
    edges, labels = random_graph(rng, n, 0.3, 2, directed=True, self_loops=True)
    g = graph(n, edges, labels, symmetric=False)
    dg = mg.DeviceGraph(g)
    assert dg.info["symmetric"] == 0
    for t in range(4):
        k = int(rng.integers(1, 5))
        qe, ql = random_query(rng, k, 0.3, 2, directed=True)
        if t % 2:
            qe = qe + [(k - 1, k - 1)]
        q = mg.CSRGraph.query(k, qe, ql, directed=True)
        want = oracle_count(g, q)
        c, st = dg.count(q, stats=True)
        assert c == want["count"]
        assert st["balg_bytes"] == want["balg"]
        if n <= 12:
            assert c == brute_count(n, edges, labels, k, qe, ql)
        assert np.array_equal(dg.emit(q), oracle_rows(g, q))
    dg.free()


def test_golden_counts_gpu():
    cache = {}
    for name, lname, key, want in golden_cases():
        if (name, lname) not in cache:
            cache[(name, lname)] = (golden_graph(name, lname), None)
            cache[(name, lname)] = (cache[(name, lname)][0],
                                    mg.DeviceGraph(cache[(name, lname)][0]))
        g, dg = cache[(name, lname)]
        assert dg.count(golden_query(key)) == want, (name, lname, key)
    for g, dg in cache.values():
        dg.free()


def test_edge_cases():
    g = complete(6, [0, 0, 0, 1, 1, 1])
    dg = mg.DeviceGraph(g)
    # absent label, single vertex, query larger than the graph, disconnected query
    assert dg.count(mg.CSRGraph.query(3, [(0, 1), (1, 2)], [0, 7, 0])) == 0
    assert dg.count(mg.CSRGraph.query(1, [], [1])) == 3
    assert dg.count(mg.CSRGraph.query(7, [(i, i + 1) for i in range(6)], [0] * 7)) == 0
    qd = mg.CSRGraph.query(4, [(0, 1), (2, 3)], [0, 0, 1, 1])
    assert dg.count(qd) == oracle_count(g, qd)["count"] == 6 * 6
    assert np.array_equal(dg.emit(qd), oracle_rows(g, qd))
    assert dg.emit(mg.CSRGraph.query(3, [(0, 1), (1, 2)], [0, 7, 0])).shape == (0, 3)
    dg.free()


def test_emit_capacity():
    g = complete(7)
    dg = mg.DeviceGraph(g)
    q = mg.CSRGraph.query(3, [(0, 1), (1, 2), (2, 0)], [0, 0, 0])
    full = dg.emit(q)
    assert full.shape == (210, 3)
    part, n, _ = dg.emit(q, cap=50, stats=True)
    assert n == 210 and np.array_equal(part, full[:50])
    dg.free()


def test_batch_equals_single(c1):
    g, q, dg = c1
    qs = [mg.query_random(g, 3 + i % 6, 0.3, seed=1000 + i) for i in range(64)]
    single = [dg.count(x) for x in qs]
    assert dg.batch_count(qs).tolist() == single
    assert dg.batch_count(qs, chunk_rows=4096).tolist() == single
    for x, c in list(zip(qs, single))[:12]:
        assert oracle_count(g, x)["count"] == c


def test_root_ranges_sum(c1):
    g, q, dg = c1
    full = dg.count(q)
    nb = O.bucket_size(O.Graph.from_csr(g), O.query_from_csr(q), mg.plan_order(q))
    parts = [mg.shard_roots(nb, r, 3) for r in range(3)]
    got = [dg.count(q, root_range=p) for p in parts]
    assert sum(got) == full
    assert got[1] == oracle_count(g, q, root_range=parts[1])["count"]


def test_subiso_task_and_runtime(tmp_path, c1):
    g, q, dg = c1
    g.Write(str(tmp_path / "g") + "/")
    q.Write(str(tmp_path / "p") + "/")
    task = mg.SubIso(str(tmp_path / "p") + "/", str(tmp_path / "g") + "/", "",
                     str(tmp_path / "out.txt"), mode="emit")
    mg.MatrixGraph().Run(mg.TaskType.kSubIso, task)
    assert task.count == dg.count(q)
    lines = open(tmp_path / "out.txt").read().split()
    assert int(lines[0]) == task.count and len(lines) == task.count + 1


def test_rmat_small_full_parity():
    g = mg.rmat(13, n_labels=8, label_kind="zipf")
    dg = mg.DeviceGraph(g)
    og = O.Graph.from_csr(g)
    for i, shape in enumerate(mg.SHAPES):
        q = mg.query_walk(g, shape, seed=2 + i)
        want = O.count(og, O.query_from_csr(q), threads=8)
        for tail in (0, 1, 2):
            c, st = dg.count(q, stats=True, no_tail=tail)
            assert c == want["count"], (shape, tail)
            assert st["level_rows"] == want["level_rows"], (shape, tail)
            assert st["balg_count_bytes"] == want["balg_count"], (shape, tail)
            assert st["balg_bytes"] == want["balg"], (shape, tail)
        assert dg.count(q, order="strong") == want["count"]
    dg.free()


TAIL_QUERIES = [
    (3, [(0, 1), (1, 2)]),                          # wedge
    (4, [(0, 1), (1, 2), (2, 3)]),                  # 4-path
    (5, [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4)]),  # triangle with a 2-tail
    (5, [(0, 1), (0, 2), (0, 3), (3, 4)]),          # star with a 2-tail
    (6, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (4, 5)]),
]


@pytest.mark.parametrize("seed", range(10))
def test_tail_closed_form(seed):
    """Closed-form pendant tails equal enumeration, incl. label collisions and
    directed graphs with self-loops."""
    rng = np.random.default_rng(900 + seed)
    directed = seed % 2 == 1
    n = int(rng.integers(10, 40))
    edges, labels = random_graph(rng, n, 0.25, int(rng.integers(1, 3)), directed=directed,
                                 self_loops=directed)
    g = graph(n, edges, labels, symmetric=not directed)
    dg = mg.DeviceGraph(g)
    for k, qe in TAIL_QUERIES:
        ql = rng.integers(0, max(labels) + 1, k).tolist()
        if directed:
            qe = [(b, a) if rng.random() < 0.5 else (a, b) for a, b in qe]
        q = mg.CSRGraph.query(k, qe, ql, directed=directed)
        want = oracle_count(g, q)
        for tail in (1, 2):
            c, st = dg.count(q, stats=True, no_tail=tail)
            assert c == want["count"], (k, qe, ql, tail)
            assert st["level_rows"] == want["level_rows"], (k, qe, ql, tail)
            assert st["balg_bytes"] == want["balg"], (k, qe, ql, tail)
            assert st["balg_count_bytes"] == want["balg_count"], (k, qe, ql, tail)
    dg.free()


# (k, undirected edges, an order ending in two leaves of one anchor)
STAR_QUERIES = [
    (3, [(0, 1), (0, 2)], [0, 1, 2]),                       # wedge, center first
    (4, [(0, 1), (0, 2), (0, 3)], [0, 3, 1, 2]),            # 3-star
    (4, [(0, 1), (1, 2), (1, 3)], [0, 1, 2, 3]),            # leaves of a non-first anchor
    (5, [(0, 1), (1, 2), (2, 0), (0, 3), (0, 4)], [1, 2, 0, 3, 4]),  # triangle + two leaves
    (5, [(0, 1), (1, 2), (2, 3), (1, 4)], [2, 3, 1, 0, 4]),  # anchor inside the prefix
]


@pytest.mark.parametrize("seed", range(8))
def test_star_closed_form(seed):
    """Plans ending in two leaves of one anchor, counted in closed form, equal
    enumeration (counts, P_i, both algorithmic byte counts): leaves with one
    label and with two labels, directed graphs with self-loops, single and
    batch paths."""
    rng = np.random.default_rng(1300 + seed)
    directed = seed % 2 == 1
    n = int(rng.integers(10, 40))
    nl = int(rng.integers(1, 3))
    edges, labels = random_graph(rng, n, 0.3, nl, directed=directed, self_loops=directed)
    g = graph(n, edges, labels, symmetric=not directed)
    dg = mg.DeviceGraph(g)
    qs, orders, wants = [], [], []
    for k, qe, od in STAR_QUERIES:
        ql = rng.integers(0, max(labels) + 1, k).tolist()
        if seed % 4 == 0:
            ql[od[-1]] = ql[od[-2]]  # both leaves on one label
        if directed:
            qe = [(b, a) if rng.random() < 0.5 else (a, b) for a, b in qe]
        q = mg.CSRGraph.query(k, qe, ql, directed=directed)
        want = oracle_count(g, q, order=od)
        for tail in (1, 2):
            c, st = dg.count(q, stats=True, given_order=od, no_tail=tail)
            assert c == want["count"], (k, qe, ql, tail)
            assert st["level_rows"] == want["level_rows"], (k, qe, ql, tail)
            assert st["balg_bytes"] == want["balg"], (k, qe, ql, tail)
            assert st["balg_count_bytes"] == want["balg_count"], (k, qe, ql, tail)
        qs.append(q)
        orders.append(od)
        wants.append(want)
    counts, rows, _ = dg.batch_count_orders(qs, orders)
    for q, c, r, w in zip(qs, counts, rows, wants):
        assert c == w["count"] and r[:q.n + 1].tolist() == w["level_rows"]
    dg.free()


def test_subiso_exec_cli(tmp_path, c1):
    """The C++ subiso_exec (reference flags) over the C-ABI, exact count and rows."""
    import subprocess
    g, q, dg = c1
    g.Write(str(tmp_path / "g") + "/")
    q.Write(str(tmp_path / "p") + "/")
    exe = os.path.join(os.path.dirname(mg.__file__), "subiso_exec")
    out = tmp_path / "m.txt"
    r = subprocess.run([exe, "-p", str(tmp_path / "p") + "/", "-g", str(tmp_path / "g") + "/",
                        "-e", "", "-o", str(out), "-scheduler", "CHBL", "-mode", "emit"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = out.read_text().split()
    assert int(lines[0]) == dg.count(q)
    rows = np.array([[int(x) for x in ln.split(",")] for ln in lines[1:]], dtype=np.uint32)
    assert np.array_equal(rows.reshape(-1, 4), dg.emit(q))


def test_tail_aggregates_batch_and_chunks():
    """Pendant tails closed from hub aggregates (and summed in place for other
    vertices) in batches and with small level chunks equal enumeration."""
    g = mg.rmat(13, n_labels=6)
    dg = mg.DeviceGraph(g)
    rng = np.random.default_rng(5)
    qs = []
    for k, qe in TAIL_QUERIES[:4]:
        for _ in range(2):
            qs.append(mg.CSRGraph.query(k, qe, rng.integers(0, 6, k).tolist()))
    ref = [dg.count(q, no_tail=1) for q in qs]
    assert [dg.count(q) for q in qs] == ref
    assert dg.batch_count(qs).tolist() == ref
    assert dg.batch_count(qs, chunk_rows=4096).tolist() == ref
    assert dg.batch_count(qs, lanes="shared", chunk_rows=4096).tolist() == ref
    # no hubs at all: every aggregate summed in place
    dg0 = mg.DeviceGraph(g, hub_bytes=0)
    assert [dg0.count(q) for q in qs] == ref
    assert dg0.batch_count(qs).tolist() == ref
    dg0.free()
    dg.free()


def test_batch_orders_level_rows_and_budget(c1):
    """Per-query orders and prefix counts in one batch equal the oracle's; a
    per-query budget marks only over-budget queries."""
    g, q, dg = c1
    from matrixgraph_b200.order_model import random_connected_order
    rng = np.random.default_rng(11)
    qs, orders = [], []
    for i in range(24):
        x = mg.query_random(g, 3 + i % 5, 0.3, seed=3000 + i)
        qs.append(x)
        orders.append(random_connected_order(x, rng))
    counts, rows, _ = dg.batch_count_orders(qs, orders)
    for x, od, c, r in zip(qs, orders, counts, rows):
        want = oracle_count(g, x, order=od)
        assert c == want["count"]
        assert r[:x.n + 1].tolist() == want["level_rows"]
    budget = int(np.median([dg.count(x, stats=True)[1]["elements"] for x in qs]))
    counts_b, _, _ = dg.batch_count_orders(qs, [mg.plan_order(x) for x in qs],
                                           max_elements=max(budget, 1))
    singles = [dg.count(x) for x in qs]
    for cb, cs_ in zip(counts_b, singles):
        assert cb == cs_ or cb == 2 ** 64 - 1
    assert any(cb == 2 ** 64 - 1 for cb in counts_b)
    # Lane tables of 64 rows: most queries overflow their lane and are counted
    # again on the chunked path, where the budget must mark them the same way
    # instead of failing the whole batch.
    counts_o, _, st = dg.batch_count_orders(qs, [mg.plan_order(x) for x in qs],
                                            max_elements=max(budget, 1), chunk_rows=64)
    assert counts_o.tolist() == counts_b.tolist()


@pytest.fixture(scope="module")
def rmat20():
    """R-MAT scale 20 (1,048,576 vertices, edge factor 16, 32 Zipf labels): the
    C2 generator one scale down, with the five C2 query shapes."""
    g = mg.rmat(20)
    qs = [mg.query_walk(g, s, seed=2 + i) for i, s in enumerate(mg.SHAPES)]
    og = O.Graph.from_csr(g)
    dg = mg.DeviceGraph(g)
    yield g, qs, og, dg
    dg.free()


def test_rmat20_sampled_roots_all_shapes_both_tail_modes(rmat20):
    """Counts, per-prefix survivors P_i and algorithmic bytes of strided root
    samples (hubs included for all but the 4-cycle, whose top hub alone takes
    the oracle tens of seconds) equal the oracle's, with the closed-form
    pendant tail on and off."""
    g, qs, og, dg = rmat20
    threads = os.cpu_count() or 1
    for name, q in zip(mg.SHAPES, qs):
        oq = O.query_from_csr(q)
        order = O.reference_order(oq)
        nb = O.bucket_size(og, oq, order)
        first = 5 if name == "4-cycle" else 0
        for b, s in ((first, max(1, nb // 4096)), (3, max(1, nb // 8192))):
            want = O.count(og, oq, order=order, threads=threads, root_range=(b, nb),
                           root_step=s)
            assert want["count"] > 0, name
            for no_tail in (0, 1):
                c, st = dg.count(q, stats=True, root_range=(b, nb), root_step=s,
                                 no_tail=no_tail)
                assert c == want["count"], (name, b, s, no_tail)
                assert st["level_rows"] == want["level_rows"], (name, b, s, no_tail)
                assert st["balg_bytes"] == want["balg"], (name, b, s, no_tail)
                assert st["balg_count_bytes"] == want["balg_count"], (name, b, s, no_tail)


def test_root_step_partitions_and_matches_oracle():
    g = mg.chung_lu(3000, avg_deg=8, n_labels=3)
    og = O.Graph.from_csr(g)
    dg = mg.DeviceGraph(g)
    try:
        for i, shape in enumerate(mg.SHAPES):
            q = mg.query_walk(g, shape, seed=40 + i)
            oq = O.query_from_csr(q)
            full = dg.count(q)
            assert full == O.count(og, oq)["count"]
            for world in (2, 3, 7):
                parts = [dg.count(q, **mg.shard_strided(r, world)) for r in range(world)]
                assert sum(parts) == full, (shape, world)
            for b, e, s in ((0, 10 ** 9, 5), (7, 400, 3), (11, 12, 4), (0, 0, 9)):
                want = O.count(og, oq, root_range=(b, e if e else 2 ** 63), root_step=s)
                assert dg.count(q, root_range=(b, e), root_step=s) == want["count"]
            rows = dg.emit(q, root_range=(2, 10 ** 9), root_step=4)
            assert len(rows) == O.count(og, oq, root_range=(2, 2 ** 63), root_step=4)["count"]
    finally:
        dg.free()


@pytest.mark.parametrize("directed", [False, True])
def test_hub_bitmaps_never_change_results(directed):
    """Counts, P_i and emitted rows are identical whether slice probes go to
    hub bitmaps (every vertex a hub, a budget that cuts through the degree
    order) or to binary search only."""
    rng = np.random.default_rng(11 if directed else 12)
    n = 400
    edges, labels = random_graph(rng, n, 0.03, 3, directed=directed, self_loops=True)
    g = graph(n, edges, labels, symmetric=not directed)
    handles = {"none": mg.DeviceGraph(g, hub_bytes=0),
               "all": mg.DeviceGraph(g, hub_bytes=1 << 30, hub_min_degree=1),
               "cut": mg.DeviceGraph(g, hub_bytes=7 * 64, hub_min_degree=1)}
    try:
        assert handles["none"].info["hubs"] == 0
        assert handles["all"].info["hubs"] > 0 and handles["cut"].info["hubs"] > 0
        assert handles["cut"].info["hubs"] <= 7 * (1 if not directed else 1)
        for t in range(12):
            k = 3 + t % 4
            qe, ql = random_query(rng, k, 0.4, 3, directed=directed)
            q = mg.CSRGraph.query(k, qe, ql, directed=directed)
            want = oracle_count(g, q)
            for name, dg in handles.items():
                for no_tail in (0, 1):
                    c, st = dg.count(q, stats=True, no_tail=no_tail)
                    assert c == want["count"], (name, t, no_tail)
                    assert st["level_rows"] == want["level_rows"], (name, t, no_tail)
            if want["count"] <= 20000:
                rows = oracle_rows(g, q)
                for name, dg in handles.items():
                    assert np.array_equal(dg.emit(q), rows), (name, t)
    finally:
        for dg in handles.values():
            dg.free()


def test_batch_lane_pipeline_variants(c1):
    """The lane pipeline (sizes on the device, one host wait per batch) gives
    the per-query counts and prefix survivors for any lane count, with lane
    tables so small that most queries overflow and are counted again on the
    chunked path, and agrees with the level-synchronous shared-table run."""
    g, q, dg = c1
    rng = np.random.default_rng(21)
    qs = [mg.query_random(g, 3 + i % 6, 0.3, seed=5000 + i) for i in range(48)]
    qs += [mg.query_walk(g, s, seed=70 + i) for i, s in enumerate(mg.SHAPES)]
    single = [dg.count(x) for x in qs]
    orders = [mg.plan_order(x) for x in qs]
    _, ref_rows, _ = dg.batch_count_orders(qs, orders, lanes="shared")
    for lanes in (1, 3, 0):
        for chunk in (0, 64):
            got, st = dg.batch_count(qs, stats=True, lanes=lanes, chunk_rows=chunk)
            assert got.tolist() == single, (lanes, chunk)
            assert st["device_ms"] > 0
            counts, rows, _ = dg.batch_count_orders(qs, orders, lanes=lanes, chunk_rows=chunk)
            assert counts.tolist() == single
            assert rows.tolist() == ref_rows.tolist(), (lanes, chunk)
    assert dg.batch_count(qs, lanes="shared").tolist() == single
    # algorithmic bytes do not depend on how the batch ran
    balg = sum(dg.count(x, stats=True)[1]["balg_count_bytes"] for x in qs)
    for lanes, chunk in ((0, 0), (3, 64), ("shared", 0)):
        _, st = dg.batch_count(qs, stats=True, lanes=lanes, chunk_rows=chunk)
        assert st["balg_count_bytes"] == balg, (lanes, chunk)
    for x, c in list(zip(qs, single))[::7]:
        assert oracle_count(g, x)["count"] == c
    # pendant tails closed from dense aggregates inside the lanes, and without
    tq = [mg.CSRGraph.query(k, qe, rng.integers(0, 8, k).tolist()) for k, qe in TAIL_QUERIES]
    ref = [dg.count(x, no_tail=1) for x in tq]
    assert dg.batch_count(tq).tolist() == ref
    assert dg.batch_count(tq, no_tail=1).tolist() == ref


def test_bounded_device_wait_times_out_and_context_stays_usable(c1):
    """The lane pipeline's look-back wait gives up after its poll limit: a
    work/scan launch whose first tile is never handed out reports
    MG_E_TIMEOUT, and the graph handle keeps counting correctly after it."""
    import ctypes as C
    g, q, dg = c1
    for limit in (1, 64, 4096):
        status = C.c_int(12345)
        L.check(L.lib.mg_selftest_wait_timeout(dg.handle, C.byref(q.view), limit,
                                               C.byref(status)))
        assert status.value == L.MG_E_TIMEOUT, limit
    qs = [mg.query_random(g, 3 + i % 4, 0.3, seed=7000 + i) for i in range(16)]
    assert dg.batch_count(qs).tolist() == [dg.count(x) for x in qs]


def test_emit_sort_with_large_global_ids():
    """Emitted rows are sorted by the library's own radix sort over the
    global ids; ids above 2^24 exercise every digit pass, and the rows equal
    the oracle's sorted rows."""
    rng = np.random.default_rng(31)
    n = 1500
    edges, labels = random_graph(rng, n, 0.02, 2)
    g = graph(n, edges, labels)
    gid = (300_000_000 - 7 * np.arange(n)).astype(np.uint32)
    ge = g.array("globalid")
    oe = g.array("out_edges")
    ie = g.array("in_edges")
    same = oe.ctypes.data == ie.ctypes.data
    oe[:] = gid[oe]
    if not same:
        ie[:] = gid[ie]
    ge[:] = gid
    g.view.max_vid = int(gid.max())
    g.view.min_vid = int(gid.min())
    g.view.edges_globalid_by_localid = None
    g.view.localid_by_globalid = None
    dg = mg.DeviceGraph(g)
    try:
        for qe, ql in (([(0, 1), (1, 2), (2, 0)], [0, 1, 0]), ([(0, 1), (1, 2)], [1, 0, 1])):
            q = mg.CSRGraph.query(3, qe, ql)
            rows = dg.emit(q)
            assert len(rows) > 1000
            assert np.array_equal(rows, oracle_rows(g, q))
    finally:
        dg.free()


def test_subiso_exec_batch_tuned(tmp_path):
    """subiso_exec -batch, untuned and with an autotuner table (one batched
    call per tuned size bucket), prints the counts of the Python batch call;
    the autotuner's trials agree on every count."""
    import subprocess
    from matrixgraph_b200 import autotune
    g = mg.rmat(12, n_labels=4)
    dg = mg.DeviceGraph(g)
    qs = [mg.query_random(g, 3 + i % 5, 0.3, seed=4100 + i) for i in range(10)]
    want = dg.batch_count(qs).tolist()
    best = autotune.tune(dg, qs, sample=4,
                         candidates={"lanes": (2, 8), "probe_min": (1, 64), "grab": (0, 4)})
    assert set(best) == {autotune.bucket_of(q.n) for q in qs}
    table = str(tmp_path / "tune.txt")
    autotune.save_table(table, dg, best)
    loaded = autotune.load_table(table, dg)
    assert autotune.tuned_batch_count(dg, qs, loaded).tolist() == want
    g.Write(str(tmp_path / "g") + "/")
    names = []
    for i, q in enumerate(qs):
        q.Write(str(tmp_path / f"p{i}") + "/")
        names.append(str(tmp_path / f"p{i}") + "/")
    (tmp_path / "list.txt").write_text("\n".join(names) + "\n")
    exe = os.path.join(os.path.dirname(mg.__file__), "subiso_exec")
    for extra in ([], ["-tune", table]):
        out = tmp_path / "counts.txt"
        r = subprocess.run([exe, "-g", str(tmp_path / "g") + "/", "-batch",
                            str(tmp_path / "list.txt"), "-o", str(out), *extra],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        got = [int(ln.split()[-1]) for ln in out.read_text().splitlines() if ln.strip()]
        assert got == want, extra
        if extra:
            assert "tuned by" in r.stdout
    dg.free()
