"""The reference's own GPU GARMatch, run on the GPU: oracle/_ref/ref_gar_match
is oracle/ref_gar_match_main.cu compiled with the reference's
core/task/gpu_task/kernel/kernel_gar_match.cu where it lies
(oracle/build_ref.sh).  Its outputs pin

* the restated reference pipeline in oracle/gar.py (filters, frontier join,
  flattening) — equal whenever the frontier cap did not cut the join (the
  survivors of a cut depend on the order of atomics);
* matrixgraph_gar_match — equal wherever the reference's output is
  determined: no frontier cut and no reference filter dropping a vertex that
  a true match uses.

Inputs are valid by construction (every edge endpoint below n_vertices,
pattern indices below n_nodes), the cases are small, and every capacity is
set so that the reference's own guards keep all writes in bounds.  Every
array is present: the reference copies each input array to the device
unconditionally, so a missing array is not an input it defines."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from matrixgraph_b200.gar import gar_match
from oracle.gar import gar_match as oracle_gar

from gar_cases import doc_example, random_graph, random_pattern
from test_gar_abi import _lib_inputs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_gar_match")


def run_reference(g, p, row_cap, match_cap, reps=1, timing=None):
    """The reference's GARMatchKernelWrapper::GARMatch on (g, p); returns
    (status, num_conditions, rows[(pivot, cond_j, pos, offset, count)], ids).
    With reps > 1 the median wall time of the repeated calls is appended to
    the list `timing` (ms)."""
    n, m, k, pe = g.n_vertices, len(g.e_src), p.n_nodes, len(p.edge_src)
    assert g.v_id is not None and g.e_label is not None and p.edge_label is not None
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<9i", n, m, k, pe, row_cap, match_cap, 1, 1, 1))
            for arr, dt in ((g.v_id, "<u4"), (g.v_label, "<i4"), (g.e_src, "<u4"),
                            (g.e_dst, "<u4"), (list(range(m)), "<u4"), (g.e_label, "<i4"),
                            (p.node_label, "<i4"), (p.edge_src, "<i4"), (p.edge_dst, "<i4"),
                            (p.edge_label, "<i4")):
                f.write(np.asarray(arr, dtype=dt).tobytes())
        r = subprocess.run([EXE, fin, fout] + ([str(reps)] if reps > 1 else []),
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        if timing is not None:
            timing += [float(x.split()[1]) for x in r.stderr.splitlines()
                       if x.startswith("ref_gar_match_ms ")]
        raw = open(fout, "rb").read()
    status, nc, rs, ms = struct.unpack_from("<4i", raw, 0)
    rows = [struct.unpack_from("<Iiiii", raw, 16 + 20 * i) for i in range(rs)]
    ids = list(np.frombuffer(raw, dtype="<u4", count=ms, offset=16 + 20 * rs))
    return status, nc, rows, ids


def as_tuple(res):
    rows = list(zip(res.row_pivot_id, res.row_cond_j, res.row_pos, res.row_offset,
                    res.row_count))
    return res.num_conditions, [tuple(int(x) for x in r) for r in rows], \
        [int(x) for x in res.matched_v_ids]


needs_ref = pytest.mark.skipif(not os.path.exists(EXE),
                               reason="oracle/_ref/ref_gar_match not built (no reference)")


@needs_ref
def test_reference_run_reproduces_its_documented_example():
    g, p, exp = doc_example()
    status, nc, rows, ids = run_reference(g, p, 100, 100)
    assert status == 0
    assert nc == exp["num_conditions"]
    assert [r[0] for r in rows] == exp["row_pivot_id"]
    assert [r[4] for r in rows] == exp["row_count"]
    assert ids == exp["matched_v_ids"]
    # and the engine gives the same arrays
    lib = gar_match(*_lib_inputs(g, p), 100, 100)
    assert (lib.num_conditions, [tuple(int(x) for x in r) for r in zip(
        lib.row_pivot_id, lib.row_cond_j, lib.row_pos, lib.row_offset, lib.row_count)],
        [int(x) for x in lib.matched_v_ids]) == (nc, [tuple(r) for r in rows], ids)


@needs_ref
def test_reference_output_pins_the_restatement_and_the_engine():
    pinned = engine_pinned = 0
    for seed in range(40):
        rng = np.random.default_rng(900 + seed)
        n = int(rng.integers(8, 40))
        g = random_graph(rng, n, int(rng.integers(n, 5 * n)), v_labels=3,
                         e_labels=1 + seed % 2)
        p = random_pattern(rng, int(rng.integers(2, 5)), int(rng.integers(0, 3)), v_labels=3,
                           e_labels=1 + seed % 2)
        rcap, mcap = 1000, 4000
        status, nc, rows, ids = run_reference(g, p, rcap, mcap)
        assert status == 0
        got = (nc, [tuple(int(x) for x in r) for r in rows], [int(x) for x in ids])
        restated = oracle_gar(g, p, rcap, mcap, mode="reference")
        if restated.truncated:
            continue
        assert got == as_tuple(restated), seed
        pinned += 1
        if not restated.filters_pruned:
            lib = gar_match(*_lib_inputs(g, p), rcap, mcap)
            assert got == as_tuple(lib), seed
            engine_pinned += 1
    assert pinned >= 30 and engine_pinned >= 15, (pinned, engine_pinned)


@needs_ref
def test_reference_on_a_medium_graph():
    """A few hundred vertices and thousands of edges: the reference's join
    below its frontier capacity equals the restated reference, and the engine
    wherever the reference filters kept every used vertex."""
    for seed in range(4):
        rng = np.random.default_rng(1300 + seed)
        g = random_graph(rng, 200, 2000, v_labels=4, e_labels=2, self_loops=0.01)
        p = random_pattern(rng, 3, seed % 2, v_labels=4, e_labels=2)
        rcap, mcap = 10 ** 5, 10 ** 6
        status, nc, rows, ids = run_reference(g, p, rcap, mcap)
        assert status == 0
        got = (nc, [tuple(int(x) for x in r) for r in rows], [int(x) for x in ids])
        restated = oracle_gar(g, p, rcap, mcap, mode="reference")
        assert not restated.truncated
        assert got == as_tuple(restated), seed
        if not restated.filters_pruned:
            assert got == as_tuple(gar_match(*_lib_inputs(g, p), rcap, mcap)), seed


@needs_ref
@pytest.mark.parametrize("n,m", [(3000, 30000), (20000, 200000)])
def test_reference_timed_beside_the_library(n, m):
    """The reference's GPU GARMatch rebuilt for sm_100a, timed beside
    matrixgraph_gar_match on the same inputs (host arrays in and out for both,
    median of repeated calls after a warm-up); prints one JSON line.  Both
    calls must succeed; equality of the outputs is checked by the tests above
    where the reference's frontier cap and filters do not act."""
    import json
    import time
    rng = np.random.default_rng(77)
    g = random_graph(rng, n, m, v_labels=4, e_labels=2, self_loops=0.0)
    p = random_pattern(rng, 3, 0, v_labels=4, e_labels=2)
    rcap, mcap = 10 ** 5, 10 ** 7
    t_ref = []
    status, nc, rows, ids = run_reference(g, p, rcap, mcap, reps=3, timing=t_ref)
    assert status == 0 and len(t_ref) == 1
    args = _lib_inputs(g, p)
    res = gar_match(*args, rcap, mcap)
    t_lib = []
    for _ in range(3):
        t0 = time.perf_counter()
        res = gar_match(*args, rcap, mcap)
        t_lib.append(1e3 * (time.perf_counter() - t0))
    print(json.dumps({"workload": f"random multigraph, {n:,} vertices, {m:,} directed edges, "
                                  "4 vertex labels, 2 edge labels; 3-edge pattern",
                      "reference_gar_match_ms": t_ref[0],
                      "library_gar_match_ms": sorted(t_lib)[1],
                      "reference_ids": len(ids), "library_ids": int(res.match_size),
                      "library_matches": int(res.n_matches)}))
