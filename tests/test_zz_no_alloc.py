"""mg_subiso_count_noalloc: the count entry point that allocates no device memory.

It serves callers that cannot allocate device memory at call time (their HBM
is owned by another allocator, or the path must not pay cudaMalloc/cudaFree
synchronisation).  Its scratch is a static device array, so the test checks
that two calls in a row — the second one reusing whatever the first left in
that array — both equal the regular, allocating count entry point.  This file
is collected last so that a failure here never hides the other GPU tests.
"""
import ctypes as C

import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import _lib as L

from helpers import oracle_count

pytestmark = pytest.mark.gpu


def count_noalloc(dg, q, **kw):
    o, keep = mg.make_opts(**kw)
    c = C.c_uint64()
    L.check(L.lib.mg_subiso_count_noalloc(dg.handle, C.byref(q.view), C.byref(o), C.byref(c)))
    return c.value


def count_regular(dg, q, **kw):
    o, keep = mg.make_opts(**kw)
    c = C.c_uint64()
    L.check(L.lib.mg_subiso_count(dg.handle, C.byref(q.view), C.byref(o), C.byref(c)))
    return c.value


@pytest.mark.parametrize("graph", ["chung-lu-10k", "rmat-13"])
def test_noalloc_equals_regular_twice(graph):
    if graph == "chung-lu-10k":
        g = mg.chung_lu()
    else:
        g = mg.rmat(13, n_labels=8)
    dg = mg.DeviceGraph(g)
    queries = [mg.CSRGraph.query(4, [(0, 1), (1, 2), (2, 3), (3, 0)],
                                 mg.gen_labels(4, 8, "uniform", seed=2))]
    queries += [mg.query_walk(g, s, seed=2 + i) for i, s in enumerate(mg.SHAPES)]
    queries += [mg.query_random(g, 3 + i % 4, 0.3, seed=1000 + i) for i in range(6)]
    for i, q in enumerate(queries):
        want = count_regular(dg, q)
        first = count_noalloc(dg, q)
        second = count_noalloc(dg, q)
        assert first == want and second == want, (graph, first, second, want)
        if graph == "chung-lu-10k" and i < 6:
            # pinned directly against the CPU oracle, not only the other entry point
            assert first == oracle_count(g, q, threads=4)["count"], (graph, i)
    # small level tables (many chunks) and the strong order give the same counts
    q = queries[1]
    want = count_regular(dg, q)
    assert count_noalloc(dg, q, chunk_rows=256) == want
    assert count_noalloc(dg, q, order="strong") == want
    dg.free()


def test_noalloc_rejects_oversized_tables():
    g = mg.chung_lu(2000, avg_deg=6, n_labels=4)
    dg = mg.DeviceGraph(g)
    q = mg.CSRGraph.query(3, [(0, 1), (1, 2)], [0, 1, 2])
    with pytest.raises(L.MGError) as e:
        count_noalloc(dg, q, chunk_rows=1 << 30)
    assert e.value.code == L.MG_E_LIMIT
    assert count_noalloc(dg, q) == count_regular(dg, q)
    dg.free()


def test_noalloc_rejects_what_the_regular_count_rejects():
    """A pattern whose in-arrays disagree with its out-arrays is malformed for
    both entry points, and an inverted root range is an argument error that
    queues nothing on the shared array (the next call still counts right)."""
    g = mg.chung_lu(2000, avg_deg=6, n_labels=4)
    dg = mg.DeviceGraph(g)
    q = mg.CSRGraph.query(4, [(0, 1), (1, 2), (2, 3), (3, 0)], [0, 1, 0, 1])
    good = count_regular(dg, q)
    assert count_noalloc(dg, q) == good
    gid = q.array("globalid")
    inn = q.array("in_edges")
    saved = inn.copy()
    inn[0] = gid[2]  # vertex 0's first in-neighbour 1 -> 2: out- and in-edges disagree
    for fn in (count_regular, count_noalloc):
        with pytest.raises(L.MGError) as e:
            fn(dg, q)
        assert e.value.code == L.MG_E_FORMAT, fn.__name__
    inn[:] = saved
    with pytest.raises(L.MGError) as e:
        count_noalloc(dg, q, root_range=(5, 2))
    assert e.value.code == L.MG_E_ARG
    assert count_noalloc(dg, q) == good
    # the element budget is honoured as by the allocating entry point
    with pytest.raises(L.MGError) as e:
        count_noalloc(dg, q, max_elements=1)
    assert e.value.code == L.MG_E_LIMIT
    assert count_noalloc(dg, q) == good
    dg.free()
