"""matrixgraph_gar_match host logic that needs no GPU: inputs the reference
answers with an empty result before any matching, argument errors, and the
loud failure when matching is needed and no GPU is present."""
import ctypes as C

import numpy as np
import pytest

from matrixgraph_b200 import _lib as L
from matrixgraph_b200.gar import GARGraphArrays, GARPatternArrays, gar_match

from gar_cases import doc_example


def _lib_inputs(g, p):
    gg = GARGraphArrays(v_id=None if g.v_id is None else np.array(g.v_id, np.uint32),
                        v_label_idx=np.array(g.v_label, np.int32),
                        e_src=np.array(g.e_src, np.uint32), e_dst=np.array(g.e_dst, np.uint32),
                        e_label_idx=None if g.e_label is None else np.array(g.e_label, np.int32),
                        n_vertices=g.n_vertices)
    pp = GARPatternArrays(node_label_idx=np.array(p.node_label, np.int32),
                          edge_src=np.array(p.edge_src, np.int32),
                          edge_dst=np.array(p.edge_dst, np.int32),
                          edge_label_idx=None if p.edge_label is None else
                          np.array(p.edge_label, np.int32), n_nodes=p.n_nodes)
    return gg, pp


@pytest.mark.parametrize("case", ["no_edges", "bad_endpoint", "isolated", "no_label",
                                  "wrong_direction", "negative"])
def test_empty_results_without_matching(case):
    g, p, _ = doc_example()
    gg, pp = _lib_inputs(g, p)
    if case == "no_edges":
        pp = GARPatternArrays(pp.node_label_idx, np.zeros(0, np.int32), np.zeros(0, np.int32))
    elif case == "bad_endpoint":
        pp.edge_dst = np.array([2], np.int32)
    elif case == "isolated":
        pp = GARPatternArrays(np.array([0, 1, 1], np.int32), pp.edge_src, pp.edge_dst,
                              pp.edge_label_idx)
    elif case == "no_label":
        pp.edge_label_idx = np.array([6], np.int32)
    elif case == "wrong_direction":
        pp.node_label_idx = np.array([1, 0], np.int32)
    elif case == "negative":
        gg.n_vertices = -3
    rc, r = gar_match(gg, pp, 10, 10, raw=True)
    assert rc == 0
    assert (r.num_conditions, r.row_size, r.match_size, r.n_matches) == (1, 0, 0, 0)


def test_null_outputs_and_arrays_are_skipped():
    g, p, _ = doc_example()
    gg, pp = _lib_inputs(g, p)
    # no data labels / no pattern labels: empty result, status 0 (as the reference)
    rc = L.lib.matrixgraph_gar_match(None, None, 5, None, None, None, None, 0,
                                     None, 2, None, None, None, 1,
                                     None, None, None, None, None, None, 0, None, None, 0, None)
    assert rc == 0
    nc = C.c_int(-1)
    rc = L.lib.matrixgraph_gar_match(None, None, 5, None, None, None, None, 0,
                                     None, 2, None, None, None, 0,
                                     C.byref(nc), None, None, None, None, None, 0, None,
                                     None, 0, None)
    assert rc == 0 and nc.value == 1


def test_given_order_rejected():
    g, p, _ = doc_example()
    gg, pp = _lib_inputs(g, p)
    o = L.default_opts()
    o.order = L.MG_ORDER_GIVEN
    rc, r = gar_match(gg, pp, 10, 10, opts=o, raw=True)
    assert rc == L.MG_E_ARG and r.num_conditions == 1


def test_matching_without_gpu_fails_loudly():
    from conftest import gpu_count
    if gpu_count() > 0:
        pytest.skip("a GPU is present")
    g, p, _ = doc_example()
    gg, pp = _lib_inputs(g, p)
    rc, r = gar_match(gg, pp, 10, 10, raw=True)
    assert rc == L.MG_E_CUDA
    assert (r.num_conditions, r.row_size, r.match_size) == (1, 0, 0)


@pytest.mark.parametrize("seed", range(60))
def test_instance_and_flatten_against_oracle(seed):
    """The two host halves of the GAR entry on the CPU: the matching instance
    built by the library, matched by the C oracle, flattened by the library,
    equals the GAR oracle's exact output."""
    import oracle
    from matrixgraph_b200.gar import gar_flatten, gar_instance
    from oracle.gar import gar_match as oracle_gar
    from gar_cases import random_graph, random_pattern

    rng = np.random.default_rng(seed)
    n = int(rng.integers(5, 40))
    g = random_graph(rng, n, int(rng.integers(n, 5 * n)), v_labels=int(rng.integers(1, 4)),
                     e_labels=int(rng.integers(1, 4)), with_elabels=seed % 4 != 0,
                     with_ids=seed % 3 != 0)
    p = random_pattern(rng, int(rng.integers(1, 5)), int(rng.integers(0, 4)),
                       v_labels=int(rng.integers(1, 4)), e_labels=int(rng.integers(1, 4)),
                       self_loop=seed % 7 == 0, with_elabels=seed % 5 != 0)
    rcap = int(rng.choice([0, 2, 9, 10 ** 5]))
    mcap = int(rng.choice([0, 3, 17, 10 ** 6]))
    orc = oracle_gar(g, p, rcap, mcap, mode="exact")
    inst = gar_instance(*_lib_inputs(g, p))
    if inst is None:
        assert orc.n_embeddings == 0 and orc.num_conditions == 1
        return
    data, query = inst
    assert query.n >= p.n_nodes
    rows = oracle.emit(oracle.Graph.from_csr(data), oracle.query_from_csr(query))
    assert len(rows) == orc.n_embeddings
    if len(rows) == 0:
        assert orc.num_conditions == 1 and orc.row_size == 0
        return
    res = gar_flatten(rows, p.n_nodes, g.v_id, g.n_vertices, rcap, mcap)
    assert res.num_conditions == orc.num_conditions
    assert res.row_pivot_id.tolist() == orc.row_pivot_id
    assert res.row_pos.tolist() == orc.row_pos and res.row_cond_j.tolist() == orc.row_cond_j
    assert res.row_offset.tolist() == orc.row_offset
    assert res.row_count.tolist() == orc.row_count
    assert res.matched_v_ids.tolist() == orc.matched_v_ids


def test_flatten_rows_in_any_order_with_repeats():
    from matrixgraph_b200.gar import gar_flatten
    g, p, exp = doc_example()
    rows = np.array([[1, 4], [0, 3], [0, 2], [0, 3], [1, 4]], np.uint32)
    r = gar_flatten(rows, 2, g.v_id, 5, 100, 100)
    assert r.matched_v_ids.tolist() == exp["matched_v_ids"]
    assert r.row_offset.tolist() == exp["row_offset"] and r.num_conditions == 2


@pytest.mark.parametrize("seed", range(40))
def test_subdivided_instance_against_oracle(seed):
    """Patterns with two edge labels: the subdivided instance, matched by the
    C oracle and flattened by the library, equals the exact GAR output."""
    import oracle
    from matrixgraph_b200.gar import gar_flatten, gar_instance
    from oracle.gar import gar_match as oracle_gar
    from gar_cases import two_label_case

    rng = np.random.default_rng(3000 + seed)
    g, p = two_label_case(rng)
    orc = oracle_gar(g, p, 10 ** 5, 10 ** 6, mode="exact")
    inst = gar_instance(*_lib_inputs(g, p))
    if inst is None:
        assert orc.n_embeddings == 0
        return
    data, query = inst
    distinct = len({(s, d, l) for s, d, l in zip(p.edge_src, p.edge_dst, p.edge_label)})
    two = len(set(p.edge_label)) >= 2
    assert query.n == p.n_nodes + (distinct if two else 0)
    rows = oracle.emit(oracle.Graph.from_csr(data), oracle.query_from_csr(query))
    assert len(rows) == orc.n_embeddings
    if len(rows):
        res = gar_flatten(rows, p.n_nodes, g.v_id, g.n_vertices, 10 ** 5, 10 ** 6)
        assert res.matched_v_ids.tolist() == orc.matched_v_ids
        assert res.row_count.tolist() == orc.row_count
        assert res.row_pivot_id.tolist() == orc.row_pivot_id


def test_pattern_limits_before_any_device_work():
    from oracle.gar import GarGraph, GarPattern
    # every vertex label 0, edges of labels 0 and 1 in both directions along a path
    n = 20
    src = list(range(n - 1)) + list(range(1, n))
    dst = list(range(1, n)) + list(range(n - 1))
    g = GarGraph(v_id=None, v_label=[0] * n, e_src=src * 2, e_dst=dst * 2,
                 e_label=[0] * len(src) + [1] * len(src), n_vertices=n)
    # 17 pattern nodes on a path: beyond 16
    p = GarPattern([0] * 17, list(range(16)), list(range(1, 17)), [0] * 16, 17)
    rc, r = gar_match(*_lib_inputs(g, p), 10, 10, raw=True)
    assert rc == L.MG_E_LIMIT and r.num_conditions == 1
    # 9 nodes and 8 distinct edges over two edge labels: 17 subdivided vertices
    p = GarPattern([0] * 9, list(range(8)), list(range(1, 9)), [i % 2 for i in range(8)], 9)
    rc, r = gar_match(*_lib_inputs(g, p), 10, 10, raw=True)
    assert rc == L.MG_E_LIMIT and b"distinct edges" in L.lib.mg_last_error()
