"""matrixgraph_gar_match on the GPU against the GAR oracle: the reference's
documented example, random directed multigraphs with vertex and edge labels
(single-label and subdivided edge-label paths), capacity cuts, emission split
over level-0 ranges, and agreement with the restated reference wherever its
output is determined."""
import numpy as np
import pytest

from matrixgraph_b200 import _lib as L
from matrixgraph_b200.gar import gar_match
from oracle.gar import GarPattern, gar_match as oracle_gar

from gar_cases import doc_example, random_graph, random_pattern, two_label_case
from test_gar_abi import _lib_inputs

pytestmark = pytest.mark.gpu


def _same(lib, orc):
    assert lib.num_conditions == orc.num_conditions
    assert lib.row_pivot_id.tolist() == orc.row_pivot_id
    assert lib.row_cond_j.tolist() == orc.row_cond_j
    assert lib.row_pos.tolist() == orc.row_pos
    assert lib.row_offset.tolist() == orc.row_offset
    assert lib.row_count.tolist() == orc.row_count
    assert lib.matched_v_ids.tolist() == orc.matched_v_ids


def _check(g, p, rcap, mcap, opts=None):
    orc = oracle_gar(g, p, rcap, mcap, mode="exact")
    lib = gar_match(*_lib_inputs(g, p), rcap, mcap, opts=opts)
    _same(lib, orc)
    assert lib.n_matches == orc.n_embeddings
    return lib, orc


def test_documented_example():
    g, p, exp = doc_example()
    lib = gar_match(*_lib_inputs(g, p), 100, 100)
    for key, val in exp.items():
        got = getattr(lib, key)
        assert (got if isinstance(got, int) else got.tolist()) == val, key
    assert lib.n_matches == 3


@pytest.mark.parametrize("seed", range(48))
def test_random_small(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(5, 40))
    g = random_graph(rng, n, int(rng.integers(n, 5 * n)), v_labels=int(rng.integers(1, 4)),
                     e_labels=int(rng.integers(1, 4)), with_elabels=seed % 4 != 0,
                     with_ids=seed % 3 != 0)
    p = random_pattern(rng, int(rng.integers(1, 5)), int(rng.integers(0, 4)),
                       v_labels=int(rng.integers(1, 4)), e_labels=int(rng.integers(1, 4)),
                       self_loop=seed % 7 == 0, with_elabels=seed % 5 != 0)
    cap = int(rng.choice([0, 3, 17, 10 ** 6]))
    rcap = int(rng.choice([0, 2, 9, 10 ** 5]))
    _check(g, p, rcap, cap)


@pytest.mark.parametrize("seed", range(24))
def test_two_edge_labels(seed):
    rng = np.random.default_rng(3000 + seed)
    g, p = two_label_case(rng)
    _check(g, p, 10 ** 5, 10 ** 6)


@pytest.mark.parametrize("seed", range(6))
def test_random_medium(seed):
    rng = np.random.default_rng(100 + seed)
    n = 600
    g = random_graph(rng, n, 24000, v_labels=4, e_labels=3, self_loops=0.01)
    p = random_pattern(rng, 3 + seed % 2, seed % 3, v_labels=4, e_labels=3 if seed % 2 else 1)
    _check(g, p, 10 ** 6, 10 ** 7)


def test_orders_give_the_same_output():
    rng = np.random.default_rng(7)
    g = random_graph(rng, 300, 9000, v_labels=3, e_labels=2)
    p = random_pattern(rng, 4, 2, v_labels=3, e_labels=2)
    base = gar_match(*_lib_inputs(g, p), 10 ** 5, 10 ** 6)
    for order in (L.MG_ORDER_STRONG, L.MG_ORDER_LEARNED):
        o = L.default_opts()
        o.order = order
        other = gar_match(*_lib_inputs(g, p), 10 ** 5, 10 ** 6, opts=o)
        assert other.n_matches == base.n_matches > 1000
        assert other.matched_v_ids.tolist() == base.matched_v_ids.tolist()
        assert other.row_count.tolist() == base.row_count.tolist()


def test_emission_split_over_level0_ranges(monkeypatch):
    rng = np.random.default_rng(11)
    g = random_graph(rng, 200, 4000, v_labels=2, e_labels=2)
    p = random_pattern(rng, 3, 1, v_labels=2, e_labels=2)
    whole = gar_match(*_lib_inputs(g, p), 10 ** 5, 10 ** 6)
    assert whole.n_matches > 1000
    monkeypatch.setenv("MG_GAR_EMIT_ROWS", "37")
    lib, orc = _check(g, p, 10 ** 5, 10 ** 6)
    assert lib.matched_v_ids.tolist() == whole.matched_v_ids.tolist()


def test_agrees_with_restated_reference_where_determined():
    agree = 0
    for seed in range(30):
        rng = np.random.default_rng(500 + seed)
        n = int(rng.integers(8, 25))
        g = random_graph(rng, n, int(rng.integers(n, 4 * n)), v_labels=3, e_labels=2)
        p = random_pattern(rng, int(rng.integers(2, 5)), int(rng.integers(0, 3)), v_labels=3,
                           e_labels=2)
        ref = oracle_gar(g, p, 1000, 1000, mode="reference")
        if ref.truncated or ref.filters_pruned:
            continue
        _same(gar_match(*_lib_inputs(g, p), 1000, 1000), ref)
        agree += 1
    assert agree >= 15


def test_pattern_size_limit():
    rng = np.random.default_rng(3)
    g = random_graph(rng, 50, 120, v_labels=1, e_labels=2)
    # 9 nodes on a path with alternating edge labels: 9 + 8 > 16
    p = GarPattern(node_label=[0] * 9, edge_src=list(range(8)), edge_dst=list(range(1, 9)),
                   edge_label=[i % 2 for i in range(8)], n_nodes=9)
    rc, r = gar_match(*_lib_inputs(g, p), 10, 10, raw=True)
    if rc == 0:  # no usable edge for some pattern edge: empty before matching
        assert r.num_conditions == 1
    else:
        assert rc == L.MG_E_LIMIT
    # one edge label: plain path, 9 nodes accepted
    p.edge_label = [0] * 8
    _check(g, p, 10 ** 4, 10 ** 5)


def test_device_from_environment(monkeypatch):
    g, p, exp = doc_example()
    monkeypatch.setenv("MATRIXGRAPH_CUDA_DEVICE", "0")
    assert gar_match(*_lib_inputs(g, p), 100, 100).matched_v_ids.tolist() == exp["matched_v_ids"]
    monkeypatch.setenv("MATRIXGRAPH_CUDA_DEVICE", "999")  # invalid: current device
    assert gar_match(*_lib_inputs(g, p), 100, 100).matched_v_ids.tolist() == exp["matched_v_ids"]
