"""GAR match oracle: the reference restatement against the exact mode, brute
force, the reference's documented output example and its capacity rules."""
import numpy as np
import pytest

from oracle.gar import GarGraph, GarPattern, _Heap, _bitmap_count, gar_match

from gar_cases import brute_force, doc_example, random_graph, random_pattern


def _group(embs, k, g):
    """Expected flattening from a list of node maps, no capacity limits."""
    inst = (lambda v: g.v_id[v]) if g.v_id is not None else (lambda v: v)
    out = []
    for pivot in sorted({e[0] for e in embs}):
        for pos in range(k):
            out.append((inst(pivot), pos, sorted({inst(e[pos]) for e in embs if e[0] == pivot})))
    return out


def _rows(r):
    return [(r.row_pivot_id[i], r.row_pos[i],
             r.matched_v_ids[r.row_offset[i]:r.row_offset[i] + r.row_count[i]])
            for i in range(r.row_size)]


def test_documented_example_both_modes():
    g, p, exp = doc_example()
    for mode in ("reference", "exact"):
        r = gar_match(g, p, 100, 100, mode=mode)
        assert r.rc == 0 and not r.truncated and not r.filters_pruned
        for key, val in exp.items():
            assert getattr(r, key) == val, (mode, key)


def test_bitmap_count_and_heap_as_written():
    # bits 0..28 are counted, 29..31 are not
    assert _bitmap_count((1 << 29) - 1) == 29
    assert _bitmap_count(1 << 29) == 0 and _bitmap_count(1 << 31) == 0
    h = _Heap()
    for v in (5, 3, 9):
        h.insert(v)
    assert h.offset == 3 and sorted(h.data[:3]) == [3, 5, 9]
    for v in range(20, 10, -1):
        h.insert(v)
    assert h.offset == 7


@pytest.mark.parametrize("seed", range(40))
def test_exact_mode_matches_brute_force(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(4, 8))
    g = random_graph(rng, n, int(rng.integers(n, 3 * n)), v_labels=2, e_labels=2,
                     with_elabels=seed % 3 != 0, with_ids=seed % 2 == 0)
    p = random_pattern(rng, int(rng.integers(1, 4)), int(rng.integers(0, 3)), v_labels=2,
                       e_labels=2, self_loop=seed % 5 == 0, with_elabels=seed % 4 != 1)
    r = gar_match(g, p, 10 ** 6, 10 ** 6, mode="exact")
    bf = brute_force(g, p)
    covered = set(p.edge_src) | set(p.edge_dst)
    if len(covered) < p.n_nodes:
        bf = []
    assert r.n_embeddings == len(set(bf))
    assert _rows(r) == _group(bf, p.n_nodes, g)
    assert r.num_conditions == (p.n_nodes if bf else 1)


def test_reference_mode_agrees_where_determined():
    """Where no join step overflowed and no filter rejected a used vertex, the
    restated reference and the exact mode give the same output."""
    agree = pruned = truncated = 0
    for seed in range(60):
        rng = np.random.default_rng(1000 + seed)
        n = int(rng.integers(6, 20))
        g = random_graph(rng, n, int(rng.integers(n, 4 * n)), v_labels=3, e_labels=2)
        p = random_pattern(rng, int(rng.integers(2, 5)), int(rng.integers(0, 3)), v_labels=3,
                           e_labels=2)
        cap = int(rng.choice([6, 40, 10 ** 6]))
        ref = gar_match(g, p, cap, cap, mode="reference")
        ex = gar_match(g, p, cap, cap, mode="exact")
        if ref.truncated:
            truncated += 1
            continue
        if ref.filters_pruned:
            pruned += 1
            continue
        assert _rows(ref) == _rows(ex), seed
        assert ref.num_conditions == ex.num_conditions
        agree += 1
    assert agree >= 30, (agree, pruned, truncated)


def test_capacity_rules():
    g, p, exp = doc_example()
    # row capacity 3: the third row is the last
    r = gar_match(g, p, 3, 100)
    assert r.row_pivot_id == [126, 126, 138] and r.matched_v_ids == [126, 183, 115407, 138]
    # id capacity 2: the row that meets it keeps the ids that fit, then output stops
    r = gar_match(g, p, 100, 2)
    assert r.row_count == [1, 1] and r.matched_v_ids == [126, 183]
    # id capacity 0: one row with no ids
    r = gar_match(g, p, 100, 0)
    assert r.row_size == 1 and r.row_count == [0] and r.num_conditions == 2
    # row capacity 0: no rows, but matches exist
    r = gar_match(g, p, 0, 100)
    assert r.row_size == 0 and r.num_conditions == 2


def test_empty_results():
    g, p, _ = doc_example()
    for pp in (GarPattern([0, 1], [], [], [], 2),                 # no pattern edge
               GarPattern([0, 1], [0], [2], [5], 2),              # endpoint out of range
               GarPattern([0, 1, 1], [0], [1], [5], 3),           # node on no edge
               GarPattern([0, 1], [0], [1], [6], 2),              # no edge with label 6
               GarPattern([1, 0], [0], [1], [5], 2)):             # no (1 -> 0) edge
        for mode in ("reference", "exact"):
            r = gar_match(g, pp, 10, 10, mode=mode)
            assert (r.rc, r.num_conditions, r.row_size, r.match_size) == (0, 1, 0, 0)
    # data edge labels absent: pattern edge labels are not compared
    g2 = GarGraph(g.v_id, g.v_label, g.e_src, g.e_dst, None, g.n_vertices)
    assert gar_match(g2, GarPattern([0, 1], [0], [1], [6], 2), 10, 10).n_embeddings == 3


def test_restated_helpers_match_the_reference_build():
    """The heap, popcount and label hash of oracle/gar.py against outputs of
    the reference's own headers (tests/golden/make_gar_golden.py)."""
    import json
    import os

    from oracle.gar import _hash_table
    path = os.path.join(os.path.dirname(__file__), "golden", "gar_helpers.json")
    ref = json.load(open(path))
    assert [_hash_table(k) for k in range(len(ref["hash"]))] == ref["hash"]
    for x, c in ref["count"]:
        assert _bitmap_count(x) == c, x
    assert len(ref["heap"]) == 300
    for case in ref["heap"]:
        h = _Heap()
        for v in case["in"]:
            h.insert(v)
        assert h.offset == case["offset"]
        assert h.data[:h.offset] == case["data"], case["in"]
