"""The committed held-out evaluation of the learned order
(matrixgraph_b200/data/order_eval.json, written on a B200 by
`python -m matrixgraph_b200.workloads c4 OUTDIR`) against the committed
held-out set (data/heldout_seeds.json): it covers the test half in order,
counts are the recorded ones under both orders, learned orders are
permutations, and the summary is what its rows give under the censoring
rule of workloads.order_summary."""
import json
import os

from matrixgraph_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "matrixgraph_b200", "data", "order_eval.json")


def _load():
    with open(PATH) as f:
        ev = json.load(f)
    with open(W.HELDOUT_SEEDS) as f:
        sel = json.load(f)
    return ev, sel


def test_selection_record_is_order_independent():
    _, sel = _load()
    assert sel["criterion"].startswith("some seeded random connected order")
    assert sel["orders_per_seed"] == W.SELECT_ORDERS
    seeds = [q["seed"] for q in sel["queries"]]
    assert seeds == sorted(seeds) and len(set(seeds)) == len(seeds)
    assert all(sel["first_seed"] <= s < sel["first_seed"] + sel["seeds_scanned"] for s in seeds)
    assert all(6 <= q["k"] <= 10 and q["k"] == W.learned_k(q["seed"]) for q in sel["queries"])


def test_rows_cover_the_test_half_with_recorded_counts():
    ev, sel = _load()
    test, val = W.heldout_split(sel)
    rows = ev["rows"]
    assert [r["seed"] for r in rows] == [q["seed"] for q in test]
    assert not {q["seed"] for q in test} & {q["seed"] for q in val}
    for r, q in zip(rows, test):
        assert r["count"] == q["count"]
        assert sorted(r["order_learned"]) == list(range(r["k"])) == sorted(r["order_ref"])
        for name in ("ref", "learned"):
            if r[f"done_{name}"]:
                assert r[f"ms_{name}"] > 0 and r[f"elements_{name}"] > 0


def test_summary_is_what_the_rows_give():
    ev, _ = _load()
    s = ev["summary"]
    again = W.order_summary(ev["rows"], s["budget_elements"], s["planning_ms_per_query"])
    for key, v in again.items():
        assert s[key] == v, key
    assert s["n"] == len(ev["rows"])
    assert s["finished_both"] + s["finished_learned_only"] + s["finished_reference_only"] + \
        s["finished_neither"] == s["n"]
