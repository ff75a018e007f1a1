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


def test_censoring_rule_of_the_summary():
    """Queries both orders finish give measured ratios; a censored reference
    against a finished learned order is charged the budget at the learned
    order's elements per ms (a win), the reverse a loss, and queries both
    orders leave unfinished stay out of the medians."""
    rows = [
        {"done_ref": True, "done_learned": True, "ms_ref": 4.0, "ms_learned": 2.0,
         "elements_ref": 400, "elements_learned": 200},
        {"done_ref": False, "done_learned": True, "ms_ref": None, "ms_learned": 1.0,
         "elements_learned": 100},
        {"done_ref": True, "done_learned": False, "ms_ref": 1.0, "ms_learned": None,
         "elements_ref": 50},
        {"done_ref": False, "done_learned": False, "ms_ref": None, "ms_learned": None},
    ]
    s = W.order_summary(rows, budget=1000, plan_ms=0.0)
    assert (s["finished_both"], s["finished_learned_only"], s["finished_reference_only"],
            s["finished_neither"]) == (1, 1, 1, 1)
    # ratios: 2.0 (both), 1000/(100 per ms)/1 ms = 10.0 (win), 1 ms/(1000/50 ms) = 0.05 (loss)
    assert abs(s["median_speedup_device"] - 2.0) < 1e-12
    assert abs(s["median_speedup_device_both_finished"] - 2.0) < 1e-12
    assert abs(s["median_element_ratio_both_finished"] - 2.0) < 1e-12
    s2 = W.order_summary(rows, budget=1000, plan_ms=1.0)
    assert abs(s2["median_speedup_with_planning"] - 4.0 / 3.0) < 1e-12
