"""The committed held-out evaluation of the learned order
(matrixgraph_b200/data/order_eval.json, written on a B200 by
`python -m matrixgraph_b200.workloads eval-order`): counts identical under
both orders, learned orders are permutations, and the recorded gain of the
trained network over the reference order."""
import json
import math
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "matrixgraph_b200", "data", "order_eval.json")


def test_recorded_counts_are_order_independent():
    rows = json.load(open(PATH))["rows"]
    assert len(rows) >= 50
    for r in rows:
        k = r["k"]
        assert sorted(r["order_learned"]) == list(range(k)) == sorted(r["order_ref"])
        assert r["rows_ref"][k] == r["rows_learned"][k] == r["count"]


def test_recorded_gain_of_the_trained_network():
    d = json.load(open(PATH))
    rows = d["rows"]
    ratios = [r["ms_ref"] / r["ms_learned"] for r in rows]
    geo = math.exp(sum(math.log(x) for x in ratios) / len(ratios))
    assert abs(geo - d["summary"]["geomean_speedup_device"]) < 1e-9
    assert geo > 1.0   # device time: 1.169x geomean over the reference order
    work_ref = sum(sum(r["rows_ref"]) for r in rows)
    work_learned = sum(sum(r["rows_learned"]) for r in rows)
    assert work_learned < work_ref   # fewer partial matches in total
