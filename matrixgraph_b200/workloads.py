"""Seeded benchmark workloads.

* ``rmat_graph(scale)`` — symmetrised R-MAT (edge factor 16, a=0.57 b=0.19
  c=0.19), self-loops and duplicates removed, ids not permuted, 32 Zipf(1.0)
  labels: the single-query (scale 22) and batched (scale 22) data graph.
* ``shape_queries(g)`` — the five single-query shapes with random-walk labels.
* ``c5_graph()`` / ``c5_queries(g, n)`` — R-MAT scale 26 with 64 Zipf(1.2)
  labels and 6-8-vertex queries (4-clique or chorded 5-cycle plus a pendant
  path), random-walk labels.
* batched queries — random connected queries, k uniform in 3..8, a random
  recursive spanning tree plus every other pair with probability 0.3,
  random-walk labels.  Some seeds give search spaces far beyond any time
  budget on a scale-22 power-law graph (trees of common labels around hubs),
  so the batch is the first 4,096 seeds (from 1000) whose count under the
  reference order expands at most ``BATCH_BUDGET`` candidate elements.  The
  selection is deterministic (element counts are exact integers) and the kept
  seeds, sizes and counts are committed in ``data/batch_seeds.json``.

    python -m matrixgraph_b200.workloads select-batch OUT.json
    python -m matrixgraph_b200.workloads train-order OUTDIR [N]
    python -m matrixgraph_b200.workloads c4 OUTDIR [N_TRAIN]
    python -m matrixgraph_b200.workloads eval-batch MODEL_DIR/ OUT.json

Learned order: training queries are random connected queries with k uniform
in 6..10 (seeds from 100000, taken in order) on the scale-20 graph; the
enumerator records P_i for the reference order and 8 random connected orders
of each under a per-run budget of TRAIN_BUDGET elements, and every run that
finishes gives one sample per prefix (a heavy query enters through the
orders that finish, whatever its reference order costs).  The seeds and run
totals are committed with the model (data/order_train_record.json).
Held-out queries use seeds from 200000 on the scale-22 graph.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

from . import _lib as L
from .graph import SHAPES, query_random, query_walk, rmat
from .subiso import DeviceGraph

HERE = os.path.dirname(os.path.abspath(__file__))
BATCH_SEEDS = os.path.join(HERE, "data", "batch_seeds.json")
BATCH_BUDGET = 1 << 28
BATCH_FIRST_SEED = 1000
BATCH_SIZE = 4096


def rmat_graph(scale: int = 22):
    return rmat(scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=32, label_kind="zipf",
                zipf_s=1.0, label_seed=1)


def shape_queries(g, only: str = ""):
    keep = [x for x in only.split(",") if x]
    return [query_walk(g, s, seed=2 + i) for i, s in enumerate(SHAPES) if not keep or s in keep]


def batch_k(seed: int) -> int:
    """Query size of a batch seed: uniform over 3..8."""
    return int(np.random.default_rng(seed).integers(3, 9))


def batch_query(g, seed: int):
    return query_random(g, batch_k(seed), 0.3, seed)


def batch_queries(g, n: int | None = None):
    with open(BATCH_SEEDS) as f:
        rec = json.load(f)
    seeds = rec["seeds"][:n] if n else rec["seeds"]
    return [batch_query(g, s) for s in seeds], rec


def select_batch(dg: DeviceGraph, g, n: int = BATCH_SIZE, budget: int = BATCH_BUDGET,
                 first_seed: int = BATCH_FIRST_SEED, log=None):
    seeds, ks, counts, elements, dropped = [], [], [], [], []
    s = first_seed
    while len(seeds) < n:
        q = batch_query(g, s)
        try:
            c, st = dg.count(q, stats=True, max_elements=budget)
            seeds.append(s)
            ks.append(q.n)
            counts.append(int(c))
            elements.append(int(st["elements"]))
        except L.MGError as e:
            if e.code != L.MG_E_LIMIT:
                raise
            dropped.append(s)
        s += 1
        if log and (s - first_seed) % 512 == 0:
            log(f"seed {s}: kept {len(seeds)}, dropped {len(dropped)}")
    return {"graph": "rmat scale 22 (workloads.rmat_graph)", "budget_elements": budget,
            "first_seed": first_seed, "order": "reference", "seeds": seeds, "k": ks,
            "counts": counts, "elements": elements, "dropped": dropped}


# ---- large and skewed: R-MAT scale 26 (configuration C5) ---------------------
C5_SCALE = 26
C5_LABELS = 64
C5_ZIPF = 1.2
C5_FIRST_SEED = 300000


def c5_graph(scale: int = C5_SCALE):
    """Symmetrised R-MAT (edge factor 16, a=0.57 b=0.19 c=0.19, self-loops and
    repeats removed, ids not permuted) with 64 Zipf(s=1.2) labels."""
    return rmat(scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=C5_LABELS, label_kind="zipf",
                zipf_s=C5_ZIPF, label_seed=1)


def c5_shape(q: int):
    """Shape of C5 query q: k uniform in {6, 7, 8}; even q: a 4-clique plus a
    pendant path of k-4 vertices hung from one clique vertex; odd q: a 5-cycle
    plus one or two chords plus a pendant path of k-5 vertices hung from one
    cycle vertex.  Drawn from numpy's PCG64 seeded with 300000 + q."""
    rng = np.random.default_rng(C5_FIRST_SEED + q)
    k = int(rng.integers(6, 9))
    if q % 2 == 0:
        core = 4
        edges = [(a, b) for a in range(4) for b in range(a + 1, 4)]
    else:
        core = 5
        edges = [(i, (i + 1) % 5) for i in range(5)]
        chords = [(0, 2), (0, 3), (1, 3), (1, 4), (2, 4)]
        for j in rng.choice(len(chords), size=int(rng.integers(1, 3)), replace=False):
            edges.append(chords[int(j)])
    prev = int(rng.integers(0, core))
    for v in range(core, k):
        edges.append((prev, v))
        prev = v
    return k, sorted((min(a, b), max(a, b)) for a, b in edges)


def c5_queries(g, n: int, first: int = 0):
    """C5 queries first..first+n-1 with random-walk labels (seed 300000 + q)."""
    return [query_walk(g, c5_shape(q), seed=C5_FIRST_SEED + q) for q in range(first, first + n)]


# ---- learned order: training and held-out queries ---------------------------
TRAIN_SCALE = 20
TRAIN_FIRST_SEED = 100000
EVAL_FIRST_SEED = 200000
TRAIN_BUDGET = 1 << 26
EVAL_BUDGET = 1 << 27
MODEL_DIR = os.path.join(HERE, "data", "order_model") + "/"


def learned_k(seed: int) -> int:
    """Query size of a learned-order seed: uniform over 6..10."""
    return int(np.random.default_rng(seed).integers(6, 11))


def learned_query(g, seed: int):
    return query_random(g, learned_k(seed), 0.3, seed)


def select_queries(dg, g, make, first_seed, n, budget, max_candidates, log=None,
                   max_seconds=None):
    """First n seeds whose reference-order count needs at most `budget`
    candidate elements (deterministic: element counts are exact); stops early
    after max_candidates seeds or max_seconds."""
    import time
    t0 = time.time()
    kept, dropped, s = [], 0, first_seed
    while len(kept) < n and s - first_seed < max_candidates:
        if max_seconds and time.time() - t0 > max_seconds:
            break
        q = make(g, s)
        try:
            c, st = dg.count(q, stats=True, max_elements=budget)
            kept.append({"seed": s, "k": q.n, "count": int(c), "elements": int(st["elements"]),
                         "ms": st["device_ms"]})
        except L.MGError as e:
            if e.code != L.MG_E_LIMIT:
                raise
            dropped += 1
        s += 1
        if log and (s - first_seed) % 4000 == 0:
            log(f"seed {s}: kept {len(kept)} dropped {dropped}")
    return kept, dropped


def train_order(outdir: str, n_train: int = 8000, n_random: int = 8, epochs: int = 30,
                log=print):
    import time
    from .order_model import OrderModel, record_prefix_counts
    t0 = time.time()
    g = rmat_graph(TRAIN_SCALE)
    dg = DeviceGraph(g)
    kept = [{"seed": s, "k": learned_k(s)} for s in range(TRAIN_FIRST_SEED,
                                                            TRAIN_FIRST_SEED + n_train)]
    dropped = 0
    qs = [learned_query(g, r["seed"]) for r in kept]
    (sq, sm, st), records = record_prefix_counts(dg, qs, n_random, TRAIN_BUDGET, seed=7)
    censored = sum(1 for r in records if r[2] == 2 ** 64 - 1)
    log(f"samples {len(sq)} from {len(records)} runs, {censored} over budget "
        f"({time.time() - t0:.1f}s)")
    val = (sq % 10) == 9  # 90/10 split by query: validation loss
    model = OrderModel.create(seed=0)
    _, l0, _ = model.grad(dg, qs, sq[~val], sm[~val], st[~val])
    model.train(dg, qs, sq[~val], sm[~val], st[~val], epochs=epochs, batch=512, lr=2e-3, seed=1)
    _, ltr, _ = model.grad(dg, qs, sq[~val], sm[~val], st[~val])
    _, lval, _ = model.grad(dg, qs, sq[val], sm[val], st[val])
    log(f"loss: init {l0:.3f} train {ltr:.3f} validation {lval:.3f} ({time.time() - t0:.1f}s)")
    os.makedirs(os.path.join(outdir, "order_model"), exist_ok=True)
    model.save(os.path.join(outdir, "order_model") + "/")
    finished = sorted({r[0] for r in records if r[2] != 2 ** 64 - 1})
    rec = {"graph": f"rmat scale {TRAIN_SCALE} (workloads.rmat_graph)", "budget": TRAIN_BUDGET,
           "first_seed": TRAIN_FIRST_SEED, "n_queries": len(kept),
           "queries_with_a_finished_run": len(finished), "dropped": dropped,
           "runs": len(records),
           "censored_runs": censored, "samples": int(len(sq)), "epochs": epochs,
           "loss_init": l0, "loss_train": ltr, "loss_validation": lval,
           "seconds": time.time() - t0}
    with open(os.path.join(outdir, "order_train_record.json"), "w") as f:
        json.dump(rec, f)
    return rec


HELDOUT_SEEDS = os.path.join(HERE, "data", "heldout_seeds.json")
SELECT_BUDGET = 1 << 24
SELECT_ORDERS = 3


def selection_orders(q, seed: int):
    """SELECT_ORDERS random connected orders of a query, seeded by the query's
    own seed only: they depend on neither the reference nor a learned order."""
    from .order_model import random_connected_order
    rng = np.random.default_rng([seed, 0x5E1EC7])
    return [random_connected_order(q, rng) for _ in range(SELECT_ORDERS)]


def select_heldout(dg: DeviceGraph, g, first_seed: int = EVAL_FIRST_SEED,
                   budget: int = SELECT_BUDGET, max_seeds: int = 1 << 17,
                   max_seconds: float | None = None, chunk: int = 1024, log=None):
    """Held-out queries (k 6..10, seeds from first_seed, taken in order) that
    some order can count: a seed is kept when at least one of its
    SELECT_ORDERS seeded random connected orders finishes within `budget`
    candidate elements.  The criterion depends on neither order under test;
    element counts are exact, so for a given number of scanned seeds the
    selection is deterministic.  Every finished order of a query must give the
    same count, which is recorded."""
    import time
    from .order_model import UNKNOWN
    t0 = time.time()
    kept, s = [], first_seed
    while s - first_seed < max_seeds:
        if max_seconds and time.time() - t0 > max_seconds:
            break
        seeds = list(range(s, s + chunk))
        qs = [learned_query(g, x) for x in seeds]
        jobs = [(i, o) for i, q in enumerate(qs) for o in selection_orders(q, seeds[i])]
        counts, rows, _ = dg.batch_count_orders([qs[i] for i, _ in jobs], [o for _, o in jobs],
                                                max_elements=budget)
        for i, q in enumerate(qs):
            fin = [j for j in range(i * SELECT_ORDERS, (i + 1) * SELECT_ORDERS)
                   if counts[j] != UNKNOWN]
            if not fin:
                continue
            cs = {int(counts[j]) for j in fin}
            assert len(cs) == 1, (seeds[i], cs)
            work = min(int(rows[j][1:q.n].sum()) for j in fin)
            kept.append({"seed": seeds[i], "k": q.n, "count": cs.pop(), "best_random_prefixes": work})
        s += chunk
        if log:
            log(f"scanned {s - first_seed} seeds, kept {len(kept)} ({time.time() - t0:.0f} s)")
    return {"graph": "rmat scale 22 (workloads.rmat_graph)", "first_seed": first_seed,
            "seeds_scanned": s - first_seed, "budget_elements": budget,
            "orders_per_seed": SELECT_ORDERS,
            "criterion": "some seeded random connected order finishes within the budget",
            "queries": kept}


def heldout_split(rec):
    """Kept queries alternate between the held-out test set (even positions)
    and the validation set used for model selection (odd positions)."""
    qs = rec["queries"]
    return qs[0::2], qs[1::2]


def order_summary(rows, budget: int, plan_ms: float) -> dict:
    """Medians of the learned-over-reference speed-up of compare_orders rows
    (see there for the censoring rule)."""
    # A censored run reports no time, so a censored order is charged the
    # budget at the finished order's measured elements per ms.
    sp, sp_plan, el = [], [], []
    n_both = n_lrn = n_ref = n_none = 0
    for row in rows:
        a, b = row["done_ref"], row["done_learned"]
        if a and b:
            n_both += 1
            sp.append(row["ms_ref"] / row["ms_learned"])
            sp_plan.append(row["ms_ref"] / (row["ms_learned"] + plan_ms))
            el.append(row["elements_ref"] / max(1, row["elements_learned"]))
        elif b:
            n_lrn += 1
            rate = row["elements_learned"] / max(row["ms_learned"], 1e-6)
            lb = budget / rate
            sp.append(lb / row["ms_learned"])
            sp_plan.append(lb / (row["ms_learned"] + plan_ms))
        elif a:
            n_ref += 1
            rate = row["elements_ref"] / max(row["ms_ref"], 1e-6)
            ub = budget / rate
            sp.append(row["ms_ref"] / ub)
            sp_plan.append(row["ms_ref"] / (ub + plan_ms))
        else:
            n_none += 1
    med = lambda v: float(np.median(v)) if v else None  # noqa: E731
    geo = lambda v: float(np.exp(np.mean(np.log(v)))) if v else None  # noqa: E731
    summary = {"n": len(rows), "budget_elements": budget, "finished_both": n_both,
               "finished_learned_only": n_lrn, "finished_reference_only": n_ref,
               "finished_neither": n_none,
               "median_speedup_device": med(sp),
               "median_speedup_with_planning": med(sp_plan),
               "geomean_speedup_device": geo(sp),
               "median_speedup_device_both_finished": med(
                   [row["ms_ref"] / row["ms_learned"] for row in rows
                    if row["done_ref"] and row["done_learned"]]),
               "median_element_ratio_both_finished": med(el),
               "planning_ms_per_query": plan_ms,
               "censoring": "an order past the budget is charged the budget at the other "
                            "order's measured elements per ms (an estimate, not a time)"}
    return summary


def compare_orders(dg: DeviceGraph, g, recs, model, budget: int = EVAL_BUDGET):
    """Learned against reference order on the queries of `recs` (selection
    records with seed and count): both orders planned for the whole set in one
    call each (the learned one through one inference launch: its time is the
    planning cost), every query counted under both with the same element
    budget, and counts checked against the recorded ones.  An order past the
    budget is censored: a censored reference against a finished learned order
    is a win, the reverse a loss, and queries censored under both are left out of the medians.  A censored run
    reports no time, so its time is estimated as the budget at the finished
    order's measured elements per ms."""
    import time
    qs = [learned_query(g, r["seed"]) for r in recs]
    ref_orders = dg.plan_orders(qs, order="reference")
    t0 = time.perf_counter()
    lrn_orders = dg.plan_orders(qs, order="learned", model=model)
    plan_ms = 1e3 * (time.perf_counter() - t0) / max(1, len(qs))
    rows = []
    for r, q, ro, lo in zip(recs, qs, ref_orders, lrn_orders):
        row = {"seed": r["seed"], "k": q.n, "count": r["count"], "order_ref": ro,
               "order_learned": lo}
        for name, od in (("ref", ro), ("learned", lo)):
            try:
                c, st = dg.count(q, stats=True, given_order=od, max_elements=budget)
                assert c == r["count"], (r["seed"], name, c, r["count"])
                row[f"ms_{name}"] = st["device_ms"]
                row[f"elements_{name}"] = st["elements"]
                row[f"done_{name}"] = True
            except L.MGError as e:
                if e.code != L.MG_E_LIMIT:
                    raise
                row[f"ms_{name}"] = None
                row[f"done_{name}"] = False
        rows.append(row)
    return order_summary(rows, budget, plan_ms), rows


def c4_pipeline(outdir: str, n_train: int = 6000, select_seconds: float = 300.0, log=print):
    """Configuration C4 end to end on one GPU: held-out selection on the
    scale-22 graph, training of a new network on the scale-20 graph, model
    selection between the committed and the new network on the validation
    half (median device speed-up), and the held-out test comparison of the
    chosen one.  Writes heldout_seeds.json, order_model_new/,
    order_train_record_new.json and order_eval.json into outdir."""
    import time
    from .order_model import OrderModel
    t0 = time.time()
    g = rmat_graph(22)
    dg = DeviceGraph(g)
    rec = select_heldout(dg, g, max_seconds=select_seconds, log=log)
    with open(os.path.join(outdir, "heldout_seeds.json"), "w") as f:
        json.dump(rec, f)
    test, val = heldout_split(rec)
    log(f"held-out: {len(rec['queries'])} kept of {rec['seeds_scanned']} "
        f"({time.time() - t0:.0f} s)")
    dg.free()
    tr = train_order(os.path.join(outdir, "new"), n_train=n_train, log=log)
    log(f"trained ({time.time() - t0:.0f} s): {json.dumps(tr)}")
    dg = DeviceGraph(g)
    cands = {"committed": MODEL_DIR, "new": os.path.join(outdir, "new", "order_model") + "/"}
    val_res = {}
    for name, path in cands.items():
        m = OrderModel.load(path)
        sm, _ = compare_orders(dg, g, val, m)
        m.free()
        val_res[name] = sm
        log(f"validation {name}: {json.dumps(sm)}")
    pick = max(val_res, key=lambda n: val_res[n]["median_speedup_device"] or 0.0)
    m = OrderModel.load(cands[pick])
    summary, rows = compare_orders(dg, g, test, m)
    m.free()
    summary["model"] = pick
    summary["validation"] = val_res
    summary["seconds"] = time.time() - t0
    log(f"test ({pick}): {json.dumps(summary)}")
    with open(os.path.join(outdir, "order_eval.json"), "w") as f:
        json.dump({"summary": summary, "rows": rows}, f)
    dg.free()
    return summary


def eval_batch(model_dir: str, out_path: str, log=print):
    """The committed 4,096-query batch: plain per-query heuristic-order form
    against the batched forms (reference and learned orders)."""
    import time
    from .order_model import OrderModel
    g = rmat_graph(22)
    dg = DeviceGraph(g)
    model = OrderModel.load(model_dir)
    qs, rec = batch_queries(g)
    res = {"n": len(qs)}
    for _ in range(2):  # second pass is the measured one (warm)
        t = time.perf_counter()
        dev, counts = 0.0, []
        for q in qs:
            c, st = dg.count(q, stats=True)
            dev += st["device_ms"]
            counts.append(int(c))
        res["per_query_reference"] = {"wall_s": time.perf_counter() - t, "device_s": dev / 1e3}
        assert counts == rec["counts"]
    for order in ("reference", "learned"):
        for _ in range(2):
            t = time.perf_counter()
            c, st = dg.batch_count(qs, stats=True, order=order, model=model)
            wall = time.perf_counter() - t
        assert c.tolist() == rec["counts"]
        res[f"batch_{order}"] = {"wall_s": wall, "device_s": st["device_ms"] / 1e3,
                                 "launches": st["launches"], "chunks": st["chunks"]}
    for _ in range(2):
        t = time.perf_counter()
        dev = 0.0
        for q in qs:
            c, st = dg.count(q, stats=True, order="learned", model=model)
            dev += st["device_ms"]
        res["per_query_learned"] = {"wall_s": time.perf_counter() - t, "device_s": dev / 1e3}
    base = res["per_query_reference"]["wall_s"]
    res["per_query_reference"]["queries_per_s"] = len(qs) / base
    for key in ("batch_reference", "batch_learned", "per_query_learned"):
        res[key]["speedup_vs_per_query_reference"] = base / res[key]["wall_s"]
        res[key]["queries_per_s"] = len(qs) / res[key]["wall_s"]
    log(json.dumps(res))
    with open(out_path, "w") as f:
        json.dump(res, f)
    return res


def main(argv):
    if len(argv) >= 2 and argv[0] == "train-order":
        train_order(argv[1], n_train=int(argv[2]) if len(argv) > 2 else 8000)
        return 0
    if len(argv) >= 2 and argv[0] == "c4":
        c4_pipeline(argv[1], n_train=int(argv[2]) if len(argv) > 2 else 6000,
                    log=lambda m: print(m, flush=True))
        return 0
    if len(argv) >= 3 and argv[0] == "eval-batch":
        eval_batch(argv[1], argv[2])
        return 0
    if len(argv) >= 2 and argv[0] == "select-batch":
        g = rmat_graph(22)
        dg = DeviceGraph(g)
        rec = select_batch(dg, g, log=lambda m: print(m, flush=True))
        with open(argv[1], "w") as f:
            json.dump(rec, f)
        print(f"kept {len(rec['seeds'])}, dropped {len(rec['dropped'])}, "
              f"elements {sum(rec['elements'])}", flush=True)
        return 0
    print(__doc__)
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
