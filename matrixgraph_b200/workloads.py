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
    python -m matrixgraph_b200.workloads eval-order MODEL_DIR/ OUT.json [N]
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


def eval_order(model_dir: str, out_path: str, n_eval: int = 2000, log=print,
               select_seconds: float = 150.0):
    """Held-out queries (k 6..10) on the scale-22 graph: reference vs learned."""
    import time
    from .order_model import OrderModel
    t0 = time.time()
    g = rmat_graph(22)
    dg = DeviceGraph(g)
    model = OrderModel.load(model_dir)
    kept, dropped = select_queries(dg, g, learned_query, EVAL_FIRST_SEED, n_eval, EVAL_BUDGET,
                                   12 * n_eval, log, max_seconds=select_seconds)
    log(f"held-out: kept {len(kept)} dropped {dropped} ({time.time() - t0:.1f}s)")
    rows = []
    for r in kept:
        q = learned_query(g, r["seed"])
        c_ref, st_ref = dg.count(q, stats=True)
        t_plan = time.perf_counter()
        lo = dg.plan_order(q, order="learned", model=model)
        t_plan = time.perf_counter() - t_plan
        guard = max(16 * r["elements"], 1 << 24)
        try:
            c_l, st_l = dg.count(q, stats=True, given_order=lo, max_elements=guard)
            ms_l = st_l["device_ms"]
            assert c_l == c_ref, (r["seed"], c_l, c_ref)
        except L.MGError as e:
            if e.code != L.MG_E_LIMIT:
                raise
            ms_l, st_l = float("inf"), None
        try:
            _, st_s = dg.count(q, stats=True, order="strong", max_elements=guard)
            ms_s = st_s["device_ms"]
        except L.MGError as e:
            if e.code != L.MG_E_LIMIT:
                raise
            ms_s = float("inf")
        rows.append({"seed": r["seed"], "k": q.n, "count": int(c_ref),
                     "ms_ref": st_ref["device_ms"], "ms_learned": ms_l, "ms_strong": ms_s,
                     "plan_ms": 1e3 * t_plan, "order_ref": st_ref["order"],
                     "order_learned": lo, "rows_ref": st_ref["level_rows"],
                     "rows_learned": st_l["level_rows"] if st_l else None})
    sp = np.array([x["ms_ref"] / x["ms_learned"] for x in rows])
    sp_wall = np.array([x["ms_ref"] / (x["ms_learned"] + x["plan_ms"]) for x in rows])
    best = np.array([min(x["ms_ref"], x["ms_strong"], x["ms_learned"]) for x in rows])
    regret = np.array([x["ms_learned"] / b for x, b in zip(rows, best)])
    summary = {"n": len(rows), "dropped": dropped, "budget": EVAL_BUDGET,
               "median_speedup_device": float(np.median(sp)) if len(sp) else None,
               "median_speedup_with_planning": float(np.median(sp_wall)) if len(sp) else None,
               "geomean_speedup_device": float(np.exp(np.mean(np.log(sp)))) if len(sp) else None,
               "total_ms_ref": float(sum(x["ms_ref"] for x in rows)),
               "total_ms_learned": float(sum(x["ms_learned"] for x in rows)),
               "total_ms_strong": float(sum(x["ms_strong"] for x in rows)),
               "median_regret": float(np.median(regret)) if len(sp) else None,
               "learned_over_budget": int(sum(1 for x in rows if x["ms_learned"] == float("inf"))),
               "seconds": time.time() - t0}
    log(json.dumps(summary))
    with open(out_path, "w") as f:
        json.dump({"summary": summary, "rows": rows}, f)
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
    if len(argv) >= 3 and argv[0] == "eval-order":
        eval_order(argv[1], argv[2], n_eval=int(argv[3]) if len(argv) > 3 else 2000)
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
