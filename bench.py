#!/usr/bin/env python
"""Benchmark: exact embeddings/s of the subgraph-isomorphism hot path on B200.

Workload (one step): the symmetrised R-MAT scale-22 graph (4,194,304 vertices,
edge factor 16, a=0.57 b=0.19 c=0.19, self-loops and duplicates removed,
32 Zipf(s=1.0) labels) resident in HBM; five labelled queries (triangle,
4-cycle, 4-clique, 5-path, tailed triangle, labels from random walks on the
data graph) counted exactly, one query per launch sequence, reference
heuristic order.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

Under torchrun (N > 1) every rank holds a replica of the graph and counts
every N-th level-0 candidate of each query (positions rank, rank + N, ...:
the hub roots at the head of a bucket spread evenly over the ranks); counts
are summed with one all-reduce after the timed region and the step time is
the maximum over ranks.

The CPU side (``--impl reference``, and the ``cpu_baseline`` / ``same_work``
fields of this arm) runs the oracle — the exact CPU port of the reference's
matching rule, all host threads — on a fixed sample of each query's level-0
candidates (SAMPLE below).  The reference arm builds the same graph and
queries with the oracle's own generator (oracle/gen.c) and never loads the
product library.  This arm counts the identical sample on the GPU and
requires the counts to be equal.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
_T0 = time.perf_counter()
sys.path.insert(0, ROOT)

# Query shapes (undirected edge lists over k vertices); query i is labelled by
# a random walk with seed 2 + i.
SHAPES = {
    "triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "4-cycle": (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
    "4-clique": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]),
    "5-path": (5, [(0, 1), (1, 2), (2, 3), (3, 4)]),
    "tailed-triangle": (4, [(0, 1), (1, 2), (2, 0), (2, 3)]),
}
SHAPE_SEED = 2

# CPU sample of each query's level-0 candidates, as bucket positions
# begin, begin + step, ... (the bucket lists a label's vertices by ascending
# id; R-MAT ids are not permuted, so the head of a bucket holds the hubs).
# The three cheap queries are counted over the whole bucket; the 4-cycle and
# the 5-path over a systematic sample sized so the oracle takes seconds, not
# minutes (a single hub root of the 5-path takes minutes on the CPU).
SAMPLE = {
    "triangle": (0, 1),
    "4-cycle": (1, 8),
    "4-clique": (0, 1),
    "5-path": (32345, 2048),
    "tailed-triangle": (0, 1),
}


def _log(stage: str) -> None:
    """Stage timestamps on stderr (stdout carries only the JSON line)."""
    print(f"[bench +{time.perf_counter() - _T0:7.1f}s] {stage}", file=sys.stderr, flush=True)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--queries", default="",
                   help="comma-separated subset of the query shapes (profiling runs)")
    p.add_argument("--no-gar", action="store_true", help="skip the GAR match timing")
    p.add_argument("--no-batch", action="store_true",
                   help="skip the batched-workload measurement")
    p.add_argument("--hub-bytes", type=int, default=None,
                   help="hub-bitmap budget of the upload (profiling runs; default: library)")
    p.add_argument("--only-c5", action="store_true",
                   help="run only the C5 block and print its record (for profiling)")
    p.add_argument("--c5", type=int, default=8,
                   help="C5 (R-MAT scale 26) queries counted after the headline (0: skip)")
    return p.parse_args()


def shapes(only=""):
    keep = [x for x in only.split(",") if x]
    return [(i, s) for i, s in enumerate(SHAPES) if not keep or s in keep]


def config(scale, n, m, only=""):
    names = [s for _, s in shapes(only)]
    return {"workload": f"R-MAT scale {scale} ({n:,} vertices, edge factor 16, a=0.57 b=0.19 "
                        f"c=0.19, symmetrised, no self-loops/duplicates, {m:,} directed "
                        f"entries), 32 Zipf(s=1.0) labels; {len(names)} random-walk-labelled "
                        f"queries ({', '.join(names)}); one query per launch sequence, "
                        "reference heuristic order, count mode",
            "queries": names, "order": "reference", "mode": "count",
            "l2": "inputs larger than L2 (graph + indices > 1 GB) and a 256 MiB L2 flush "
                  "before every step"}


# DRAM bytes (read + write) per expand-kernel launch of this workload, from
# the one-pass ncu launch list summarised in
# profiles/launches_rmat22_5queries_traffic.md (mean over the expand launches
# of one step).
EXPAND_TRAFFIC_BYTES = 233_955_702


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}",
                                       f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 9 and t[1].replace(".", "").isdigit():
                    rows.append(t)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": sorted(reasons)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


# ---- CPU side: the oracle on the sample --------------------------------------------
def oracle_sample(og, oqs, names, threads):
    """Oracle count of each query over its SAMPLE positions (one pass).
    Returns [(name, begin, step, bucket, count, seconds)]."""
    import oracle as O
    out = []
    for name, oq in zip(names, oqs):
        order = O.reference_order(oq)
        nb = O.bucket_size(og, oq, order)
        b, s = SAMPLE[name]
        t0 = time.perf_counter()
        c = O.count(og, oq, order=order, threads=threads, root_range=(b, nb),
                    root_step=s)["count"]
        out.append((name, b, s, nb, c, time.perf_counter() - t0))
    return out


def sample_text(rows):
    return "; ".join(f"{name}: positions {b}, {b}+{s}, ... of {nb} "
                     f"({(nb - b + s - 1) // s if nb > b else 0} roots)"
                     for name, b, s, nb, _, _ in rows)


SAMPLE_DOC = ("oracle (exact CPU port of the reference matching rule, all host threads) over "
              "level-0 candidate positions begin, begin + step, ... of each query's label "
              "bucket (whole bucket when step = 1): ")


def run_reference(args):
    """The CPU reference arm: the oracle over the sample, on the box's host
    cores; workload built by the oracle's own generator (no product code)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O
    threads = os.cpu_count() or 1
    g = O.rmat(args.scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=32, label_kind="zipf",
               zipf_s=1.0, label_seed=1, threads=threads)
    sel = shapes(args.queries)
    names = [s for _, s in sel]
    oqs = []
    for i, name in sel:
        k, e = SHAPES[name]
        oqs.append(O.query_from_edges(k, e, O.walk_labels(g, k, e, SHAPE_SEED + i)))
    og = g.oracle_graph()
    _log("reference workload built")
    rows = None
    for _ in range(args.warmup):
        rows = oracle_sample(og, oqs, names, threads)
    times, counts = [], 0
    for _ in range(args.steps):
        rows = oracle_sample(og, oqs, names, threads)
        times.append(sum(r[5] for r in rows))
        counts = sum(r[4] for r in rows)
    ms = 1e3 * statistics.mean(times)
    value = counts / (ms / 1e3) if ms > 0 else 0.0
    sample = SAMPLE_DOC + sample_text(rows)
    line = {"impl": "reference", "metric": "exact embeddings/s", "value": value,
            "unit": "embeddings/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config(args.scale, g.n, g.m, args.queries),
            "cpu_baseline": {"value": value, "unit": "embeddings/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "embeddings/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "sample_counts": {r[0]: r[4] for r in rows}}
    print(json.dumps(line), flush=True)


# ---- GPU side --------------------------------------------------------------------
def workload(scale, only=""):
    import matrixgraph_b200 as mg
    g = mg.rmat(scale, 16, 0.57, 0.19, 0.19, seed=0, n_labels=32, label_kind="zipf",
                zipf_s=1.0, label_seed=1)
    qs = [mg.query_walk(g, SHAPES[s], seed=SHAPE_SEED + i) for i, s in shapes(only)]
    return g, qs


def same_work(dg, qs, names, cpu_rows, device, e2e_graph):
    """The GPU on exactly the oracle's sampled roots: counts (asserted equal),
    device time (CUDA events inside the library) and end-to-end time through
    the C-ABI from host buffers (upload + counts)."""
    import matrixgraph_b200 as mg
    import torch
    ref = {r[0]: r for r in cpu_rows}
    gpu_counts, dev_ms = [], 0.0
    for _ in range(2):  # second pass timed (first one warms the handle)
        gpu_counts, dev_ms = [], 0.0
        for name, q in zip(names, qs):
            _, b, s, nb, _, _ = ref[name]
            c, st = dg.count(q, stats=True, root_range=(b, nb), root_step=s)
            gpu_counts.append(c)
            dev_ms += st["device_ms"]
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    dg2 = mg.DeviceGraph(e2e_graph, device)
    for name, q in zip(names, qs):
        _, b, s, nb, _, _ = ref[name]
        dg2.count(q, root_range=(b, nb), root_step=s)
    dg2.free()
    e2e_s = time.perf_counter() - t0
    cpu_counts = [ref[n][4] for n in names]
    cpu_s = sum(ref[n][5] for n in names)
    equal = gpu_counts == cpu_counts
    return {"sample": SAMPLE_DOC + sample_text([ref[n] for n in names]),
            "oracle_counts": cpu_counts, "gpu_counts": gpu_counts, "equal": equal,
            "cpu_seconds": cpu_s, "gpu_device_seconds": dev_ms / 1e3,
            "gpu_e2e_seconds": e2e_s,
            "speedup_device": cpu_s / (dev_ms / 1e3) if dev_ms > 0 else None,
            "speedup_e2e": cpu_s / e2e_s if e2e_s > 0 else None}


def c3_oracle_sample(g, og, every=32, max_elements=10 ** 7, max_count=10 ** 8):
    """Oracle counts of a systematic sample of the 4,096-query batch: every
    `every`-th query among those whose reference order expands at most
    `max_elements` candidates and whose recorded count is at most `max_count`
    (the oracle enumerates every match, so the count bounds its time).
    Returns {index: count}."""
    import oracle as O
    from matrixgraph_b200 import workloads as W
    qs, rec = W.batch_queries(g)
    picked = [i for i in range(0, len(qs), every)
              if rec["elements"][i] <= max_elements and rec["counts"][i] <= max_count]
    threads = os.cpu_count() or 1
    return {i: O.count(og, O.query_from_csr(qs[i]), threads=threads)["count"] for i in picked}


def c1_inputs():
    """Configuration C1: Chung-Lu (10,000 vertices, exponent 2.5, mean degree
    10, seed 0, 8 uniform labels, seed 1) and a 4-cycle with labels uniform
    over the 8 (seed 2)."""
    import matrixgraph_b200 as mg
    g = mg.chung_lu()
    q = mg.CSRGraph.query(4, SHAPES["4-cycle"][1], mg.gen_labels(4, 8, "uniform", seed=2))
    return g, q


def c1_oracle_run(threads):
    """The oracle's count and sorted rows of C1 (CPU leg, timed)."""
    import oracle as O
    g, q = c1_inputs()
    og, oq = O.Graph.from_csr(g), O.query_from_csr(q)
    t0 = time.perf_counter()
    c = O.count(og, oq, threads=threads)["count"]
    t1 = time.perf_counter()
    rows = O.emit(og, oq)
    return {"count": c, "rows": rows, "count_s": t1 - t0, "emit_s": time.perf_counter() - t1,
            "threads": threads}


def c1_workload(device, oracle_res):
    """C1 on the GPU: upload, count and emit (device time of each from the
    library's events, median of 5 after a warm-up), compared with the
    oracle's count and sorted rows."""
    import numpy as np

    import matrixgraph_b200 as mg
    g, q = c1_inputs()
    dg = mg.DeviceGraph(g, device)
    cnt_ms, emit_ms = [], []
    for _ in range(6):
        c, st = dg.count(q, stats=True)
        cnt_ms.append(st["device_ms"])
        rows, _, st2 = dg.emit(q, stats=True)
        emit_ms.append(st2["device_ms"])
    dg.free()
    out = {"workload": "Chung-Lu n=10,000 (exponent 2.5, mean degree 10, 8 uniform labels), "
                       "labelled 4-cycle; count and sorted emit",
           "count": int(c), "rows": int(len(rows)),
           "gpu_count_ms": statistics.median(cnt_ms[1:]),
           "gpu_emit_ms": statistics.median(emit_ms[1:])}
    if oracle_res is not None:
        out.update({"oracle_count": oracle_res["count"],
                    "equal": int(c) == oracle_res["count"] and
                    np.array_equal(rows, oracle_res["rows"]),
                    "cpu_count_s": oracle_res["count_s"], "cpu_emit_s": oracle_res["emit_s"],
                    "cpu_threads": oracle_res["threads"]})
    return out


def batched_workload(g, dg, oracle_counts=None):
    """The 4,096-query batch on the same resident graph: the per-query
    heuristic-order form (one call per query) against batched calls — the
    lane pipeline (every query a fixed launch sequence with device-side sizes
    on 8 concurrent streams, one host wait per batch) with the reference and
    with learned orders (planning included) — wall clock.  Every form's counts
    equal the per-query counts, and a systematic sample equals the oracle."""
    from matrixgraph_b200 import workloads as W
    from matrixgraph_b200.order_model import OrderModel
    qs, rec = W.batch_queries(g)
    model = OrderModel.load(W.MODEL_DIR)
    out = {"workload": f"{len(qs)} random connected queries (k 3-8, p_extra 0.3, random-walk "
                       "labels; seeds kept when the reference order needs <= 2^28 elements, "
                       "matrixgraph_b200/data/batch_seeds.json), count mode"}
    ref_counts = None
    for name, fn in (("per_query_reference", lambda: [dg.count(q) for q in qs]),
                     ("batch_reference", lambda: dg.batch_count(qs).tolist()),
                     ("batch_learned", lambda: dg.batch_count(qs, order="learned",
                                                              model=model).tolist())):
        fn()  # warm-up
        t0 = time.perf_counter()
        counts = [int(c) for c in fn()]
        wall = time.perf_counter() - t0
        if ref_counts is None:
            ref_counts = counts
        assert counts == ref_counts, name
        out[name] = {"seconds": wall, "queries_per_s": len(qs) / wall}
        _log(f"batched {name}: {wall:.2f} s")
    t0 = time.perf_counter()
    dg.plan_orders(qs, order="learned", model=model)
    out["batch_learned"]["planning_seconds"] = time.perf_counter() - t0
    base = out["per_query_reference"]["seconds"]
    for name in ("batch_reference", "batch_learned"):
        out[name]["speedup_vs_per_query_reference"] = base / out[name]["seconds"]
    out["counts_equal_recorded"] = ref_counts == rec["counts"]
    if oracle_counts:
        out["oracle_sample"] = {"queries": sorted(oracle_counts),
                                "equal": all(ref_counts[i] == c for i, c in oracle_counts.items())}
        assert out["oracle_sample"]["equal"], "batch counts differ from the oracle"
    model.free()
    return out


def gar_workload(reps=3):
    """matrixgraph_gar_match end to end (host arrays in, grouped output back,
    graph upload included) on an R-MAT scale-18 multigraph seen as directed
    edges with 8 uniform vertex labels and 4 uniform edge labels: a tailed
    triangle whose edges use three edge labels (subdivided instance) and the
    same shape with one edge label."""
    import numpy as np

    import matrixgraph_b200 as mg
    from matrixgraph_b200.gar import GARGraphArrays, GARPatternArrays, gar_match
    g = mg.rmat(18, 16, 0.57, 0.19, 0.19, seed=0, n_labels=8, label_kind="uniform",
                label_seed=1)
    off = g.array("out_off").astype(np.int64)
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(off))
    dst = g.array("out_edges").astype(np.uint32)
    rng = np.random.default_rng(5)
    ga = GARGraphArrays(v_id=(10 ** 6 + np.arange(g.n)).astype(np.uint32),
                        v_label_idx=g.array("labels").astype(np.int32), e_src=src, e_dst=dst,
                        e_label_idx=rng.integers(0, 4, len(src)).astype(np.int32))
    out = {"workload": f"R-MAT scale 18 ({g.n} vertices, {len(src)} directed edges), 8 vertex "
                       "labels, 4 edge labels; tailed triangle 0->1->2->0, 2->3; "
                       "row capacity 2^20, id capacity 2^24; host arrays in and out"}
    for name, elab in (("three_edge_labels", [0, 1, 0, 2]), ("one_edge_label", [0, 0, 0, 0])):
        pa = GARPatternArrays(node_label_idx=np.array([0, 1, 2, 3], np.int32),
                              edge_src=np.array([0, 1, 2, 2], np.int32),
                              edge_dst=np.array([1, 2, 0, 3], np.int32),
                              edge_label_idx=np.array(elab, np.int32))
        gar_match(ga, pa, 1 << 20, 1 << 24)  # warm-up
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            r = gar_match(ga, pa, 1 << 20, 1 << 24)
            times.append(time.perf_counter() - t0)
        out[name] = {"seconds": statistics.median(times), "matches": r.n_matches,
                     "rows": r.row_size, "ids": r.match_size}
        _log(f"gar {name}: {out[name]['seconds']:.2f} s")
    return out


C5_GOLDEN = os.path.join(ROOT, "tests", "golden", "c5_samples.json")


def c5_workload(n_queries):
    """Configuration C5: R-MAT scale 26 (67,108,864 vertices, ~2.1e9 directed
    entries) with 64 Zipf(1.2) labels, queries of 6-8 vertices (4-clique or
    chorded 5-cycle plus a pendant path).  Their reference-order counts run to
    10^13-10^15 embeddings, so each query is counted over a systematic sample
    of its level-0 candidates: positions s/2, s/2 + s, ... with the smallest
    stride s (from bucket/256 upward by factors of 4) whose enumeration needs
    at most 2^33 candidate elements (element counts are exact, so the sample
    does not depend on timing).  Parity: the GPU counts the fixed low-degree
    samples of tests/golden/c5_samples.json, whose counts (and sorted rows,
    through their SHA-256) the oracle computed on the CPU
    (tests/golden/make_c5_golden.py)."""
    import hashlib

    import numpy as np

    import matrixgraph_b200 as mg
    from matrixgraph_b200 import _lib as L
    from matrixgraph_b200 import workloads as W
    t0 = time.perf_counter()
    g = W.c5_graph()
    gen_s = time.perf_counter() - t0
    dg = mg.DeviceGraph(g, 0)
    upload_s = time.perf_counter() - t0 - gen_s
    info = dg.info
    _log(f"C5 graph generated ({gen_s:.0f} s) and uploaded ({upload_s:.0f} s)")
    qs = W.c5_queries(g, n_queries)
    sizes = np.bincount(g.array("labels"), minlength=W.C5_LABELS)
    out = {"workload": f"R-MAT scale 26 ({g.n:,} vertices, {g.m_out:,} directed entries), 64 "
                       f"Zipf(1.2) labels; first {n_queries} C5 queries (k 6-8), reference "
                       "order, count mode over systematic root samples",
           "gen_seconds": gen_s, "upload_seconds": upload_s,
           "device_bytes": info["device_bytes"], "queries": []}
    budget = 1 << 33
    tot_ms = tot_emb = tot_balgc = 0
    for i, q in enumerate(qs):
        nb = int(sizes[int(q.array("labels")[mg.plan_order(q)[0]])])
        step = max(1, nb // 256)
        rec = None
        while step <= nb:
            try:
                c, st = dg.count(q, stats=True, root_range=(step // 2, nb), root_step=step,
                                 max_elements=budget)
                rec = {"q": i, "k": q.n, "bucket": nb, "begin": step // 2, "step": step,
                       "roots": (nb - step // 2 + step - 1) // step, "count": c,
                       "device_ms": st["device_ms"], "elements": st["elements"],
                       "balg_count_bytes": st["balg_count_bytes"]}
                break
            except L.MGError as e:
                if e.code != L.MG_E_LIMIT:
                    raise
                step *= 4
        if rec is None:
            rec = {"q": i, "k": q.n, "bucket": nb, "over_budget": True}
        else:
            tot_ms += rec["device_ms"]
            tot_emb += rec["count"]
            tot_balgc += rec["balg_count_bytes"]
        out["queries"].append(rec)
    out["embeddings_per_s"] = tot_emb / (tot_ms / 1e3) if tot_ms else None
    out["balg_count_gbs"] = tot_balgc / (tot_ms / 1e3) / 1e9 if tot_ms else None
    out["device_ms"] = tot_ms
    _log("C5 samples counted")
    # parity against the committed oracle counts of fixed low-degree samples
    parity = []
    try:
        with open(C5_GOLDEN) as f:
            gold = json.load(f)
    except OSError:
        gold = {"queries": []}
    for rec in gold["queries"]:
        if "count" not in rec:
            continue
        q = mg.query_walk(g, (rec["k"], [tuple(e) for e in rec["edges"]]),
                          seed=W.C5_FIRST_SEED + rec["q"])
        same_query = q.array("labels").tolist() == rec["labels"]
        rr, rs = (rec["begin"], rec["end"]), rec.get("step", 1)
        c, st = dg.count(q, stats=True, root_range=rr, root_step=rs)
        p = {"q": rec["q"], "roots": (rec["end"] - rec["begin"] + rs - 1) // rs,
             "oracle": rec["count"],
             "gpu": c, "equal": same_query and c == rec["count"] and
             st["level_rows"] == rec["level_rows"]}
        if "rows_sha256" in rec:
            rows = dg.emit(q, root_range=rr, root_step=rs)
            h = hashlib.sha256(np.ascontiguousarray(rows, dtype="<u4").tobytes()).hexdigest()
            p["rows_equal"] = h == rec["rows_sha256"]
        parity.append(p)
    out["parity"] = {"source": "tests/golden/c5_samples.json", "samples": parity,
                     "all_equal": bool(parity) and all(p["equal"] and p.get("rows_equal", True)
                                                       for p in parity)}
    dg.free()
    return out


def heldout_eval(dg, g, n=512):
    """Learned vs reference order on held-out queries (configuration C4): the
    first n queries of the committed held-out test set
    (matrixgraph_b200/data/heldout_seeds.json: random connected, k 6-10, walk
    labels, seeds from 200000 kept when one of three seeded random orders
    counts them within 2^24 candidate elements — a criterion that depends on
    neither order under test; even positions are the test set, odd ones
    chose the model) on the resident scale-22 graph, each counted under both
    orders with the same element budget; counts must equal the recorded
    ones."""
    from matrixgraph_b200 import workloads as W
    from matrixgraph_b200.order_model import OrderModel
    with open(W.HELDOUT_SEEDS) as f:
        rec = json.load(f)
    test, _ = W.heldout_split(rec)
    model = OrderModel.load(W.MODEL_DIR)
    summary, _ = W.compare_orders(dg, g, test[:n], model)
    model.free()
    summary["workload"] = (f"{min(n, len(test))} held-out queries of "
                           "matrixgraph_b200/data/heldout_seeds.json (test half; k 6-10, "
                           "p_extra 0.3, walk labels) on the R-MAT scale-22 graph; budget "
                           f"{summary['budget_elements']} candidate elements per count")
    summary["model"] = "matrixgraph_b200/data/order_model"
    return summary


def run_mine(args):
    import torch

    import matrixgraph_b200 as mg
    if args.only_c5:
        print(json.dumps(c5_workload(args.c5)), flush=True)
        return
    world, rank, local = dist_setup()
    device = local
    t0 = time.perf_counter()
    g, qs = workload(args.scale, args.queries)
    names = [s for _, s in shapes(args.queries)]
    gen_s = time.perf_counter() - t0
    _log("workload generated")
    # The oracle runs before this process initialises CUDA.
    cpu, cpu_rows, c3_oracle, c1_oracle = None, None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O
        threads = os.cpu_count() or 1
        og = O.Graph.from_csr(g)
        oqs = [O.query_from_csr(q) for q in qs]
        cpu_rows = oracle_sample(og, oqs, names, threads)
        if not args.no_batch and args.scale == 22 and not args.queries:
            c3_oracle = c3_oracle_sample(g, og)
        if not args.queries:
            c1_oracle = c1_oracle_run(threads)
        del og
        c, s = sum(r[4] for r in cpu_rows), sum(r[5] for r in cpu_rows)
        cpu = {"value": c / s if s > 0 else 0.0, "unit": "embeddings/s", "cores": threads,
               "kind": "port", "sample": SAMPLE_DOC + sample_text(cpu_rows)}
        _log("cpu baseline done")
    torch.cuda.set_device(device)
    # Level-0 candidates of this rank: positions rank, rank + world, ...
    shard = mg.shard_strided(rank, world)
    dg = mg.DeviceGraph(g, device, hub_bytes=args.hub_bytes)
    info = dg.info
    _log("graph uploaded")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device=f"cuda:{device}")

    def step(collect):
        flush.zero_()
        torch.cuda.synchronize(device)
        per_q, launches, balg, balgc, counts = [], 0, 0, 0, []
        for q in qs:
            c, st = dg.count(q, stats=True, **shard)
            per_q.append(st["device_ms"])
            launches += st["launches"]
            balg += st["balg_bytes"]
            balgc += st["balg_count_bytes"]
            counts.append(c)
        if collect is not None:
            collect.append((sum(per_q), launches, balg, balgc, counts, per_q))

    for _ in range(args.warmup):
        step(None)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    clk = Clocks(device)
    clk.start()
    recs = []
    host0 = time.perf_counter()
    for _ in range(args.steps):
        step(recs)
    torch.cuda.synchronize(device)
    host_ms = 1e3 * (time.perf_counter() - host0) / args.steps
    if world > 1:
        torch.distributed.barrier()
    clocks = clk.stop()
    _log("timed steps done")
    ms_step = statistics.mean(r[0] for r in recs)
    per_query_ms = [statistics.mean(r[5][i] for r in recs) for i in range(len(qs))]
    counts, launches, balg, balgc = recs[-1][4], recs[-1][1], recs[-1][2], recs[-1][3]
    if world > 1:
        t = torch.tensor([ms_step], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(t.item())
        c = torch.tensor(counts + [balgc, balg, launches], dtype=torch.int64,
                         device=f"cuda:{device}")
        torch.distributed.all_reduce(c)
        vals = c.tolist()
        counts, balgc, balg, launches = vals[:len(qs)], vals[-3], vals[-2], vals[-1]
    emb = sum(counts)
    value = emb / (ms_step / 1e3)

    # End to end through the public API from host buffers: upload (graph
    # arrays host -> device, derived indices), the counts, counts back.
    e2e_times = []
    h2d = (g.n + 1) * 4 + g.m_out * 4 + 4 * g.n * 3 + sum(q.n * 4 * 4 + q.m_out * 8 for q in qs)
    d2h = 8 * len(qs)
    e2e_parts = []
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        dg2 = mg.DeviceGraph(g, device)
        t1 = time.perf_counter()
        for q in qs:
            dg2.count(q, **shard)
        t2 = time.perf_counter()
        dg2.free()
        t3 = time.perf_counter()
        e2e_times.append(t3 - t0)
        e2e_parts.append((t1 - t0, t2 - t1, t3 - t2))
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    e2e_split = ({"upload_s": statistics.median(p[0] for p in e2e_parts),
                  "counts_s": statistics.median(p[1] for p in e2e_parts),
                  "free_s": statistics.median(p[2] for p in e2e_parts)} if e2e_parts else None)
    _log("end-to-end runs done")
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())

    # Kernel-timing pass (after the timed region): every expand launch between
    # a CUDA event pair on the library's stream.
    expand_ms, expand_launches = 0.0, 0
    for q in qs:
        _, st = dg.count(q, stats=True, kernel_events=1, **shard)
        expand_ms += st["expand_ms"]
        expand_launches += st["expand_launches"]
    _log("kernel-timing pass done")

    same = None
    if cpu_rows is not None:
        same = same_work(dg, qs, names, cpu_rows, device, g)
        _log(f"same-work check: equal={same['equal']}")

    # Blocks after the headline: an exception is recorded in the line instead
    # of losing it; a failed parity check (AssertionError) also makes the
    # process exit non-zero once the line is printed.
    failures = []

    def guarded(name, fn):
        try:
            return fn()
        except Exception as e:
            _log(f"{name} failed: {e!r}")
            if isinstance(e, AssertionError):
                failures.append(f"{name}: {e!r}")
            return {"error": repr(e)}

    c1 = None
    if world == 1 and not args.queries:
        c1 = guarded("C1", lambda: c1_workload(device, c1_oracle))
        _log(f"C1 done: equal={c1.get('equal')}")

    peak, peak_kind = peaks()
    # The dominant kernel is the expand kernel (over 90% of device time): its
    # algorithmic bytes per launch are the step's B_alg (count-mode
    # definition) over its launches, its duration the event-timed mean.
    per_launch_bytes = balgc / max(1, expand_launches)
    per_launch_s = expand_ms / 1e3 / max(1, expand_launches)
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": EXPAND_TRAFFIC_BYTES,
                "kernel": "k_expand (all launch shapes)",
                "basis": "B_alg (count-mode definition, the merge-intersection byte count) "
                         "per expand launch / CUDA-event mean launch duration; peak "
                         f"{peak_kind} copy bandwidth; traffic = ncu DRAM read+write bytes "
                         "per expand launch of this workload",
                "expand_launches_per_step": expand_launches,
                "expand_ms_per_step": expand_ms,
                "balg_count_bytes_per_step": balgc, "balg_bytes_per_step": balg,
                "step_rate_gbs": balgc / (ms_step / 1e3) / 1e9}
    batch = None
    if world == 1 and not args.no_batch and args.scale == 22 and not args.queries:
        batch = guarded("batched", lambda: batched_workload(g, dg, c3_oracle))
        _log("batched workload done")
    heldout = None
    if world == 1 and not args.no_batch and args.scale == 22 and not args.queries:
        heldout = guarded("held-out", lambda: heldout_eval(dg, g))
        _log("held-out order evaluation done")
    c5 = None
    if world == 1 and args.c5 > 0 and not args.queries:
        dg.free()
        c5 = guarded("C5", lambda: c5_workload(args.c5))
        _log("C5 workload done")
    gar = None
    if world == 1 and not args.no_gar:
        gar = guarded("GAR", gar_workload)
        _log("gar workload done")
    if rank == 0:
        line = {"metric": "exact embeddings/s", "value": value, "unit": "embeddings/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": config(args.scale, g.n, g.m_out, args.queries),
                "queries_per_s": len(qs) / (ms_step / 1e3),
                "counts": counts, "per_query_ms": dict(zip(names, per_query_ms)),
                "host_ms_per_step": host_ms, "roofline": roofline, "cpu_baseline": cpu,
                "same_work": same,
                "e2e": ({"value": emb / e2e_s, "unit": "embeddings/s",
                         "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                         "seconds_per_step": e2e_s, "split": e2e_split}
                        if e2e_times else None),
                "clocks": clocks, "gpu_launches": launches * args.steps,
                "batched": batch, "learned_order_heldout": heldout, "gar_match": gar,
                "c5": c5, "c1": c1,
                "graph": {"n": info["n"], "m_out": info["m_out"],
                          "device_bytes": info["device_bytes"], "max_degree": info["max_degree"],
                          "gen_seconds": gen_s}}
        print(json.dumps(line), flush=True)
    dg.free()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if same is not None and not same["equal"]:
        sys.exit("same-work counts differ from the oracle")
    if c1 is not None and c1.get("equal") is False:
        sys.exit("C1 count or rows differ from the oracle")
    c5_parity = (c5 or {}).get("parity") or {}
    if c5_parity.get("samples") and not c5_parity.get("all_equal"):
        sys.exit("C5 fixture counts or rows differ from the oracle")
    if failures:
        sys.exit("; ".join(failures))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mine(args)


if __name__ == "__main__":
    main()
