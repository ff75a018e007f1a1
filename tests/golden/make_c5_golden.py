"""Writes tests/golden/c5_samples.json: oracle counts of small level-0 samples
of the first C5 queries (R-MAT scale 26, 64 Zipf(1.2) labels, 6-8-vertex
queries), computed on the CPU by the oracle over the graph built by the
oracle's own generator (oracle/gen.c, pinned bit-exact against the product
generator by tests/test_oracle_generators.py).  bench.py counts the same
samples on the GPU and requires equal counts (and equal sorted rows, through
their SHA-256, where the sample has at most 20,000 matches).

Where tests/golden/c5_roots.json (written on a GPU by scan_c5_roots.py, which
only chooses positions) lists roots of a query with 1 to 10^6 matches, the
sample is the single root among them with the most matches that the oracle
counts within 10 s; the oracle's count is the expected value.  Otherwise
the sample is the low-degree end of the query's level-0 bucket,
[nb - r, nb), with r the largest power of two (up to 2^16) whose oracle count
stays at or below 10^6 and finishes within 10 s.  When that sample has no
match, systematic samples over the bucket past its first 1% (positions
nb/100, nb/100 + s, ... for s = nb/8, nb/16, ... down to nb/4096) are tried
and the first with a match under the same limits is kept.  Each attempt runs
in a forked child that is killed at 30 s (a vertex near a hub can take the
oracle minutes).  Needs about 40 GB of host memory; several minutes on 8
cores.

    python tests/golden/make_c5_golden.py [n_queries]
"""
import hashlib
import json
import os
import select
import signal
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from matrixgraph_b200.workloads import (C5_FIRST_SEED, C5_LABELS, C5_SCALE,  # noqa: E402
                                        C5_ZIPF, c5_shape)


def timed(fn, limit):
    """fn() in a forked child, killed after `limit` seconds; its JSON result or None."""
    rfd, wfd = os.pipe()
    pid = os.fork()
    if pid == 0:
        try:
            os.close(rfd)
            os.write(wfd, json.dumps(fn()).encode())
        finally:
            os._exit(0)
    os.close(wfd)
    deadline = time.monotonic() + limit
    data, eof = b"", False
    while not eof:
        left = deadline - time.monotonic()
        if left <= 0:
            break
        ready, _, _ = select.select([rfd], [], [], left)
        if ready:
            chunk = os.read(rfd, 1 << 16)
            eof = not chunk
            data += chunk
    if not eof:
        os.kill(pid, signal.SIGKILL)
    os.waitpid(pid, 0)
    os.close(rfd)
    return json.loads(data.decode()) if eof and data else None


def main():
    nq = int(sys.argv[1]) if len(sys.argv) > 1 else 16
    threads = os.cpu_count() or 1
    t0 = time.time()
    g = O.rmat(C5_SCALE, 16, 0.57, 0.19, 0.19, seed=0, n_labels=C5_LABELS, label_kind="zipf",
               zipf_s=C5_ZIPF, label_seed=1, threads=threads)
    print(f"graph {g.n} vertices {g.m} entries in {time.time() - t0:.0f} s", flush=True)
    og = g.oracle_graph()
    print(f"oracle graph built at {time.time() - t0:.0f} s", flush=True)
    out = {"graph": f"R-MAT scale {C5_SCALE}, edge factor 16, a=0.57 b=0.19 c=0.19, seed 0, "
                    f"symmetrised, {C5_LABELS} Zipf({C5_ZIPF}) labels (seed 1)",
           "n": g.n, "m": g.m, "queries": []}
    roots = {}
    try:
        with open(os.path.join(HERE, "c5_roots.json")) as f:
            roots = {r["q"]: r for r in json.load(f)["queries"]}
    except OSError:
        pass
    for q in range(nq):
        k, edges = c5_shape(q)
        labels = O.walk_labels(g, k, edges, C5_FIRST_SEED + q)
        oq = O.query_from_edges(k, edges, labels)
        order = O.reference_order(oq)
        nb = O.bucket_size(og, oq, order)
        best = None
        for cand in sorted(roots.get(q, {}).get("roots", []), key=lambda x: -x["count"])[:8]:
            rr = (cand["pos"], cand["pos"] + 1)
            t1 = time.perf_counter()
            res = timed(lambda: O.count(og, oq, order=order, threads=threads,
                                        root_range=rr), 30)
            dt = time.perf_counter() - t1
            if res is not None and 0 < res["count"] <= 10 ** 6 and dt <= 10:
                best = {"begin": rr[0], "end": rr[1], "step": 1, "count": res["count"],
                        "level_rows": res["level_rows"], "oracle_seconds": dt}
                break
        r = 1
        while best is None and r <= min(nb, 1 << 16):
            rr = (nb - r, nb)
            t1 = time.perf_counter()
            res = timed(lambda: O.count(og, oq, order=order, threads=threads,
                                        root_range=rr), 30)
            dt = time.perf_counter() - t1
            if res is None or res["count"] > 10 ** 6:
                break
            best = {"begin": rr[0], "end": rr[1], "step": 1, "count": res["count"],
                    "level_rows": res["level_rows"], "oracle_seconds": dt}
            if dt > 10:
                break
            r *= 2
        if best is None or best["count"] == 0:
            j = 3
            while nb >> j >= 1 and j <= 12:
                b, st = nb // 100, max(1, nb >> j)
                t1 = time.perf_counter()
                res = timed(lambda: O.count(og, oq, order=order, threads=threads,
                                            root_range=(b, nb), root_step=st), 30)
                dt = time.perf_counter() - t1
                if res is None or res["count"] > 10 ** 6:
                    break
                if res["count"] > 0:
                    best = {"begin": b, "end": nb, "step": st, "count": res["count"],
                            "level_rows": res["level_rows"], "oracle_seconds": dt}
                    break
                j += 1
        rec = {"q": q, "k": k, "edges": edges, "labels": labels, "order": order, "bucket": nb}
        if best is not None:
            rec.update(best)
            if best["count"] <= 20000:
                rows = O.emit(og, oq, order=order, cap=best["count"],
                              root_range=(best["begin"], best["end"]), root_step=best["step"])
                rec["rows_sha256"] = hashlib.sha256(
                    np.ascontiguousarray(rows, dtype="<u4").tobytes()).hexdigest()
        out["queries"].append(rec)
        print(json.dumps(rec), flush=True)
    with open(os.path.join(HERE, "c5_samples.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
