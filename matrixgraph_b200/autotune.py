"""Autotuner of the batch launch parameters.

For a resident data graph and a sample of a batch's queries, each query-size
bucket is timed under every candidate setting of

* ``lanes``      concurrent per-query launch pipelines of a batch call,
* ``probe_min``  shortest hub slice probed in the hub bitmap (binary search
                 below it),
* ``grab``       expand tiles a block takes from the work queue at a time,

and the fastest setting is kept.  Results go to a small text table keyed by
the graph's signature and the bucket, read back by :func:`load_table` and by
``subiso_exec -tune <file>``::

    # signature k_lo k_hi lanes probe_min grab seconds
    n4194304.m128315120.L32.d163479 3 4 8 1 0 0.412

Settings never change counts, only time; every trial's counts are checked
against the first.
"""
from __future__ import annotations

import itertools
import os
import time
from typing import Sequence

BUCKETS = ((1, 3), (4, 4), (5, 6), (7, 16))
CANDIDATES = {"lanes": (4, 8, 16), "probe_min": (1, 16, 256), "grab": (0, 16)}


def signature(dg) -> str:
    """Graph signature: vertices, directed entries, labels, maximum degree."""
    i = dg.info
    return f"n{i['n']}.m{i['m_out']}.L{i['n_labels']}.d{i['max_degree']}"


def bucket_of(k: int) -> tuple[int, int]:
    for lo, hi in BUCKETS:
        if lo <= k <= hi:
            return lo, hi
    return BUCKETS[-1]


def tune(dg, queries: Sequence, sample: int = 256, reps: int = 1, candidates=None,
         **count_kw) -> dict:
    """Best setting per size bucket: {(k_lo, k_hi): (settings, seconds)}."""
    cand = dict(CANDIDATES, **(candidates or {}))
    keys = list(cand)
    by_bucket: dict = {}
    for q in queries:
        by_bucket.setdefault(bucket_of(q.n), []).append(q)
    best = {}
    for b, qs in sorted(by_bucket.items()):
        qs = qs[:sample]
        ref = None
        for values in itertools.product(*(cand[k] for k in keys)):
            opts = dict(zip(keys, values))
            dg.batch_count(qs, **opts, **count_kw)  # warm-up
            t = float("inf")
            for _ in range(reps):
                t0 = time.perf_counter()
                counts = dg.batch_count(qs, **opts, **count_kw).tolist()
                t = min(t, time.perf_counter() - t0)
            if ref is None:
                ref = counts
            assert counts == ref, "a launch setting changed a count"
            if b not in best or t < best[b][1]:
                best[b] = (opts, t)
    return best


def save_table(path: str, dg, best: dict) -> None:
    """Writes (or updates) the rows of this graph's signature."""
    sig = signature(dg)
    rows = []
    if os.path.exists(path):
        with open(path) as f:
            rows = [ln for ln in f if ln.strip() and not ln.startswith("#")
                    and ln.split()[0] != sig]
    for (lo, hi), (o, t) in sorted(best.items()):
        rows.append(f"{sig} {lo} {hi} {o['lanes']} {o['probe_min']} {o['grab']} {t:.4f}\n")
    with open(path, "w") as f:
        f.write("# signature k_lo k_hi lanes probe_min grab seconds\n")
        f.writelines(rows)


def load_table(path: str, dg) -> dict:
    """{(k_lo, k_hi): settings} of this graph's signature (empty if none)."""
    sig = signature(dg)
    out = {}
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if len(t) >= 7 and not ln.startswith("#") and t[0] == sig:
                out[(int(t[1]), int(t[2]))] = {"lanes": int(t[3]), "probe_min": int(t[4]),
                                               "grab": int(t[5])}
    return out


def tuned_batch_count(dg, queries: Sequence, table: dict, **count_kw):
    """Counts of a batch, each size bucket run with its tuned setting."""
    import numpy as np
    out = np.zeros(len(queries), dtype=np.uint64)
    groups: dict = {}
    for i, q in enumerate(queries):
        groups.setdefault(bucket_of(q.n), []).append(i)
    for b, idx in groups.items():
        opts = table.get(b, {})
        out[idx] = dg.batch_count([queries[i] for i in idx], **opts, **count_kw)
    return out
