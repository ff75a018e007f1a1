"""Seeded benchmark workloads.

* ``rmat_graph(scale)`` — symmetrised R-MAT (edge factor 16, a=0.57 b=0.19
  c=0.19), self-loops and duplicates removed, ids not permuted, 32 Zipf(1.0)
  labels: the single-query (scale 22) and batched (scale 22) data graph.
* ``shape_queries(g)`` — the five single-query shapes with random-walk labels.
* batched queries — random connected queries, k uniform in 3..8, a random
  recursive spanning tree plus every other pair with probability 0.3,
  random-walk labels.  Some seeds give search spaces far beyond any time
  budget on a scale-22 power-law graph (trees of common labels around hubs),
  so the batch is the first 4,096 seeds (from 1000) whose count under the
  reference order expands at most ``BATCH_BUDGET`` candidate elements.  The
  selection is deterministic (element counts are exact integers) and the kept
  seeds, sizes and counts are committed in ``data/batch_seeds.json``.

    python -m matrixgraph_b200.workloads select-batch OUT.json
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


def main(argv):
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
