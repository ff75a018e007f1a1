"""The N>1 host path of bench.py on CPU: two gloo ranks shard every query's
level-0 candidates with shard_roots, count their shard (the oracle stands in
for each rank's GPU) and sum with one all-reduce; the sum is the full count."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import matrixgraph_b200 as mg
import oracle as O


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = mg.chung_lu(2000, avg_deg=8, n_labels=4)
    qs = [mg.query_walk(g, s, seed=2 + i) for i, s in enumerate(mg.SHAPES)]
    sizes = mg.level0_sizes(g, qs)
    og = O.Graph.from_csr(g)
    local = []
    for q, n in zip(qs, sizes):
        lo, hi = mg.shard_roots(n, rank, world)
        local.append(O.count(og, O.query_from_csr(q), root_range=(lo, hi))["count"])
    t = torch.tensor(local, dtype=torch.int64)
    dist.all_reduce(t)
    if rank == 0:
        full = [O.count(og, O.query_from_csr(q))["count"] for q in qs]
        np.save(out, np.array([t.tolist(), full], dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_counts_sum_to_full(tmp_path):
    out = str(tmp_path / "r.npy")
    mp.spawn(_rank, args=(2, _port(), out), nprocs=2, join=True)
    summed, full = np.load(out)
    assert summed.tolist() == full.tolist()
    assert sum(full) > 0
