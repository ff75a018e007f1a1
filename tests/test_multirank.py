"""The N>1 host path of bench.py on CPU: two gloo ranks take every second
level-0 candidate of each query (shard_strided), count their shard (the
oracle stands in for each rank's GPU) and sum with one all-reduce; the sum is
the full count, for single queries and for a batch's per-query vector."""
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
    g = mg.rmat(11, 8, n_labels=8)
    qs = [mg.query_walk(g, s, seed=2 + i) for i, s in enumerate(mg.SHAPES)]
    qs += [mg.query_random(g, 3 + i % 3, 0.3, seed=1000 + i) for i in range(8)]
    og = O.Graph.from_csr(g)
    sh = mg.shard_strided(rank, world)
    local = []
    for q in qs:
        b = sh["root_range"][0]
        local.append(O.count(og, O.query_from_csr(q), root_range=(b, 2 ** 63),
                             root_step=sh["root_step"])["count"])
    t = torch.tensor(local, dtype=torch.int64)
    dist.all_reduce(t)  # the one exchange: the per-query count vector
    if rank == 0:
        full = [O.count(og, O.query_from_csr(q))["count"] for q in qs]
        np.save(out, np.array([t.tolist(), full], dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_strided_counts_sum_to_full(tmp_path):
    out = str(tmp_path / "r.npy")
    mp.spawn(_rank, args=(2, _port(), out), nprocs=2, join=True)
    summed, full = np.load(out)
    assert summed.tolist() == full.tolist()
    assert sum(full) > 0


def test_strided_shards_partition_and_balance_a_hub_first_bucket():
    """On an R-MAT bucket (hubs first) contiguous halves give rank 0 most of
    the adjacency volume of the roots; the stride splits it nearly evenly."""
    g = mg.rmat(14, n_labels=4)
    lab = g.array("labels")
    deg = np.diff(g.array("out_off").astype(np.int64))
    bucket = np.flatnonzero(lab == 0)  # ascending ids, as the engine's bucket
    for world in (2, 4, 8):
        parts = [np.arange(len(bucket))[mg.shard_strided(r, world)["root_range"][0]::world]
                 for r in range(world)]
        assert sorted(np.concatenate(parts).tolist()) == list(range(len(bucket)))
        strided = [deg[bucket[p]].sum() for p in parts]
        contiguous = [deg[bucket[lo:hi]].sum() for lo, hi in
                      (mg.shard_roots(len(bucket), r, world) for r in range(world))]
        assert max(strided) / np.mean(strided) < 1.25, (world, strided)
        assert max(contiguous) / np.mean(contiguous) > 1.5, (world, contiguous)
    assert mg.shard_strided(0, 1) == {}


def test_weighted_shards_partition_and_balance_a_hub_first_bucket():
    """Contiguous shards cut from the Σdeg prefix sum partition the bucket and
    balance its adjacency volume, where count-based halves do not."""
    g = mg.rmat(14, n_labels=4)
    q = mg.CSRGraph.query(3, [(0, 1), (1, 2)], [0, 1, 0])
    costs = mg.root_costs(g, q)
    assert len(costs) == int((g.array("labels") == 0).sum())
    for world in (2, 4, 8):
        rng = [mg.shard_roots_weighted(costs, r, world) for r in range(world)]
        assert rng[0][0] == 0 and rng[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(rng, rng[1:]))
        vol = [costs[lo:hi].sum() for lo, hi in rng]
        assert max(vol) / np.mean(vol) < 1.25, (world, vol)
    assert mg.shard_roots_weighted(costs, 0, 1) == (0, len(costs))


def test_batch_shares_partition_and_balance():
    rng = np.random.default_rng(3)
    costs = rng.pareto(1.2, 4096) + 1
    for world in (1, 2, 4, 8):
        parts = [mg.shard_batch(costs, r, world) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        load = [costs[p].sum() for p in parts]
        assert max(load) - min(load) <= costs.max() + 1e-9


def _rank_batch(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = mg.rmat(11, 8, n_labels=8)
    qs = [mg.query_random(g, 3 + i % 4, 0.3, seed=2000 + i) for i in range(16)]
    og = O.Graph.from_csr(g)
    # cost estimate: the level-0 volume of each query (same on every rank)
    costs = [float(mg.root_costs(g, q).sum()) for q in qs]
    local = torch.zeros(len(qs), dtype=torch.int64)
    for i in mg.shard_batch(costs, rank, world):
        local[i] = O.count(og, O.query_from_csr(qs[i]))["count"]
    dist.all_reduce(local)  # the one exchange: the per-query count vector
    # single query over weighted contiguous shards
    q = qs[0]
    lo, hi = mg.shard_roots_weighted(mg.root_costs(g, q), rank, world)
    part = torch.tensor([O.count(og, O.query_from_csr(q), root_range=(lo, hi))["count"]
                         if hi > lo else 0], dtype=torch.int64)
    dist.all_reduce(part)
    if rank == 0:
        full = [O.count(og, O.query_from_csr(x))["count"] for x in qs]
        np.save(out, np.array([local.tolist() + [int(part.item())], full + [full[0]]],
                              dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_batch_and_weighted_shards_sum_to_full(tmp_path):
    out = str(tmp_path / "b.npy")
    mp.spawn(_rank_batch, args=(2, _port(), out), nprocs=2, join=True)
    summed, full = np.load(out)
    assert summed.tolist() == full.tolist()
    assert sum(full) > 0
