"""Learned matching order: Python side of the order model in libmg_subiso.so.

The network (2 message-passing layers, 64 hidden units, CUDA forward/backward
kernels, Adam; BF16 inference) predicts log(1 + P(S)) for connected vertex
sets S of a query; ``MG_ORDER_LEARNED`` then picks the order with the least
predicted work.  Training labels are the per-prefix survivor counts P_i that
the enumerator itself records (``DeviceGraph.batch_count_orders``) for the
reference order and random connected orders of sampled queries.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Sequence

import numpy as np

from . import _lib as L
from .graph import CSRGraph, query_edges
from .subiso import DeviceGraph, plan_order

UNKNOWN = np.uint64(2 ** 64 - 1)


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _qarr(qs):
    return (C.POINTER(L.CsrView) * len(qs))(*[C.pointer(q.view) for q in qs])


class OrderModel:
    def __init__(self, handle: int):
        self.handle = handle

    @classmethod
    def create(cls, device: int = 0, seed: int = 0) -> "OrderModel":
        h = C.c_void_p()
        L.check(L.lib.mg_order_model_create(device, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "OrderModel":
        h = C.c_void_p()
        L.check(L.lib.mg_order_model_load(path.encode(), device, C.byref(h)))
        return cls(h.value)

    def save(self, path: str) -> None:
        L.check(L.lib.mg_order_model_save(self.handle, path.encode()))

    @staticmethod
    def num_params() -> int:
        return L.lib.mg_order_model_num_params()

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params(), dtype=np.float32)
        L.check(L.lib.mg_order_model_get_params(self.handle, _f32p(out)))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        L.check(L.lib.mg_order_model_set_params(self.handle, _f32p(p)))

    def grad(self, dg: DeviceGraph, qs, sq, sm, st):
        """(gradient, mean squared error, FP32 predictions) over the samples."""
        sq, sm = np.ascontiguousarray(sq, np.uint32), np.ascontiguousarray(sm, np.uint32)
        st = np.ascontiguousarray(st, np.float32)
        g = np.zeros(self.num_params(), dtype=np.float32)
        pred = np.zeros(len(sq), dtype=np.float32)
        loss = C.c_float()
        L.check(L.lib.mg_order_model_grad(self.handle, dg.handle, _qarr(qs), len(qs),
                                          sq.ctypes.data_as(L.P32), sm.ctypes.data_as(L.P32),
                                          _f32p(st), len(sq), _f32p(g), C.byref(loss),
                                          _f32p(pred)))
        return g, loss.value, pred

    def train(self, dg: DeviceGraph, qs, sq, sm, st, epochs=20, batch=512, lr=1e-3,
              seed=0) -> float:
        sq, sm = np.ascontiguousarray(sq, np.uint32), np.ascontiguousarray(sm, np.uint32)
        st = np.ascontiguousarray(st, np.float32)
        loss = C.c_float()
        L.check(L.lib.mg_order_model_train(self.handle, dg.handle, _qarr(qs), len(qs),
                                           sq.ctypes.data_as(L.P32), sm.ctypes.data_as(L.P32),
                                           _f32p(st), len(sq), epochs, batch, lr, seed,
                                           C.byref(loss)))
        return loss.value

    def predict(self, dg: DeviceGraph, qs, sq, sm) -> np.ndarray:
        """BF16 predictions of log(1 + P(S))."""
        sq, sm = np.ascontiguousarray(sq, np.uint32), np.ascontiguousarray(sm, np.uint32)
        out = np.zeros(len(sq), dtype=np.float32)
        L.check(L.lib.mg_order_model_predict(self.handle, dg.handle, _qarr(qs), len(qs),
                                             sq.ctypes.data_as(L.P32), sm.ctypes.data_as(L.P32),
                                             len(sq), _f32p(out)))
        return out

    def free(self) -> None:
        if self.handle:
            L.lib.mg_order_model_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def features(dg: DeviceGraph, q: CSRGraph):
    x = np.zeros((16, 8), dtype=np.float32)
    e = np.zeros((16, 16), dtype=np.float32)
    adj = np.zeros(16, dtype=np.uint32)
    L.check(L.lib.mg_order_model_features(dg.handle, C.byref(q.view), _f32p(x), _f32p(e),
                                          adj.ctypes.data_as(L.P32)))
    return x, e, adj


def random_connected_order(q: CSRGraph, rng: np.random.Generator) -> list[int]:
    """Uniform start, then a uniform choice among vertices adjacent to the prefix."""
    k = q.n
    adj = [0] * k
    for a, b in query_edges(q):
        if a != b:
            adj[a] |= 1 << b
            adj[b] |= 1 << a
    order = [int(rng.integers(0, k))]
    placed = 1 << order[0]
    while len(order) < k:
        cand = [v for v in range(k) if not (placed >> v) & 1 and adj[v] & placed]
        if not cand:
            cand = [v for v in range(k) if not (placed >> v) & 1]
        v = int(cand[int(rng.integers(0, len(cand)))])
        order.append(v)
        placed |= 1 << v
    return order


def prefix_samples(q_index: int, order: Sequence[int], level_rows) -> list[tuple]:
    """(query, mask of the first i vertices, log(1 + P_i)) for i = 1..k."""
    out, mask = [], 0
    for i, v in enumerate(order, start=1):
        mask |= 1 << int(v)
        out.append((q_index, mask, math.log1p(float(level_rows[i]))))
    return out


def record_prefix_counts(dg: DeviceGraph, qs, n_random: int, budget: int, seed: int,
                         chunk: int = 2048):
    """Runs each query under the reference order and ``n_random`` random
    connected orders (per-query element budget) and returns training samples
    plus the raw records (query index, order, count, P_i)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for qi, q in enumerate(qs):
        jobs.append((qi, plan_order(q)))
        for _ in range(n_random):
            jobs.append((qi, random_connected_order(q, rng)))
    samples, records = [], []
    for s in range(0, len(jobs), chunk):
        part = jobs[s:s + chunk]
        counts, rows, _ = dg.batch_count_orders([qs[qi] for qi, _ in part], [o for _, o in part],
                                                max_elements=budget)
        for (qi, od), c, r in zip(part, counts, rows):
            records.append((qi, od, int(c), r[:len(od) + 1].tolist()))
            if c != UNKNOWN:
                samples.extend(prefix_samples(qi, od, r))
    sq = np.array([x[0] for x in samples], dtype=np.uint32)
    sm = np.array([x[1] for x in samples], dtype=np.uint32)
    st = np.array([x[2] for x in samples], dtype=np.float32)
    return (sq, sm, st), records
