"""Subgraph isomorphism over a device-resident data graph.

Host-side mirror of the reference's subiso entry points:

* ``SubIso(pattern_path, data_graph_path, data_graph_edgelist_path,
  output_path).Run()`` — core/task/gpu_task/subiso.cuh:43-51, subiso.cu:236-260;
* ``MatrixGraph(scheduler).Run(TaskType.kSubIso, task)`` —
  core/matrixgraph.cuh:36-42, core/matrixgraph.cu:30-46.

The reference prints a capped, non-exact join row count and exits the
process on CUDA errors (core/util/cuda_check.cuh:8-14); here ``Run`` stores
the exact count (and, in emit mode, the sorted matches), writes them to
``output_path`` when one is given, and raises :class:`MGError` on failure.
All device work goes through libmg_subiso.so.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import time
from typing import Sequence

import numpy as np

from . import _lib as L
from .graph import CSRGraph

ORDERS = {"reference": L.MG_ORDER_REFERENCE, "heuristic": L.MG_ORDER_REFERENCE,
          "strong": L.MG_ORDER_STRONG, "learned": L.MG_ORDER_LEARNED,
          "given": L.MG_ORDER_GIVEN}


def make_opts(order="reference", filters=L.MG_FILTER_ALL, chunk_rows=0, given_order=None,
              model=None, root_range=None, mem_budget_bytes=0, root_step=0,
              grab=0, no_tail=0, max_elements=0, probe_min=0, kernel_events=0, lanes=0,
              matrix_filter=None):
    o = L.default_opts()
    o.no_tail = no_tail
    o.max_elements = max_elements
    o.order = ORDERS[order] if isinstance(order, str) else int(order)
    o.filters = filters
    o.chunk_rows = chunk_rows
    o.mem_budget_bytes = mem_budget_bytes
    o.root_step = root_step
    o.probe_min = probe_min
    o.kernel_events = kernel_events
    o.lanes = L.MG_LANES_SHARED if lanes == "shared" else int(lanes)
    o.grab = grab
    keep = None
    if given_order is not None:
        keep = np.ascontiguousarray(np.asarray(given_order, dtype=np.uint32))
        o.given_order = keep.ctypes.data_as(L.P32)
        o.order = L.MG_ORDER_GIVEN
    if model is not None:
        o.model = model.handle if hasattr(model, "handle") else model
    if matrix_filter is not None:
        o.matrix_filter = (matrix_filter.handle if hasattr(matrix_filter, "handle")
                           else matrix_filter)
    if root_range is not None:
        o.root_begin, o.root_end = int(root_range[0]), int(root_range[1])
    return o, keep


def stats_dict(st: L.Stats) -> dict:
    k = st.k
    return {"k": k, "order": list(st.order[:k]), "level_rows": list(st.level_rows[:k + 1]),
            "balg_bytes": st.balg_bytes, "balg_count_bytes": st.balg_count_bytes,
            "device_ms": st.device_ms, "launches": st.launches, "chunks": st.chunks,
            "elements": st.elements, "expand_ms": st.expand_ms,
            "expand_launches": st.expand_launches}


def plan_order(q: CSRGraph, order="reference", graph: "DeviceGraph | None" = None,
               given_order=None, model=None) -> list[int]:
    o, keep = make_opts(order=order, given_order=given_order, model=model)
    out = (C.c_uint32 * L.MG_MAX_QUERY_VERTICES)()
    k = C.c_uint32()
    L.check(L.lib.mg_plan_order(graph.handle if graph else None, C.byref(q.view), C.byref(o),
                                out, C.byref(k)))
    return list(out[:k.value])


class DeviceGraph:
    """A data graph resident on one GPU with its derived indices."""

    def __init__(self, g: CSRGraph, device: int = 0, hub_bytes: int | None = None,
                 hub_min_degree: int = 0):
        """Uploads ``g``; ``hub_bytes`` caps the hub bitmaps (None: the library
        default, 0: none), ``hub_min_degree`` is the smallest hub degree."""
        h = C.c_void_p()
        uo = L.UploadOpts(L.MG_HUB_AUTO if hub_bytes is None else int(hub_bytes),
                          int(hub_min_degree), 0)
        L.check(L.lib.mg_graph_upload_ex(C.byref(g.view), device, C.byref(uo), C.byref(h)))
        self.handle = h.value
        self.device = device

    @property
    def info(self) -> dict:
        i = L.GraphInfo()
        L.check(L.lib.mg_graph_get_info(self.handle, C.byref(i)))
        return {f: getattr(i, f) for f, _ in L.GraphInfo._fields_}

    def count(self, q: CSRGraph, stats: bool = False, **kw):
        o, keep = make_opts(**kw)
        c = C.c_uint64()
        st = L.Stats()
        L.check(L.lib.mg_subiso_count_ex(self.handle, C.byref(q.view), C.byref(o), C.byref(c),
                                         C.byref(st)))
        return (c.value, stats_dict(st)) if stats else c.value

    def emit(self, q: CSRGraph, cap: int | None = None, stats: bool = False, **kw):
        """Sorted matches, one row of k global ids per match (query-id order)."""
        o, keep = make_opts(**kw)
        if cap is None:
            cap = self.count(q, **kw)
        rows = np.zeros((max(cap, 1), q.n), dtype=np.uint32)
        n = C.c_uint64()
        st = L.Stats()
        rc = L.lib.mg_subiso_emit_ex(self.handle, C.byref(q.view), C.byref(o),
                                     rows.ctypes.data_as(L.P32), cap, C.byref(n), C.byref(st))
        if rc not in (L.MG_OK, L.MG_E_CAPACITY):
            L.check(rc)
        out = rows[:min(cap, n.value)]
        if stats:
            return out, n.value, stats_dict(st)
        return out

    def batch_count(self, qs: Sequence[CSRGraph], stats: bool = False, **kw):
        o, keep = make_opts(**kw)
        arr = (C.POINTER(L.CsrView) * len(qs))(*[C.pointer(q.view) for q in qs])
        counts = np.zeros(len(qs), dtype=np.uint64)
        st = L.Stats()
        L.check(L.lib.mg_subiso_batch_count_ex(self.handle, arr, len(qs), C.byref(o),
                                               counts.ctypes.data_as(C.POINTER(C.c_uint64)),
                                               C.byref(st)))
        return (counts, stats_dict(st)) if stats else counts

    def batch_count_orders(self, qs: Sequence[CSRGraph], orders, **kw):
        """Counts and per-prefix survivors P_i of each query under its own order.

        Returns (counts[nq], level_rows[nq, 17], stats)."""
        o, keep = make_opts(**kw)
        nq = len(qs)
        arr = (C.POINTER(L.CsrView) * nq)(*[C.pointer(q.view) for q in qs])
        ords = np.zeros((nq, L.MG_MAX_QUERY_VERTICES), dtype=np.uint32)
        for i, od in enumerate(orders):
            ords[i, :len(od)] = od
        counts = np.zeros(nq, dtype=np.uint64)
        rows = np.zeros((nq, L.MG_MAX_QUERY_VERTICES + 1), dtype=np.uint64)
        st = L.Stats()
        L.check(L.lib.mg_subiso_batch_count_orders(
            self.handle, arr, nq, ords.ctypes.data_as(L.P32), C.byref(o),
            counts.ctypes.data_as(C.POINTER(C.c_uint64)),
            rows.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(st)))
        return counts, rows, stats_dict(st)

    def plan_order(self, q: CSRGraph, order="reference", **kw) -> list[int]:
        return plan_order(q, order=order, graph=self, **kw)

    def plan_orders(self, qs: Sequence[CSRGraph], order="reference", **kw) -> list[list[int]]:
        """Orders of many queries in one call (one inference launch when learned)."""
        o, keep = make_opts(order=order, **kw)
        nq = len(qs)
        arr = (C.POINTER(L.CsrView) * nq)(*[C.pointer(q.view) for q in qs])
        out = np.zeros((nq, L.MG_MAX_QUERY_VERTICES), dtype=np.uint32)
        L.check(L.lib.mg_plan_orders(self.handle, arr, nq, C.byref(o), out.ctypes.data_as(L.P32)))
        return [out[i, :q.n].tolist() for i, q in enumerate(qs)]

    def free(self) -> None:
        if self.handle:
            L.lib.mg_graph_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def level0_sizes(g: CSRGraph, qs: Sequence[CSRGraph], order="reference") -> list[int]:
    """Level-0 candidates of each query: the label bucket of its first vertex."""
    lab = g.array("labels")
    vals, cnts = np.unique(lab, return_counts=True)
    size = dict(zip(vals.tolist(), cnts.tolist()))
    out = []
    for q in qs:
        first = plan_order(q, order=order)[0]
        out.append(int(size.get(int(q.array("labels")[first]), 0)))
    return out


def shard_roots(n_roots: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous level-0 candidate range of one rank (independent shards)."""
    base, rem = divmod(n_roots, world)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def root_costs(g: CSRGraph, q: CSRGraph, order="reference") -> np.ndarray:
    """Estimated cost of each level-0 candidate of a query, in bucket order:
    its degree (the length of the lists its subtree starts from).  The bucket
    of the first vertex of the order lists that label's vertices by
    ascending id, as the engine's label bucket does."""
    lab = g.array("labels")
    first = plan_order(q, order=order)[0]
    bucket = np.flatnonzero(lab == q.array("labels")[first])
    return np.diff(g.array("out_off").astype(np.int64))[bucket]


def shard_roots_weighted(costs, rank: int, world: int) -> tuple[int, int]:
    """Contiguous level-0 range of one rank cut from the prefix sum of the
    candidates' estimated costs: rank r takes the candidates whose cost
    prefix falls in [r/world, (r+1)/world) of the total, so a bucket whose
    head holds the hubs is not handed to rank 0 whole.  The ranges of all
    ranks partition the bucket."""
    c = np.asarray(costs, dtype=np.float64)
    n = len(c)
    if world <= 1 or n == 0:
        return (0, n) if rank == 0 or world <= 1 else (n, n)
    tot = c.sum()
    if tot <= 0:
        return shard_roots(n, rank, world)
    mid = np.cumsum(c) - 0.5 * c  # cost midpoint of each candidate
    cut = lambda r: int(np.searchsorted(mid, tot * r / world, side="left"))  # noqa: E731
    return cut(rank), cut(rank + 1) if rank + 1 < world else n


def shard_batch(costs, rank: int, world: int) -> list[int]:
    """Query indices of one rank's share of a batch: queries in decreasing
    estimated cost, each to the rank with the least cost so far (ties to the
    lower rank).  Deterministic, so every rank computes the same split
    without an exchange; the shares partition the batch."""
    c = np.asarray(costs, dtype=np.float64)
    load = np.zeros(max(1, world))
    mine = []
    for i in sorted(range(len(c)), key=lambda j: (-c[j], j)):
        r = int(np.argmin(load))
        load[r] += c[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def shard_strided(rank: int, world: int) -> dict:
    """Count options of one rank's shard: level-0 candidates at bucket
    positions rank, rank + world, rank + 2*world, ...  A label bucket lists
    its vertices by id, and generators without id permutation (R-MAT) put
    the hubs first, so contiguous ranges would hand every hub to rank 0; a
    stride spreads them evenly.  The shards partition the bucket."""
    if world <= 1:
        return {}
    return {"root_range": (rank, 0), "root_step": world}


# ---- reference-shaped task / runtime ------------------------------------------
class TaskType(enum.IntEnum):
    """core/common/types.h:47-60."""
    kGEMM = 0
    kMatrixAnalysis = 1
    kPPRQuery = 2
    kSubIso = 3
    kGARMatch = 4
    kCPUSubIso = 5
    kWCC = 6
    kSSSP = 7
    kBFS = 8
    kPageRank = 9
    kGEMV = 10


class SchedulerType(enum.IntEnum):
    """core/components/scheduler/scheduler.h (ignored by subiso, as in the reference)."""
    kCHBL = 0
    kEvenSplit = 1
    kRoundRobin = 2


class SubIso:
    """``SubIso`` task: pattern and data graph CSR directories in, exact matches
    out.  ``matrix_paths``: the six matrix directories of the reference's
    CPUSubIso (matrix_path1..6, core/task/cpu_task/cpu_subiso.cuh:32-39);
    when given, the lossy MatrixFilter drops level-0 candidates."""

    def __init__(self, pattern_path: str, data_graph_path: str,
                 data_graph_edgelist_path: str = "", output_path: str = "",
                 mode: str = "count", order: str = "reference", device: int = 0,
                 model=None, matrix_paths=None):
        self.pattern_path = pattern_path
        self.data_graph_path = data_graph_path
        self.data_graph_edgelist_path = data_graph_edgelist_path  # unused, as in the reference
        self.output_path = output_path
        self.mode = mode
        self.order = order
        self.device = device
        self.model = model
        self.matrix_paths = list(matrix_paths) if matrix_paths else None
        self.count = None
        self.rows = None
        self.timings = {}

    def LoadData(self):
        self.p_ = CSRGraph.Read(self.pattern_path)
        self.g_ = CSRGraph.Read(self.data_graph_path)

    def Run(self):
        t0 = time.perf_counter()
        self.LoadData()
        t1 = time.perf_counter()
        dg = DeviceGraph(self.g_, self.device)
        mf = None
        try:
            if self.matrix_paths:
                from .matrix_filter import MatrixFilter
                mf = MatrixFilter.load(self.matrix_paths, self.device)
            t2 = time.perf_counter()
            kw = {"order": self.order, "model": self.model, "matrix_filter": mf}
            self.count = dg.count(self.p_, **kw)
            if self.mode == "emit":
                self.rows = dg.emit(self.p_, cap=self.count, **kw)
            t3 = time.perf_counter()
        finally:
            if mf is not None:
                mf.free()
            dg.free()
        self.timings = {"load_s": t1 - t0, "upload_s": t2 - t1, "match_s": t3 - t2}
        if self.output_path:
            self.Write(self.output_path)
        return self.count

    def Write(self, path: str):
        os.makedirs(os.path.dirname(os.path.abspath(path)) or ".", exist_ok=True)
        with open(path, "w") as f:
            f.write(f"{self.count}\n")
            if self.rows is not None:
                for r in self.rows:
                    f.write(",".join(str(int(x)) for x in r) + "\n")


class MatrixGraph:
    """Runtime dispatch (core/matrixgraph.cu:30-79): only kSubIso is served."""

    def __init__(self, scheduler: SchedulerType = SchedulerType.kCHBL):
        self.scheduler = scheduler

    def Run(self, task_type: TaskType, task):
        if task_type != TaskType.kSubIso:
            raise L.MGError(L.MG_E_ARG, f"task type {TaskType(task_type).name} is not served")
        return task.Run()
