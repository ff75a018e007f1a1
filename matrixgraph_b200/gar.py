"""GAR pattern match over edge lists (``matrixgraph_gar_match``).

Host-side mirror of the reference's C-style GAR entry
``GARMatch::Run(g arrays, p arrays, out arrays)``
(core/task/gpu_task/gar_match.cuh:41-66, core/go_api/matrixgraph_go_api.h:30-55)
with its input and output types GARGraphArrays, GARPatternArrays and
GARMatchArrays (core/data_structures/gar_*_arrays.h).  The matching runs in
libmg_subiso.so (include/mg_gar_match.h).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

_PI32 = C.POINTER(C.c_int32)


@dataclass
class GARGraphArrays:
    """Data graph: vertices by local index (instance ids ``v_id``, labels
    ``v_label_idx``), directed edges by local index with labels."""
    v_id: np.ndarray | None
    v_label_idx: np.ndarray | None
    e_src: np.ndarray
    e_dst: np.ndarray
    e_id: np.ndarray | None = None
    e_label_idx: np.ndarray | None = None
    n_vertices: int | None = None

    def __post_init__(self):
        if self.n_vertices is None:
            self.n_vertices = 0 if self.v_label_idx is None else len(self.v_label_idx)


@dataclass
class GARPatternArrays:
    node_label_idx: np.ndarray | None
    edge_src: np.ndarray
    edge_dst: np.ndarray
    edge_label_idx: np.ndarray | None = None
    n_nodes: int | None = None

    def __post_init__(self):
        if self.n_nodes is None:
            self.n_nodes = 0 if self.node_label_idx is None else len(self.node_label_idx)


@dataclass
class GARMatchArrays:
    """Pivot-grouped output: row i = (pivot, condition, position) with the
    ids ``matched_v_ids[row_offset[i] : row_offset[i] + row_count[i]]``."""
    num_conditions: int = 0
    row_pivot_id: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    row_cond_j: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    row_pos: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    row_offset: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    row_count: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    matched_v_ids: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    n_matches: int = 0   # distinct matches (not part of the reference output)

    @property
    def row_size(self) -> int:
        return len(self.row_pivot_id)

    @property
    def match_size(self) -> int:
        return len(self.matched_v_ids)

    def rows(self):
        """(pivot, cond_j, pos, ids) per row."""
        return [(int(self.row_pivot_id[i]), int(self.row_cond_j[i]), int(self.row_pos[i]),
                 self.matched_v_ids[self.row_offset[i]:self.row_offset[i] + self.row_count[i]]
                 .tolist()) for i in range(self.row_size)]


def _arr(a, dt):
    if a is None:
        return None, None
    x = np.ascontiguousarray(np.asarray(a, dtype=dt))
    return x, x.ctypes.data_as(C.POINTER(np.ctypeslib.as_ctypes_type(dt)))


def gar_match(g: GARGraphArrays, p: GARPatternArrays, row_capacity: int, match_capacity: int,
              opts: L.Opts | None = None, raw: bool = False):
    """Runs ``mg_gar_match_ex``; returns GARMatchArrays, or (status, result)
    when ``raw`` (no exception on a non-zero status)."""
    keep = []

    def a(x, dt):
        arr, ptr = _arr(x, dt)
        keep.append(arr)
        return ptr

    rcap, mcap = int(row_capacity), int(match_capacity)
    out = {
        "pivot": np.zeros(max(rcap, 0), np.uint32), "cond": np.zeros(max(rcap, 0), np.int32),
        "pos": np.zeros(max(rcap, 0), np.int32), "off": np.zeros(max(rcap, 0), np.int32),
        "cnt": np.zeros(max(rcap, 0), np.int32), "ids": np.zeros(max(mcap, 0), np.uint32),
    }
    nc, rs, ms = C.c_int(-5), C.c_int(-5), C.c_int(-5)
    nm = C.c_uint64()
    rc = L.lib.mg_gar_match_ex(
        a(g.v_id, np.uint32), a(g.v_label_idx, np.int32), int(g.n_vertices),
        a(g.e_src, np.uint32), a(g.e_dst, np.uint32), a(g.e_id, np.uint32),
        a(g.e_label_idx, np.int32), 0 if g.e_src is None else len(g.e_src),
        a(p.node_label_idx, np.int32), int(p.n_nodes),
        a(p.edge_src, np.int32), a(p.edge_dst, np.int32), a(p.edge_label_idx, np.int32),
        0 if p.edge_src is None else len(p.edge_src),
        C.byref(nc), out["pivot"].ctypes.data_as(L.P32), out["cond"].ctypes.data_as(_PI32),
        out["pos"].ctypes.data_as(_PI32), out["off"].ctypes.data_as(_PI32),
        out["cnt"].ctypes.data_as(_PI32), rcap, C.byref(rs),
        out["ids"].ctypes.data_as(L.P32), mcap, C.byref(ms),
        C.byref(opts) if opts is not None else None, C.byref(nm))
    res = GARMatchArrays(num_conditions=nc.value, row_pivot_id=out["pivot"][:rs.value].copy(),
                         row_cond_j=out["cond"][:rs.value].copy(),
                         row_pos=out["pos"][:rs.value].copy(),
                         row_offset=out["off"][:rs.value].copy(),
                         row_count=out["cnt"][:rs.value].copy(),
                         matched_v_ids=out["ids"][:ms.value].copy(), n_matches=nm.value)
    if raw:
        return rc, res
    L.check(rc)
    return res


def gar_instance(g: GARGraphArrays, p: GARPatternArrays):
    """The matching instance (data CSRGraph, query CSRGraph) that
    ``gar_match`` runs on the GPU, or None when the answer is empty without
    matching."""
    from .graph import CSRGraph
    keep = []

    def a(x, dt):
        arr, ptr = _arr(x, dt)
        keep.append(arr)
        return ptr

    dv, qv = L.CsrView(), L.CsrView()
    do, qo = C.c_void_p(), C.c_void_p()
    L.check(L.lib.mg_gar_instance(
        a(g.v_id, np.uint32), a(g.v_label_idx, np.int32), int(g.n_vertices),
        a(g.e_src, np.uint32), a(g.e_dst, np.uint32), a(g.e_label_idx, np.int32),
        0 if g.e_src is None else len(g.e_src),
        a(p.node_label_idx, np.int32), int(p.n_nodes),
        a(p.edge_src, np.int32), a(p.edge_dst, np.int32), a(p.edge_label_idx, np.int32),
        0 if p.edge_src is None else len(p.edge_src),
        C.byref(dv), C.byref(do), C.byref(qv), C.byref(qo)))
    if not do.value:
        return None
    return CSRGraph(dv, do.value), CSRGraph(qv, qo.value)


def gar_flatten(rows: np.ndarray, n_nodes: int, v_id, n_vertices: int, row_capacity: int,
                match_capacity: int) -> GARMatchArrays:
    """GARMatchArrays from match rows whose first ``n_nodes`` columns are the
    pattern nodes' local indices."""
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.uint32))
    if rows.ndim != 2:
        rows = rows.reshape(-1, max(1, n_nodes))
    vid, vptr = _arr(v_id, np.uint32)
    rcap, mcap = int(row_capacity), int(match_capacity)
    piv = np.zeros(max(rcap, 0), np.uint32)
    cond, pos, off, cnt = (np.zeros(max(rcap, 0), np.int32) for _ in range(4))
    ids = np.zeros(max(mcap, 0), np.uint32)
    nc, rs, ms = C.c_int(), C.c_int(), C.c_int()
    L.check(L.lib.mg_gar_flatten(
        rows.ctypes.data_as(L.P32), rows.shape[0], rows.shape[1], n_nodes, vptr,
        int(n_vertices), C.byref(nc), piv.ctypes.data_as(L.P32), cond.ctypes.data_as(_PI32),
        pos.ctypes.data_as(_PI32), off.ctypes.data_as(_PI32), cnt.ctypes.data_as(_PI32), rcap,
        C.byref(rs), ids.ctypes.data_as(L.P32), mcap, C.byref(ms)))
    del vid
    return GARMatchArrays(num_conditions=nc.value, row_pivot_id=piv[:rs.value],
                          row_cond_j=cond[:rs.value], row_pos=pos[:rs.value],
                          row_offset=off[:rs.value], row_count=cnt[:rs.value],
                          matched_v_ids=ids[:ms.value])
