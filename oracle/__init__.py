"""ctypes binding of the CPU oracle (oracle/oracle.c) — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
and reference legs, as the checker and the timed CPU port.  The product
(matrixgraph_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
MAXK = 16


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
        os.path.join(HERE, "oracle.c")):
    build()

_lib = C.CDLL(LIB_PATH)
P32 = C.POINTER(C.c_uint32)


class OrcQuery(C.Structure):
    _fields_ = [("k", C.c_uint32), ("label_raw", C.c_uint32 * MAXK),
                ("out_mask", C.c_uint32 * MAXK), ("n_edges", C.c_uint32),
                ("esrc", C.c_uint32 * (MAXK * MAXK)), ("edst", C.c_uint32 * (MAXK * MAXK))]


class OrcResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("level_rows", C.c_uint64 * (MAXK + 1)),
                ("balg", C.c_uint64), ("balg_count", C.c_uint64)]


_lib.orc_graph_from_arrays.restype = C.c_void_p
_lib.orc_graph_from_arrays.argtypes = [C.c_uint32, C.c_uint32, P32, P32, P32, P32, P32, P32,
                                       C.POINTER(C.c_int)]
_lib.orc_read_dir.restype = C.c_void_p
_lib.orc_read_dir.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
_lib.orc_graph_free.argtypes = [C.c_void_p]
_lib.orc_graph_info.argtypes = [C.c_void_p, P32, P32, C.POINTER(C.c_int),
                                C.POINTER(C.c_uint64)]
_lib.orc_query_from_arrays.argtypes = [C.c_uint32, P32, P32, P32, P32, C.POINTER(OrcQuery)]
_lib.orc_order_reference.argtypes = [C.POINTER(OrcQuery), P32]
_lib.orc_count.argtypes = [C.c_void_p, C.POINTER(OrcQuery), P32, C.c_uint32, C.c_int,
                           C.c_uint64, C.c_uint64, C.POINTER(OrcResult)]
_lib.orc_emit.argtypes = [C.c_void_p, C.POINTER(OrcQuery), P32, C.c_uint32, P32, C.c_uint64,
                          C.POINTER(C.c_uint64)]
_lib.orc_bucket_size.restype = C.c_uint32
_lib.orc_bucket_size.argtypes = [C.c_void_p, C.POINTER(OrcQuery), P32]


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _p(a):
    return a.ctypes.data_as(P32)


class Graph:
    """Oracle-side data graph (own normalisation of the reference arrays)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_arrays(cls, n, max_vid, globalid, out_off, out_edges, in_off, in_edges, labels):
        arrs = [_u32(x) for x in (globalid, out_off, out_edges, in_off, in_edges, labels)]
        err = C.c_int()
        h = _lib.orc_graph_from_arrays(n, max_vid, *[_p(a) for a in arrs], C.byref(err))
        if not h:
            raise RuntimeError(f"oracle graph build failed: {err.value}")
        return cls(h)

    @classmethod
    def from_csr(cls, g):
        """From a matrixgraph_b200.CSRGraph (reads its reference arrays)."""
        return cls.from_arrays(g.n, g.max_vid, g.array("globalid"), g.array("out_off"),
                               g.array("out_edges"), g.array("in_off"), g.array("in_edges"),
                               g.array("labels"))

    @classmethod
    def read_dir(cls, path: str):
        err = C.c_int()
        h = _lib.orc_read_dir(path.encode(), C.byref(err))
        if not h:
            raise RuntimeError(f"oracle read failed: {err.value}")
        return cls(h)

    def info(self):
        n, L, m = C.c_uint32(), C.c_uint32(), C.c_uint64()
        s = C.c_int()
        _lib.orc_graph_info(self.h, C.byref(n), C.byref(L), C.byref(s), C.byref(m))
        return {"n": n.value, "L": L.value, "symmetric": bool(s.value), "m_out": m.value}

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:  # _lib is None at interpreter exit
            _lib.orc_graph_free(self.h)
            self.h = None


def make_query(k, globalid, out_off, out_edges, labels) -> OrcQuery:
    q = OrcQuery()
    arrs = [_u32(x) for x in (globalid, out_off, out_edges, labels)]
    rc = _lib.orc_query_from_arrays(k, *[_p(a) for a in arrs], C.byref(q))
    if rc:
        raise RuntimeError(f"oracle query build failed: {rc}")
    return q


def query_from_csr(q) -> OrcQuery:
    return make_query(q.n, q.array("globalid"), q.array("out_off"), q.array("out_edges"),
                      q.array("labels"))


def reference_order(q: OrcQuery) -> list[int]:
    out = (C.c_uint32 * MAXK)()
    _lib.orc_order_reference(C.byref(q), out)
    return list(out[:q.k])


def count(g: Graph, q: OrcQuery, order=None, filters=3, threads=1, root_range=None) -> dict:
    order = reference_order(q) if order is None else list(order)
    o = _u32(order)
    r = OrcResult()
    rb, re_ = (0, 2 ** 64 - 1) if root_range is None else root_range
    rc = _lib.orc_count(g.h, C.byref(q), _p(o), filters, threads, rb, re_, C.byref(r))
    if rc:
        raise RuntimeError(f"oracle count failed: {rc}")
    return {"count": r.count, "level_rows": list(r.level_rows[:q.k + 1]), "balg": r.balg,
            "balg_count": r.balg_count, "order": order}


def emit(g: Graph, q: OrcQuery, order=None, filters=3, cap=None) -> np.ndarray:
    order = reference_order(q) if order is None else list(order)
    if cap is None:
        cap = count(g, q, order, filters)["count"]
    rows = np.zeros((max(cap, 1), q.k), dtype=np.uint32)
    n = C.c_uint64()
    rc = _lib.orc_emit(g.h, C.byref(q), _p(_u32(order)), filters, _p(rows), cap, C.byref(n))
    if rc:
        raise RuntimeError(f"oracle emit failed: {rc}")
    return rows[:min(cap, n.value)]


def bucket_size(g: Graph, q: OrcQuery, order) -> int:
    return _lib.orc_bucket_size(g.h, C.byref(q), _p(_u32(order)))
