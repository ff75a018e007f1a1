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


if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(os.path.join(HERE, f)) for f in ("oracle.c", "gen.c")):
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
                           C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(OrcResult)]
PP32 = C.POINTER(P32)
_lib.orc_gen_rmat_csr.argtypes = [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                  C.c_uint64, C.c_int, PP32, PP32, C.POINTER(C.c_uint64)]
_lib.orc_csr_symmetric.argtypes = [C.c_uint32, P32, P32, C.c_uint64, C.c_int, PP32, PP32,
                                   C.POINTER(C.c_uint64)]
_lib.orc_gen_labels.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64,
                                P32]
_lib.orc_walk_labels.argtypes = [C.c_uint32, P32, P32, P32, C.c_uint32, P32, C.c_uint64,
                                 C.c_uint64, P32]
_lib.orc_random_query_shape.argtypes = [C.c_uint32, C.c_double, C.c_uint64, P32]
_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]
_lib.orc_emit.argtypes = [C.c_void_p, C.POINTER(OrcQuery), P32, C.c_uint32, C.c_uint64,
                          C.c_uint64, C.c_uint64, P32, C.c_uint64, C.POINTER(C.c_uint64)]
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


def count(g: Graph, q: OrcQuery, order=None, filters=3, threads=1, root_range=None,
          root_step=1) -> dict:
    """Exact count over the level-0 candidates at bucket positions
    begin, begin + root_step, ... below end (root_range None: the whole bucket)."""
    order = reference_order(q) if order is None else list(order)
    o = _u32(order)
    r = OrcResult()
    rb, re_ = (0, 2 ** 64 - 1) if root_range is None else root_range
    rc = _lib.orc_count(g.h, C.byref(q), _p(o), filters, threads, rb, re_, max(1, root_step),
                        C.byref(r))
    if rc:
        raise RuntimeError(f"oracle count failed: {rc}")
    return {"count": r.count, "level_rows": list(r.level_rows[:q.k + 1]), "balg": r.balg,
            "balg_count": r.balg_count, "order": order}


def emit(g: Graph, q: OrcQuery, order=None, filters=3, cap=None, root_range=None,
         root_step=1) -> np.ndarray:
    """Sorted match rows over the level-0 positions begin, begin + root_step, ...
    below end (root_range None: the whole bucket)."""
    order = reference_order(q) if order is None else list(order)
    rb, re_ = (0, 2 ** 64 - 1) if root_range is None else root_range
    if cap is None:
        cap = count(g, q, order, filters, root_range=(rb, re_), root_step=root_step)["count"]
    rows = np.zeros((max(cap, 1), q.k), dtype=np.uint32)
    n = C.c_uint64()
    rc = _lib.orc_emit(g.h, C.byref(q), _p(_u32(order)), filters, rb, re_, max(1, root_step),
                       _p(rows), cap, C.byref(n))
    if rc:
        raise RuntimeError(f"oracle emit failed: {rc}")
    return rows[:min(cap, n.value)]


def bucket_size(g: Graph, q: OrcQuery, order) -> int:
    return _lib.orc_bucket_size(g.h, C.byref(q), _p(_u32(order)))


# ---- checker-side generators (oracle/gen.c) ---------------------------------------
class PlainGraph:
    """Symmetrised data graph as plain sorted CSR arrays (identity ids), built by
    oracle/gen.c without the product library."""

    def __init__(self, n, off, adj, labels):
        self.n, self.off, self.adj, self.labels = n, off, adj, labels

    @property
    def m(self):
        return int(self.off[-1])

    def oracle_graph(self) -> Graph:
        gid = np.arange(self.n, dtype=np.uint32)
        return Graph.from_arrays(self.n, self.n - 1, gid, self.off, self.adj, self.off,
                                 self.adj, self.labels)

    def degree(self):
        return np.diff(self.off.astype(np.int64))


def _take(p, size):
    out = np.ctypeslib.as_array(p, shape=(max(size, 1),))[:size].copy()
    _libc.free(C.cast(p, C.c_void_p))
    return out


def gen_labels(n, L, kind="uniform", s=1.0, seed=1):
    out = np.zeros(n, dtype=np.uint32)
    rc = _lib.orc_gen_labels(n, 0 if kind == "uniform" else 1, L, s, seed, _p(out))
    if rc:
        raise RuntimeError(f"oracle labels failed: {rc}")
    return out


def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=0, n_labels=32, label_kind="zipf",
         zipf_s=1.0, label_seed=1, threads=None) -> PlainGraph:
    """Symmetrised R-MAT graph (self-loops and repeats removed, ids not permuted)."""
    threads = threads or os.cpu_count() or 1
    op, ap, m = P32(), P32(), C.c_uint64()
    rc = _lib.orc_gen_rmat_csr(scale, edge_factor, a, b, c, seed, threads, C.byref(op),
                               C.byref(ap), C.byref(m))
    if rc:
        raise RuntimeError(f"oracle rmat failed: {rc}")
    n = 1 << scale
    off, adj = _take(op, n + 1), _take(ap, m.value)
    return PlainGraph(n, off, adj, gen_labels(n, n_labels, label_kind, zipf_s, label_seed))


def _masks(k, edges):
    adjm = np.zeros(16, dtype=np.uint32)
    for u, w in edges:
        adjm[u] |= 1 << w
        adjm[w] |= 1 << u
    return adjm


def walk_labels(g: PlainGraph, k, edges, seed, stream=0x57414C4B):
    """Query labels copied from a random walk on g along the BFS tree of the query."""
    out = np.zeros(16, dtype=np.uint32)
    rc = _lib.orc_walk_labels(g.n, _p(g.off), _p(g.adj), _p(g.labels), k, _p(_masks(k, edges)),
                              seed, stream, _p(out))
    if rc:
        raise RuntimeError(f"oracle walk failed: {rc}")
    return out[:k].tolist()


def random_query_edges(k, p_extra, seed):
    """Edges of a random connected query (spanning tree + extra pairs)."""
    adjm = np.zeros(16, dtype=np.uint32)
    rc = _lib.orc_random_query_shape(k, p_extra, seed, _p(adjm))
    if rc:
        raise RuntimeError(f"oracle random query failed: {rc}")
    return [(u, w) for u in range(k) for w in range(u + 1, k) if adjm[u] >> w & 1]


def query_from_edges(k, edges, labels) -> OrcQuery:
    """Symmetrised query over local ids 0..k-1 with sorted adjacency."""
    nb = [set() for _ in range(k)]
    for u, w in edges:
        nb[u].add(w)
        nb[w].add(u)
    off = np.zeros(k + 1, dtype=np.uint32)
    adj = []
    for u in range(k):
        adj += sorted(nb[u])
        off[u + 1] = len(adj)
    return make_query(k, np.arange(k), off, adj or [0], labels)
