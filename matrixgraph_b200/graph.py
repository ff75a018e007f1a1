"""Host graphs in the reference's binary CSR layout, and seeded generators.

:class:`CSRGraph` mirrors ``ImmutableCSR`` of the reference
(core/data_structures/immutable_csr.cuh): ``Read(root_path)`` /
``Write(root_path)`` over a directory prefix ending in '/', holding
``meta.yaml``, ``graphs/0.bin`` and ``label/0.bin``.  Memory is owned by the
native library; numpy views are exposed for inspection.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

import numpy as np

from . import _lib as L

# Query shapes of the single-query benchmark (undirected edge lists).
SHAPES = {
    "triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "4-cycle": (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
    "4-clique": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]),
    "5-path": (5, [(0, 1), (1, 2), (2, 3), (3, 4)]),
    "tailed-triangle": (4, [(0, 1), (1, 2), (2, 0), (2, 3)]),
}


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(L.P32)


class CSRGraph:
    """A graph (data graph or pattern) in reference CSR layout, host memory."""

    def __init__(self, view: L.CsrView, owner: int | None, keep: tuple = ()):
        self.view = view
        self._owner = owner
        self._keep = keep

    # -- construction ---------------------------------------------------------
    @classmethod
    def Read(cls, root_path: str) -> "CSRGraph":
        """Reads a CSR directory (``root_path`` must end in '/')."""
        v = L.CsrView()
        owner = C.c_void_p()
        L.check(L.lib.mg_csr_dir_open(root_path.encode(), C.byref(v), C.byref(owner)))
        return cls(v, owner.value)

    read = Read

    @classmethod
    def from_edges(cls, n: int, src, dst, labels=None, symmetrize=False, no_self=False,
                   dedup=False) -> "CSRGraph":
        s, d = _u32(src), _u32(dst)
        lab = _u32(labels if labels is not None else np.zeros(n))
        flags = (L.MG_BUILD_SYMMETRIZE if symmetrize else 0) | \
            (L.MG_BUILD_NO_SELF if no_self else 0) | (L.MG_BUILD_DEDUP if dedup else 0)
        v = L.CsrView()
        owner = C.c_void_p()
        L.check(L.lib.mg_csr_from_edges(n, _ptr(s), _ptr(d), len(s), _ptr(lab), flags,
                                        C.byref(v), C.byref(owner)))
        return cls(v, owner.value)

    @classmethod
    def from_csv(cls, path: str, label_range: int = 1) -> "CSRGraph":
        v = L.CsrView()
        owner = C.c_void_p()
        L.check(L.lib.mg_csr_from_csv(path.encode(), label_range, C.byref(v), C.byref(owner)))
        return cls(v, owner.value)

    @classmethod
    def query(cls, k: int, edges: Iterable[tuple[int, int]], labels: Sequence[int],
              directed: bool = False) -> "CSRGraph":
        """A pattern from an edge list (symmetrised unless ``directed``)."""
        e = list(edges)
        eu = _u32([a for a, _ in e] or [0])
        ev = _u32([b for _, b in e] or [0])
        lab = _u32(labels)
        v = L.CsrView()
        owner = C.c_void_p()
        L.check(L.lib.mg_query_from_edges(k, _ptr(eu), _ptr(ev), len(e), _ptr(lab),
                                          1 if directed else 0, C.byref(v), C.byref(owner)))
        return cls(v, owner.value)

    def Write(self, root_path: str) -> None:
        L.check(L.lib.mg_csr_dir_write(root_path.encode(), C.byref(self.view)))

    write = Write

    # -- accessors ----------------------------------------------------------------
    def _arr(self, name: str, size: int) -> np.ndarray:
        p = getattr(self.view, name)
        if not p or size == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(p, shape=(size,))

    @property
    def n(self) -> int:
        return self.view.n

    @property
    def m_out(self) -> int:
        return self.view.m_out

    @property
    def m_in(self) -> int:
        return self.view.m_in

    @property
    def max_vid(self) -> int:
        return self.view.max_vid

    def array(self, name: str) -> np.ndarray:
        n, v = self.view.n, self.view
        sizes = {"globalid": n, "indeg": n, "outdeg": n, "in_off": n + 1, "out_off": n + 1,
                 "in_edges": v.m_in, "out_edges": v.m_out, "labels": n,
                 "edges_globalid_by_localid": v.max_vid + 1,
                 "localid_by_globalid": v.max_vid + 1}
        return self._arr(name, sizes[name])

    def close(self) -> None:
        if self._owner:
            L.lib.mg_csr_dir_close(self._owner)
            self._owner = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- generators -------------------------------------------------------------------
def _take_edges(src_p, dst_p, m: int) -> tuple[np.ndarray, np.ndarray]:
    s = np.ctypeslib.as_array(src_p, shape=(max(m, 1),))[:m].copy()
    d = np.ctypeslib.as_array(dst_p, shape=(max(m, 1),))[:m].copy()
    L.lib.mg_free_buffer(C.cast(src_p, C.c_void_p))
    L.lib.mg_free_buffer(C.cast(dst_p, C.c_void_p))
    return s, d


def gen_labels(n: int, L_: int, kind: str = "uniform", s: float = 1.0, seed: int = 1):
    out = np.zeros(n, dtype=np.uint32)
    L.check(L.lib.mg_gen_labels(n, 0 if kind == "uniform" else 1, L_, s, seed, _ptr(out)))
    return out


def chung_lu(n: int = 10000, beta: float = 2.5, avg_deg: float = 10.0, seed: int = 0,
             n_labels: int = 8, label_kind: str = "uniform", zipf_s: float = 1.0,
             label_seed: int = 1, threads: int = 0) -> CSRGraph:
    """Undirected Chung-Lu power-law graph, symmetrised, no self-loops."""
    sp, dp, m = L.P32(), L.P32(), C.c_uint64()
    L.check(L.lib.mg_gen_chung_lu(n, beta, avg_deg, seed, threads, C.byref(sp), C.byref(dp),
                                  C.byref(m)))
    s, d = _take_edges(sp, dp, m.value)
    lab = gen_labels(n, n_labels, label_kind, zipf_s, label_seed)
    return CSRGraph.from_edges(n, s, d, lab, symmetrize=True, no_self=True, dedup=True)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 0, n_labels: int = 32, label_kind: str = "zipf",
         zipf_s: float = 1.0, label_seed: int = 1, threads: int = 0) -> CSRGraph:
    """Symmetrised R-MAT graph, self-loops and duplicates removed, ids not permuted."""
    sp, dp, m = L.P32(), L.P32(), C.c_uint64()
    L.check(L.lib.mg_gen_rmat(scale, edge_factor, a, b, c, seed, threads, C.byref(sp),
                              C.byref(dp), C.byref(m)))
    mm = m.value
    n = 1 << scale
    lab = gen_labels(n, n_labels, label_kind, zipf_s, label_seed)
    # Edge arrays stay in native memory until the CSR is built.
    v = L.CsrView()
    owner = C.c_void_p()
    try:
        L.check(L.lib.mg_csr_from_edges(n, sp, dp, mm, _ptr(lab),
                                        L.MG_BUILD_SYMMETRIZE | L.MG_BUILD_NO_SELF |
                                        L.MG_BUILD_DEDUP, C.byref(v), C.byref(owner)))
    finally:
        L.lib.mg_free_buffer(C.cast(sp, C.c_void_p))
        L.lib.mg_free_buffer(C.cast(dp, C.c_void_p))
    return CSRGraph(v, owner.value)


def query_walk(g: CSRGraph, shape: str | tuple, seed: int) -> CSRGraph:
    """Labelled query of a named (or (k, edges)) shape, labels by random walk on ``g``."""
    k, edges = SHAPES[shape] if isinstance(shape, str) else shape
    eu = _u32([x for x, _ in edges])
    ev = _u32([y for _, y in edges])
    v = L.CsrView()
    owner = C.c_void_p()
    L.check(L.lib.mg_gen_query_walk(C.byref(g.view), k, _ptr(eu), _ptr(ev), len(edges), seed,
                                    C.byref(v), C.byref(owner)))
    return CSRGraph(v, owner.value)


def query_random(g: CSRGraph, k: int, p_extra: float, seed: int) -> CSRGraph:
    """Random connected query: recursive spanning tree + extra edges, walk labels."""
    v = L.CsrView()
    owner = C.c_void_p()
    L.check(L.lib.mg_gen_query_random(C.byref(g.view), k, p_extra, seed, C.byref(v),
                                      C.byref(owner)))
    return CSRGraph(v, owner.value)


def query_edges(q: CSRGraph) -> list[tuple[int, int]]:
    """Directed edges (local ids) of a pattern in CSR order."""
    gid = q.array("globalid")
    g2l = {int(x): i for i, x in enumerate(gid)}
    off, adj = q.array("out_off"), q.array("out_edges")
    return [(u, g2l[int(adj[e])]) for u in range(q.n) for e in range(off[u], off[u + 1])]
