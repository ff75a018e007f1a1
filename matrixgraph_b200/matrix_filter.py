"""Lossy learned candidate filter compatible with the reference's MatrixFilter
(core/task/cpu_task/cpu_subiso.cu:237-277): a small MLP over the squared
difference of a query vertex's and a data vertex's embeddings rejects the
pair when its sigmoid output is below 0.1.  Its six matrices use the
reference's container (core/data_structures/matrix.cu:12-35): a directory
with ``meta.yaml`` (``x``, ``y``) and ``embedding.bin`` (float32, row-major).

    mf = MatrixFilter.load([m1, m2, m3, m4, m5, m6])   # -m1..-m6 of the reference
    dg.count(q, matrix_filter=mf)                       # level-0 candidates filtered

Counts under the filter drop every match whose first-position vertex is
rejected; without it (the default) counts are exact."""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

from . import _lib as L


def write_matrix(dirpath: str, a) -> None:
    """Writes a 2-D float32 array in the reference's matrix container."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if a.ndim != 2:
        raise ValueError("a matrix is two-dimensional")
    os.makedirs(dirpath, exist_ok=True)
    a.tofile(os.path.join(dirpath, "embedding.bin"))
    with open(os.path.join(dirpath, "meta.yaml"), "w") as f:
        f.write(f"dtype: float32\nendian: little\norder: row_major\nx: {a.shape[0]}\n"
                f"y: {a.shape[1]}\n")


def read_matrix(dirpath: str) -> np.ndarray:
    meta = {}
    with open(os.path.join(dirpath, "meta.yaml")) as f:
        for ln in f:
            if ":" in ln:
                k, v = ln.split(":", 1)
                meta[k.strip()] = v.strip()
    x, y = int(meta["x"]), int(meta["y"])
    a = np.fromfile(os.path.join(dirpath, "embedding.bin"), dtype="<f4", count=x * y)
    return a.reshape(x, y)


class MatrixFilter:
    """Device copy of the six matrices (mg_matrix_filter_load)."""

    def __init__(self, handle):
        self.handle = handle

    @classmethod
    def load(cls, dirs: Sequence[str], device: int = 0) -> "MatrixFilter":
        if len(dirs) != 6:
            raise ValueError("six matrix directories (-m1..-m6)")
        paths = [os.path.join(d, "") for d in dirs]
        arr = (C.c_char_p * 6)(*[p.encode() for p in paths])
        h = C.c_void_p()
        L.check(L.lib.mg_matrix_filter_load(arr, device, C.byref(h)))
        return cls(h)

    def keep(self, u: int, v) -> np.ndarray:
        """1 where the filter keeps (query vertex u, data vertex v[i])."""
        v = np.ascontiguousarray(np.asarray(v, dtype=np.uint32))
        out = np.zeros(len(v), dtype=np.uint8)
        L.check(L.lib.mg_matrix_filter_keep(self.handle, int(u), v.ctypes.data_as(L.P32),
                                            len(v), out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def free(self) -> None:
        if self.handle:
            L.lib.mg_matrix_filter_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
