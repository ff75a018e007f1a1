"""Builds libmg_subiso.so (CUDA for sm_100a + host C++) in-tree, and the
C++ host programs (subiso_exec) that link it.

Run as ``python -m matrixgraph_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmg_subiso.so")
EXE = os.path.join(PKG, "subiso_exec")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-Wall", "-Wno-unused-function",
             "-I", INCLUDE, "-I", CSRC]


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu") or f.endswith(".cpp"):
            out.append(os.path.join(CSRC, f))
    return out


def _headers():
    hs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC)
           if f.endswith(".h") or f.endswith(".cuh")]
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source that changed and links libmg_subiso.so."""
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if not _stale(obj, [src] + headers) and not ptxas_info:
            continue
        if src.endswith(".cu"):
            cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + \
                ["-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
        jobs.append(cmd)
    logs = []
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for out in ex.map(_run, jobs):
                logs.append(out)
    if _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    _build_host(nvcc)
    text = "\n".join(logs)
    if verbose and text:
        print(text)
    return text


def _build_host(nvcc: str) -> None:
    """subiso_exec: the reference's CLI over the C-ABI (host C++ only)."""
    if not os.path.isdir(HOST):
        return
    srcs = [os.path.join(HOST, f) for f in sorted(os.listdir(HOST)) if f.endswith(".cpp")]
    hdrs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    if not srcs:
        return
    incs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    if not _stale(EXE, srcs + hdrs + incs + [LIB]):
        return
    _run(["g++"] + CXX_FLAGS + ["-I", HOST] + srcs + ["-o", EXE, "-L", PKG, "-lmg_subiso",
                                                       "-Wl,-rpath,$ORIGIN"])


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv) or "up to date")
