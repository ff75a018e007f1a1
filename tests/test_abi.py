"""The C-ABI library: symbols, error behaviour without a GPU, host logic."""
import ctypes as C
import os
import re

import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b((?:mg|matrixgraph)_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = header_functions()
    assert len(names) >= 20 and "matrixgraph_gar_match" in names
    for n in names:
        assert hasattr(L.lib, n), n
        assert n in L.EXPORTED, f"{n} has no ctypes signature"


def test_version_and_defaults():
    assert b"sm_100a" in L.lib.mg_version()
    o = L.default_opts()
    assert o.order == L.MG_ORDER_REFERENCE and o.filters == L.MG_FILTER_ALL


def test_null_arguments_are_errors_not_crashes():
    c = C.c_uint64()
    assert L.lib.mg_subiso_count(None, None, None, C.byref(c)) == L.MG_E_ARG
    assert b"null" in L.lib.mg_last_error()
    assert L.lib.mg_csr_dir_open(None, None, None) == L.MG_E_ARG
    assert L.lib.mg_graph_upload(None, 0, None) == L.MG_E_ARG


def test_upload_without_gpu_fails_loudly():
    from conftest import gpu_count
    if gpu_count() > 0:
        pytest.skip("a GPU is present")
    g = mg.chung_lu(200, avg_deg=4)
    with pytest.raises(L.MGError) as e:
        mg.DeviceGraph(g)
    assert e.value.code in (L.MG_E_CUDA, L.MG_E_ARG)


def test_query_limits():
    with pytest.raises(L.MGError) as e:
        mg.CSRGraph.query(17, [(0, 1)], [0] * 17)
    assert e.value.code == L.MG_E_LIMIT
    q = mg.CSRGraph.query(3, [(0, 1), (1, 2)], [0, 0, 0])
    with pytest.raises(L.MGError):
        mg.plan_order(q, order="strong")  # needs a graph handle
    assert sorted(mg.plan_order(q, given_order=[2, 0, 1])) == [0, 1, 2]
    with pytest.raises(L.MGError) as e:
        mg.plan_order(q, given_order=[0, 0, 1])
    assert e.value.code == L.MG_E_ARG


def test_reference_order_examples():
    # 4-cycle 0-1-2-3-0: CSR edge order (0,1),(0,3),(1,0),(1,2),... -> 0,1,3,2
    q = mg.CSRGraph.query(4, [(0, 1), (1, 2), (2, 3), (3, 0)], [0] * 4)
    assert mg.plan_order(q) == [0, 1, 3, 2]
    # disconnected pattern: every vertex still placed
    q = mg.CSRGraph.query(5, [(0, 1), (3, 4)], [0] * 5)
    order = mg.plan_order(q)
    assert sorted(order) == list(range(5)) and order[:2] == [0, 1]


def test_shard_roots_partition():
    for n in (0, 1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            parts = [mg.shard_roots(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            for (a, b), (c, d) in zip(parts, parts[1:]):
                assert b == c and a <= b


def test_subiso_exec_flags():
    import subprocess
    exe = os.path.join(ROOT, "matrixgraph_b200", "subiso_exec")
    r = subprocess.run([exe, "-g", "x/"], capture_output=True, text=True)
    assert r.returncode != 0 and "-p" in r.stderr
    r = subprocess.run([exe, "-p", "/nonexistent/", "-g", "/nonexistent/"], capture_output=True,
                       text=True)
    assert r.returncode != 0 and "Error" in r.stderr
