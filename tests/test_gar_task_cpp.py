"""The C++ GARMatch task mirror (host/matrixgraph.h) over the C-ABI."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "matrixgraph_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("gar_task") / "gar_task")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(PKG, "host"), os.path.join(ROOT, "tests", "gar_task_main.cpp"),
                    os.path.join(PKG, "host", "matrixgraph.cpp"), "-o", out, "-L", PKG,
                    "-lmg_subiso", f"-Wl,-rpath,{PKG}"], check=True)
    return out


def run(exe, mode):
    r = subprocess.run([exe, mode], capture_output=True, text=True, check=True)
    lines = r.stdout.strip().splitlines()
    head = dict(kv.split("=") for kv in lines[0].split())
    rows = [tuple(int(x) for x in ln.split()[1:]) for ln in lines[1:-1]]
    ids = [int(x) for x in lines[-1].split()[1:]]
    return {k: int(v) for k, v in head.items()}, rows, ids


def test_empty_pattern_needs_no_gpu(exe):
    head, rows, ids = run(exe, "no_edges")
    assert head == {"status": 0, "num_conditions": 1, "row_size": 0, "match_size": 0}
    assert rows == [] and ids == []


def test_example_without_gpu_reports_cuda_status(exe):
    from conftest import gpu_count
    if gpu_count() > 0:
        pytest.skip("a GPU is present")
    head, rows, ids = run(exe, "example")
    assert head["status"] == -6 and head["num_conditions"] == 1 and rows == []


@pytest.mark.gpu
def test_example_on_gpu(exe):
    head, rows, ids = run(exe, "example")
    assert head == {"status": 0, "num_conditions": 2, "row_size": 4, "match_size": 5}
    assert rows == [(126, 0, 0, 0, 1), (126, 1, 1, 1, 2), (138, 0, 0, 3, 1),
                    (138, 1, 1, 4, 1)]
    assert ids == [126, 183, 115407, 138, 192]
