"""subiso_exec flag handling on the CPU: errors before any device work, the
batch list, and the loud failure of the device step without a GPU."""
import os
import subprocess

import pytest

import matrixgraph_b200 as mg

EXE = os.path.join(os.path.dirname(mg.__file__), "subiso_exec")


def run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=120)


@pytest.fixture(scope="module")
def dirs(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    g = mg.chung_lu(300, avg_deg=5, n_labels=3)
    g.Write(str(d / "g") + "/")
    for i, (edges, labels) in enumerate([([(0, 1), (1, 2), (2, 0)], [0, 1, 2]),
                                         ([(0, 1), (1, 2)], [0, 0, 1])]):
        mg.CSRGraph.query(3, edges, labels).Write(str(d / f"p{i}") + "/")
    (d / "list.txt").write_text(f"{d}/p0/\n# a comment\n\n{d}/p1/\n")
    (d / "bad.txt").write_text(f"{d}/p0/\n{d}/missing/\n")
    (d / "empty.txt").write_text("# nothing\n")
    return d


def test_flag_errors(dirs):
    assert run("-g", f"{dirs}/g/").returncode == 1                       # no -p, no -batch
    r = run("-p", f"{dirs}/p0/", "-g", f"{dirs}/g/", "-order", "fastest")
    assert r.returncode == 1 and "unknown order" in r.stderr
    r = run("-p", f"{dirs}/p0/", "-g", f"{dirs}/g/", "-order", "learned")
    assert r.returncode == 1 and "-model" in r.stderr
    r = run("-g", f"{dirs}/g/", "-batch", f"{dirs}/nope.txt")
    assert r.returncode == 1 and "cannot read the batch list" in r.stderr
    r = run("-g", f"{dirs}/g/", "-batch", f"{dirs}/empty.txt")
    assert r.returncode == 1 and "names no pattern" in r.stderr
    r = run("-p", f"{dirs}/p0/", "-g", f"{dirs}/g/", "-bogus", "1")
    assert r.returncode == 1 and "unknown flag" in r.stderr


def test_batch_list_reads_every_pattern_before_the_device(dirs):
    r = run("-g", f"{dirs}/g/", "-batch", f"{dirs}/bad.txt")
    assert r.returncode == 1 and "missing" in r.stderr


def test_device_step_fails_loudly_without_gpu(dirs):
    from conftest import gpu_count
    if gpu_count() > 0:
        pytest.skip("a GPU is present")
    for args in (("-p", f"{dirs}/p0/", "-g", f"{dirs}/g/"),
                 ("-g", f"{dirs}/g/", "-batch", f"{dirs}/list.txt", "-order", "strong")):
        r = run(*args)
        assert r.returncode == 1 and "Error" in r.stderr
