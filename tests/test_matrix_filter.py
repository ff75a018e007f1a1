"""The lossy MatrixFilter on the CPU: the reference's matrix container, the
restated filter against a float64 computation, shape checks of the loader
(they fail before any device work) and the subiso_exec flags."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import matrixgraph_b200 as mg
from matrixgraph_b200 import _lib as L
from matrixgraph_b200.matrix_filter import MatrixFilter, read_matrix, write_matrix
from oracle import matrix_filter as OMF


def weights(rng, k, n, dim=8, hidden=16, keep_frac=0.5):
    """Random filter matrices; b2 puts about keep_frac of the (u=0, v) pairs
    above the threshold."""
    q = rng.normal(size=(k, dim)).astype(np.float32)
    d = rng.normal(size=(n, dim)).astype(np.float32)
    w1 = (rng.normal(size=(hidden, dim)) / np.sqrt(dim)).astype(np.float32)
    b1 = rng.normal(size=(1, hidden)).astype(np.float32) * 0.1
    w2 = rng.normal(size=(hidden, 1)).astype(np.float32)
    z = OMF.logits(q, d, w1, b1, w2, np.zeros((1, 1), np.float32), 0, np.arange(n))
    b2 = np.float32(np.log(0.1 / 0.9) - np.quantile(z, 1 - keep_frac))
    return [q, d, w1, b1, w2, np.array([[b2]], np.float32)]


def save(tmp, mats):
    dirs = []
    for i, m in enumerate(mats):
        d = os.path.join(str(tmp), f"m{i + 1}") + "/"
        write_matrix(d, m)
        dirs.append(d)
    return dirs


def test_container_round_trip(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    write_matrix(str(tmp_path / "m"), a)
    assert np.array_equal(read_matrix(str(tmp_path / "m")), a)
    meta = (tmp_path / "m" / "meta.yaml").read_text()
    assert "x: 3" in meta and "y: 4" in meta


def test_restated_filter_against_float64():
    rng = np.random.default_rng(1)
    mats = weights(rng, 4, 500)
    keep, unsure = OMF.keep(*mats, 2, np.arange(500))
    q, d, w1, b1, w2, b2 = [m.astype(np.float64) for m in mats]
    z1 = np.maximum(((q[2][None, :] - d) ** 2) @ w1.T + b1, 0)
    z2 = z1 @ w2[:, 0] + b2[0, 0]
    s = 1 / (1 + np.exp(-z2))
    clear = np.abs(s - 0.1) > 1e-4
    assert np.array_equal(keep[clear], (s >= 0.1)[clear])
    assert 0.2 < keep.mean() < 0.8
    assert not unsure.any()


def test_loader_rejects_bad_shapes_before_the_device(tmp_path):
    rng = np.random.default_rng(2)
    good = weights(rng, 3, 50)
    cases = {
        "width": (1, np.zeros((50, 7), np.float32)),      # data width != query width
        "hidden": (2, np.zeros((65, 8), np.float32)),     # more than 64 hidden units
        "w2": (4, np.zeros((16, 2), np.float32)),         # W2 not hidden x 1
        "b2": (5, np.zeros((1, 2), np.float32)),          # b2 not one value
    }
    for name, (i, bad) in cases.items():
        mats = list(good)
        mats[i] = bad
        dirs = save(tmp_path / name, mats)
        with pytest.raises(L.MGError) as e:
            MatrixFilter.load(dirs)
        assert e.value.code == L.MG_E_FORMAT, name
    dirs = save(tmp_path / "short", good)
    with open(os.path.join(dirs[1], "embedding.bin"), "r+b") as f:
        f.truncate(100)
    with pytest.raises(L.MGError) as e:
        MatrixFilter.load(dirs)
    assert e.value.code == L.MG_E_FORMAT
    ok = save(tmp_path / "ok", good)
    with pytest.raises(L.MGError) as e:
        MatrixFilter.load(ok[:5] + [str(tmp_path / "absent") + "/"])
    assert e.value.code == L.MG_E_IO
    arr = (C.c_char_p * 6)(*([b"x/"] * 5 + [b""]))
    h = C.c_void_p()
    assert L.lib.mg_matrix_filter_load(arr, 0, C.byref(h)) == L.MG_E_ARG


def test_subiso_exec_matrix_flags(tmp_path):
    exe = os.path.join(os.path.dirname(mg.__file__), "subiso_exec")
    r = subprocess.run([exe, "-p", "p/", "-g", "g/", "-m1", "a/", "-m2", "b/"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "-m1 .. -m6" in r.stderr
    (tmp_path / "list.txt").write_text("p/\n")
    args = [exe, "-g", "g/", "-batch", str(tmp_path / "list.txt")]
    for i in range(1, 7):
        args += [f"-m{i}", f"m{i}/"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "single pattern" in r.stderr


def test_options_carry_the_filter_handle():
    o, _ = mg.make_opts(matrix_filter=12345)
    assert o.matrix_filter == 12345
    o, _ = mg.make_opts()
    assert not o.matrix_filter
