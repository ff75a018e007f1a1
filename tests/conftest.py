"""Test configuration: the `gpu` marker and the in-tree builds."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # Both libraries are built in-tree before any test imports them.
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_mg_build", os.path.join(ROOT, "matrixgraph_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()


def gpu_count() -> int:
    """CUDA devices visible through the driver API (0 without a driver)."""
    import ctypes
    try:
        cu = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return 0
    if cu.cuInit(0) != 0:
        return 0
    n = ctypes.c_int(0)
    if cu.cuDeviceGetCount(ctypes.byref(n)) != 0:
        return 0
    return n.value


def pytest_collection_modifyitems(config, items):
    if gpu_count() > 0:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
