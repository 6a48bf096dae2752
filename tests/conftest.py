import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def _has_gpu() -> bool:
    try:
        import ctypes

        import ed_lattice_b200._edgpu_lib as L
        n = ctypes.c_int()
        return L.lib().edg_device_count(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


HAS_GPU = None


def pytest_collection_modifyitems(config, items):
    global HAS_GPU
    if HAS_GPU is None:
        HAS_GPU = _has_gpu()
    if HAS_GPU:
        return
    # `-m gpu` asks for the GPU parity tests explicitly: without a device they must fail,
    # not skip, so that a missing GPU or a broken libedgpu.so cannot pass silently.
    if "gpu" in (config.option.markexpr or "") and "not gpu" not in config.option.markexpr:
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
