"""Test configuration: the `gpu` marker and shared helpers.

Tests marked ``gpu`` need a CUDA device and the built library; everything else
runs on the CPU (the oracle, the codecs, the host-side set-up and the library's
exports).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and libspgrid_gpu_solver.so")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def native_lib():
    from spgrid_topo_opt_b200 import build, native
    build.build()
    return native.load()
