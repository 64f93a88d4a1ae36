"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the built libmobyb200.so; they are
the parity tests of the CUDA path against the CPU oracle.  Everything else
runs on the CPU (oracle known-answer tests, host-side logic, C-ABI exports).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmobyb200.so")


def _have_gpu() -> bool:
    try:
        import mobydiff_b200 as M
        return M.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O
