"""Test configuration: the `gpu` marker and shared fixtures.

CPU tests (-m "not gpu") cover the oracle against the reference's known
answers, the voxelizer, the host logic and the C-ABI exports; GPU tests
(-m gpu) run the CUDA engine against the oracle through the C ABI.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the engine library (when nvcc is present) and the oracle once."""
    from oracle.build import build_oracle

    build_oracle()
    lib = ROOT / "simlab_b200" / "libsimlab_lbm.so"
    if not lib.exists():
        from simlab_b200.build import build_library

        build_library()
    yield
