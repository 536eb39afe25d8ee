"""Shared pytest configuration.

Marker ``gpu``: the test needs a CUDA GPU (sm_100a) and calls the product
through its C ABI (libmrt.so). Everything else runs on CPU.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); runs the product through its C ABI")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    from oracle import build_oracle
    build_oracle.build()
    return oracle


@pytest.fixture(scope="session")
def mrt_lib():
    import miniraytrace_b200 as mrt
    from miniraytrace_b200 import build
    build.build()
    return mrt


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(mrt_lib):
    """Asserts a GPU is present (gpu tests must not silently pass without one)."""
    assert gpu_available(), "gpu-marked test run without a CUDA device"
    return mrt_lib
