"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the built libaerosim.so; everything else
runs on the CPU (the oracle, host logic, and the C-ABI export check).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and libaerosim.so")
    config.addinivalue_line("markers", "slow: long CPU-only oracle run")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu_engine_cls():
    """LBMEngine class; fails (not skips) when the library is missing on a GPU box."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from aerosim_b200 import _native, engine
    _native.load()
    return engine.LBMEngine
