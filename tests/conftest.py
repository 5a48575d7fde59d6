"""Shared pytest setup: import paths, the `gpu` marker, common fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "aether-core-engine_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
for p in (PKG_DIR, ORACLE_DIR, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def af():
    """The product package with its CUDA library loaded (GPU tests only)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import aether_fluid
    aether_fluid.load()
    return aether_fluid


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O
