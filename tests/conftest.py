"""Shared fixtures. GPU tests carry ``@pytest.mark.gpu``; everything else runs on a CPU-only host."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "molecular-dynamics_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a) and the built libmdgpu.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def golden():
    def load(name: str):
        return np.load(os.path.join(GOLDEN, name + ".npz"))

    return load


@pytest.fixture(scope="session")
def md():
    """The product through its C-ABI (ctypes over libmdgpu.so). Fails, never skips, when the library or the
    GPU is missing: a GPU test must not pass on a fallback."""
    import mdgpu

    if mdgpu.device_count() < 1:
        raise RuntimeError("no CUDA device visible to libmdgpu")
    return mdgpu
