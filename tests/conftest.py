"""Test configuration: import paths, the `gpu` marker, shared fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(ROOT, "highordermrisim.jl_b200")
for p in (PKG_ROOT, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100) and runs libhoms kernels")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.build()
    return o


@pytest.fixture(scope="session")
def homs_lib():
    from homs import build
    build.build()
    from homs import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def gpu_context(homs_lib):
    from homs import _lib
    ctx = _lib.Context(0)
    yield ctx
    ctx.close()


def nrmse(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
