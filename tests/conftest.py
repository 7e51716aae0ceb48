"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and call the product
through its C ABI (n-body-simulation_b200/lib/libnbx.so); the CPU checker
(oracle/) is only ever the reference side of a comparison."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "n-body-simulation_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_ref.npz")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def nbx():
    lib = os.path.join(PKG, "lib", "libnbx.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)
    import nbx as m
    m.lib()
    return m


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def same_bits(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def rel_err(ax, ay, bx, by):
    """|a - b| / max(|b|, 1e-30) per element (vecRelError, CheckCuda.cu:56-61)."""
    ax, ay, bx, by = (np.asarray(v, np.float64) for v in (ax, ay, bx, by))
    return np.hypot(ax - bx, ay - by) / np.maximum(np.hypot(bx, by), 1e-30)
