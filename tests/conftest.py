"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on a CPU-only machine."""
from __future__ import annotations

import importlib
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(ROOT, "accel-plus_b200", "libaccelgpu.so")
    port = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "accel-plus_b200"), "-j8"], check=True)
    if not os.path.exists(port):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def A():
    return importlib.import_module("accel-plus_b200")


@pytest.fixture(scope="session")
def LT():
    return importlib.import_module("accel-plus_b200.lattices")


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


@pytest.fixture(scope="session")
def G():
    return dict(np.load(os.path.join(GOLDEN, "golden.npz")))


@pytest.fixture(scope="session")
def MG():
    sys.path.insert(0, GOLDEN)
    import make_golden
    return make_golden


@pytest.fixture(scope="session")
def ctx(A):
    if A.device_count() < 1:
        pytest.skip("no CUDA device")
    c = A.Context(0)
    yield c
    c.close()


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    """Bitwise equality, NaN payloads included."""
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(np.int64),
                                                 np.ascontiguousarray(b).view(np.int64))


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a-b| over live particles, each coordinate scaled by its RMS over the live set
    (relative error for coordinates that pass through zero)."""
    live = ~np.isnan(a[:, 0]) & ~np.isnan(b[:, 0])
    if not live.any():
        return 0.0
    x, y = a[live], b[live]
    scale = np.sqrt(np.mean(y * y, axis=0))
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(x - y) / scale))
