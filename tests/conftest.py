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


def _scale(r: np.ndarray) -> np.ndarray:
    live = ~np.isnan(r[:, 0])
    sc = np.sqrt(np.mean(r[live] ** 2, axis=0)) if live.any() else np.ones(6)
    sc[sc == 0] = 1.0
    return sc


def rel_err_each(a: np.ndarray, b: np.ndarray, scale: np.ndarray) -> np.ndarray:
    """Per-particle max over coordinates of |a - b| / scale (NaN rows give inf)."""
    with np.errstate(invalid="ignore"):
        d = np.abs(a - b) / scale
    out = np.max(d, axis=1)
    out[np.isnan(out)] = np.inf
    return out


class Sensitivity:
    """The oracle's view of a grid: loss turns, final states, and which points are on the chaotic
    aperture boundary or on irregular orbits, found by re-tracking with x and y perturbed by
    +-eps (relative, plus eps x 1 mm absolute)."""

    def __init__(self, O, ring, grid: np.ndarray, nturn: int, nx: int, ny: int, eps: float = 1e-12):
        self.final = grid.copy()
        self.lt = O.port_track(ring, self.final, nturn, nthreads=8)
        sc = _scale(self.final)
        sens = np.zeros(len(grid), dtype=bool)
        amp = np.zeros(len(grid))
        for sgn in (1.0, -1.0):
            g = grid.copy()
            for k in (0, 2):
                g[:, k] = g[:, k] * (1 + sgn * eps) + sgn * eps * 1e-3
            lt = O.port_track(ring, g, nturn, nthreads=8)
            sens |= lt != self.lt
            amp = np.maximum(amp, rel_err_each(g, self.final, sc) / eps)
        fate = (self.lt < 0).reshape(ny, nx)
        near = np.zeros_like(fate)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ys = slice(max(0, dy), ny + min(0, dy))
                yd = slice(max(0, -dy), ny + min(0, -dy))
                xs = slice(max(0, dx), nx + min(0, dx))
                xd = slice(max(0, -dx), nx + min(0, -dx))
                near[yd, xd] |= fate[ys, xs] != fate[yd, xd]
        self.boundary = sens | near.ravel()
        # regular: survives, and a 1e-12 perturbation stays below 1e-9 at the end
        self.regular = (self.lt < 0) & ~self.boundary & (amp * eps < 1e-9)
        self.scale = sc


def check_loss_turns(lt: np.ndarray, ref_lt: np.ndarray, allowed: np.ndarray, max_frac: float = 0.25):
    """Loss turns identical except at chaotic-boundary points, which stay a minority."""
    bad = lt != ref_lt
    assert not np.any(bad & ~allowed), np.nonzero(bad & ~allowed)
    assert bad.mean() <= max_frac
