"""Reference outputs for the WigTable element (oracle/_ref).

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_wigtable_golden.py

Each case is one WigTable element whose kick tables are registered with the engine, written with
the engine's lattice writer at 17 digits, then read and tracked for one turn by the reference
library (AWigTable::create and AWigTable::pass, accel.cpp:1294-1377).  The particles cover the
grid and the region outside it, where the reference extrapolates from the edge cells.  Writes
wigtable.npz: elem_in, and per case the grid, the two tables and the tracked particles.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def tables():
    """name -> (length, nslice, xl, yl, xkick, ykick); kicks are [len(yl)][len(xl)]."""
    rng = np.random.default_rng(7)
    out = {}
    xl = np.linspace(-0.02, 0.02, 11)
    yl = np.linspace(-0.01, 0.01, 5)
    X, Y = np.meshgrid(xl, yl)
    xk = 1e-4 * np.sin(60 * X) * np.cos(40 * Y) + 2e-6 * rng.standard_normal(X.shape)
    yk = 5e-5 * np.cos(50 * X) * np.sin(70 * Y) + 2e-6 * rng.standard_normal(X.shape)
    out["thin"] = (0.0, 1, xl, yl, xk, yk)
    out["thick"] = (1.2, 8, xl, yl, xk, yk)
    # uneven grid, y descending, a larger table
    xl2 = np.sort(rng.uniform(-0.03, 0.03, 23))
    yl2 = np.sort(rng.uniform(-0.012, 0.012, 9))[::-1].copy()
    X2, Y2 = np.meshgrid(xl2, yl2)
    xk2 = 3e-4 * X2 * Y2 / 1e-4 + 1e-6 * rng.standard_normal(X2.shape)
    yk2 = -2e-4 * (X2 ** 2 - Y2 ** 2) / 1e-4 + 1e-6 * rng.standard_normal(X2.shape)
    out["uneven"] = (0.8, 3, xl2, yl2, xk2, yk2)
    return out


def particles():
    rng = np.random.default_rng(11)
    n = 40
    r = np.zeros((n, 6))
    r[:, 0] = rng.uniform(-0.035, 0.035, n)   # part of them outside the grids
    r[:, 1] = rng.uniform(-1e-3, 1e-3, n)
    r[:, 2] = rng.uniform(-0.016, 0.016, n)
    r[:, 3] = rng.uniform(-1e-3, 1e-3, n)
    r[:, 4] = rng.uniform(-1e-3, 1e-3, n)
    r[:, 5] = rng.uniform(-2e-3, 2e-3, n)
    r[0, :] = 0.0                              # on a grid line
    r[1, 0], r[1, 2] = 0.02, 0.01              # on the last grid point
    return r


def elems(A, name, spec):
    length, nslice, xl, yl, xk, yk = spec
    tid = A.wigtable(xl, yl, xk, yk)
    return [A.elem(A.WIGTABLE, "WT", length, nslice=nslice, f=[tid])]


def main():
    import oracle as O
    A = importlib.import_module("accel-plus_b200")
    r0 = particles()
    out = {"elem_in": r0}
    for name, spec in tables().items():
        fd, path = tempfile.mkstemp(suffix=".lat")
        os.close(fd)
        A.write_lattice(path, elems(A, name, spec))
        line = O.RefLine(path)
        os.unlink(path)
        r = r0.copy()
        line.track(r, 1)
        out[f"elem_{name}"] = r
        print(name, np.abs(r - r0).max())
    np.savez_compressed(os.path.join(HERE, "wigtable.npz"), **out)


if __name__ == "__main__":
    main()
