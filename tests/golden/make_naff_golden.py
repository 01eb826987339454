"""Tune fixtures from the reference's own naff (oracle/_ref), for the engine's host NAFF.

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_naff_golden.py

Writes naff.npz: turn-by-turn records (synthetic lines with harmonics and noise, and x / y of
particles tracked through the 32-cell FODO by the oracle), the frequency windows, and the
reference's frequencies.
"""
from __future__ import annotations

import ctypes as C
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import oracle as O
    LT = importlib.import_module("accel-plus_b200.lattices")
    ref = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libaccel_ref.so"))
    ref.ref_naff.restype = C.c_double
    ref.ref_naff.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double]
    rng = np.random.default_rng(21)
    recs, lows, his = [], [], []
    n = 1024
    i = np.arange(n)
    for nu, amp2 in ((0.2371, 0.1), (0.4123, 0.3), (0.0817, 0.05)):
        x = np.cos(2 * np.pi * nu * i + 0.3) + amp2 * np.cos(2 * np.pi * 2 * nu * i) + 1e-3 * rng.normal(size=n)
        recs.append(x)
        lows.append(0.0)
        his.append(0.5)
    ring = LT.fodo_ring()
    r = np.zeros((2, 6))
    r[:, 0] = [1e-3, 4e-3]
    r[:, 2] = [5e-4, 1e-3]
    xs, ys = [], []
    for t in range(n):
        xs.append(r[:, 0].copy())
        ys.append(r[:, 2].copy())
        O.port_track(ring, r, 1)
    xs, ys = np.array(xs).T, np.array(ys).T
    for k in range(2):
        recs += [xs[k], ys[k]]
        lows += [0.1, 0.1]
        his += [0.5, 0.5]
    out = []
    for x, lo, hi in zip(recs, lows, his):
        buf = np.ascontiguousarray(x, dtype=np.float64).copy()
        out.append(ref.ref_naff(len(buf), buf.ctypes.data, lo, hi))
    np.savez_compressed(os.path.join(HERE, "naff.npz"), records=np.array(recs), xlow=np.array(lows),
                        xhi=np.array(his), nu=np.array(out))
    print("nu", out)


if __name__ == "__main__":
    main()
