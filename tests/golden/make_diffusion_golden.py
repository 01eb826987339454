"""Tune diffusion and tracked tunes from the reference library itself (oracle/_ref), as fixtures.

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_diffusion_golden.py

Ring: the 4D DBA (no cavity, radiation off).  ALine::trackDiffusion (aline.cpp:716-779) on
points along two lines in (x, y), from well inside the dynamic aperture to beyond it, for
NTURN turns (rounded up to a power of two, 1,024), and ALine::tracktune (aline.cpp:1159-1186)
at three amplitudes.  Writes diffusion.npz: x0, y0, nux, nuy, dif, total, and the tracktune
points and tunes.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NTURN = 1000
TUNE_PTS = [(1e-3, 5e-4), (5e-3, 2e-3), (1e-2, 1e-3)]


def points():
    a = np.array([0.5, 1, 2, 3, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 25, 30]) * 1e-3
    x0 = np.concatenate([a, a])
    y0 = np.concatenate([0.4 * a, 1e-5 + 0 * a])
    return x0, y0


def main():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, LT.dba_4d_ring())
    line = O.RefLine(path)
    os.unlink(path)
    O.ref().ref_set_threads(1)
    x0, y0 = points()
    nux, nuy, dif, tot = line.trackDiffusion(NTURN, x0, y0)
    tunes = np.array([line.tracktune(NTURN, x, y) for x, y in TUNE_PTS])
    np.savez_compressed(os.path.join(HERE, "diffusion.npz"), x0=x0, y0=y0, nux=nux, nuy=nuy, dif=dif,
                        total=np.array([tot]), nturn=np.array([NTURN]), tune_pts=np.array(TUNE_PTS),
                        tunes=tunes)
    print("nux", nux, "\nnuy", nuy, "\ndif", dif, "\ntotal", tot, "\ntunes", tunes)


if __name__ == "__main__":
    main()
