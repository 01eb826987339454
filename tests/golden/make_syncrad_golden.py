"""The reference's lumped radiation element (ASyncRad, accel.cpp:1806-1854) in its two random
modes, as statistical fixtures from the reference library itself (oracle/_ref).

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_syncrad_golden.py

Ring: the 4D DBA (no cavity, bend radiation off) with one SyncRad element of length 0.2 m at
its end (3 GeV, U0 0.9 MeV, Jx 1.3, Jy 1.0, emittances 2 nm / 20 pm, sigma_delta 1e-3, beta
5 m / 3 m).  ALine::set_rad_onoff maps the deck's radiation flag onto it (aline.cpp:273-289):
LUMP turns damping and excitation on, LUMP_QE excitation alone (LUMP_DAMP, deterministic, is an
element case of golden.npz).  Every particle starts at the origin, so the spread after TURNS
turns is the excitation's.  The reference draws its deviates from rand(), shared by OpenMP
threads, so it runs as PROCS single-threaded processes with distinct srand seeds, PER particles
each.  Writes syncrad_lump.npz: for each mode the moments (mean[6], sigma[6], cross[6], live
count) of all PROCS x PER particles.
"""
from __future__ import annotations

import importlib
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROCS, PER, TURNS = 8, 2048, 300
SYNCRAD_F = [3000.0, 0.9, 1.3, 1.0, 2e-9, 2e-11, 1e-3, 5.0, 3.0]


def ring(A, LT):
    """The 4D DBA with the lumped radiation element at its end (radiation flag set by the caller)."""
    return LT.dba_4d_ring() + [A.elem(A.SYNCRAD, "SR", 0.2, f=SYNCRAD_F)]


def moments(r):
    live = ~np.isnan(r[:, 0])
    x = r[live]
    m = x.mean(axis=0)
    d = x - m
    sig = np.sqrt((d * d).mean(axis=0))
    pairs = [(0, 1), (2, 3), (0, 5), (1, 5), (2, 4), (3, 4)]
    cross = np.array([(d[:, a] * d[:, b]).mean() for a, b in pairs])
    return m, sig, cross, int(live.sum())


def worker(args):
    seed, path, flag = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    line = O.RefLine(path)
    line.set_flags(rad=flag, cavity=0)
    O.ref().ref_srand(seed)
    r = np.zeros((PER, 6))
    line.track(r, TURNS, threads=1)
    return r


def main():
    sys.path.insert(0, ROOT)
    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, ring(A, LT))
    out = {"n": np.array([PROCS * PER]), "turns": np.array([TURNS]), "syncrad_f": np.array(SYNCRAD_F)}
    for name, flag, base in (("lump", A.RAD_LUMP, 3000), ("lump_qe", A.RAD_LUMP_QE, 4000)):
        with mp.get_context("spawn").Pool(PROCS) as pool:
            parts = pool.map(worker, [(base + k, path, flag) for k in range(PROCS)])
        m, sig, cross, nl = moments(np.concatenate(parts))
        out[f"{name}_mean"], out[f"{name}_sigma"], out[f"{name}_cross"] = m, sig, cross
        out[f"{name}_nlive"] = np.array([nl])
        print(name, "sigma", sig, "mean", m, "live", nl, flush=True)
    os.unlink(path)
    np.savez_compressed(os.path.join(HERE, "syncrad_lump.npz"), **out)


if __name__ == "__main__":
    main()
