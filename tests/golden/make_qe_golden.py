"""Quantum-excitation statistics from the reference library itself (oracle/_ref), as fixtures.

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_qe_golden.py [growth | equilibrium [BATCH]]

The 18-cell DBA with radiation + quantum excitation (RADQE) and the cavity on; every particle
starts at the origin, so after T turns the spread is entirely the excitation's (the mean carries
the deterministic energy loss and synchrotron motion).  The reference draws its normal deviates
from rand(), which is shared by OpenMP threads; to keep the draws race-free it runs here as
PROCS single-threaded processes with distinct srand seeds, PER particles each.

growth       qe_moments.npz: the moments (mean[6], sigma[6], cross[6], live count) of all
             PROCS x PER particles after TURNS turns from the origin (about two minutes).
equilibrium  qe_equilibrium.npz: a Gaussian bunch (sigma_z 3 mm, sigma_delta 1e-3, 10 nm / 10 pm
             emittances matched to the ring-entrance Twiss) tracked for EQ_TURNS turns, which is
             about three transverse damping times; the moments (mean, sigma, cross, live count)
             of all particles every EQ_EVERY turns (about an hour on 8 cores).  BATCH b > 0 draws
             other particles and other srand seeds and writes qe_equilibrium_b<b>.npz, so that
             independent batches can be pooled.
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
PROCS, PER, TURNS = 8, 2048, 200
EQ_PER, EQ_TURNS, EQ_EVERY, EQ_SEED = 1024, 10000, 1000, 5


def worker(args):
    seed, path = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A = importlib.import_module("accel-plus_b200")
    line = O.RefLine(path)
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    O.ref().ref_srand(seed)
    r = np.zeros((PER, 6))
    line.track(r, TURNS, threads=1)
    return r


def worker_eq(args):
    seed, path, r = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A = importlib.import_module("accel-plus_b200")
    line = O.RefLine(path)
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    O.ref().ref_srand(seed)
    snaps = []
    for _ in range(EQ_TURNS // EQ_EVERY):
        line.track(r, EQ_EVERY, threads=1)
        snaps.append(r.copy())
    return np.stack(snaps)


def entrance_m66(A, O, ring):
    """One-turn matrix of the ring at its entrance, radiation and cavity off (the reference's
    central difference)."""
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, ring)
    line = O.RefLine(path)
    os.unlink(path)
    line.set_flags(rad=0, cavity=0)
    return line.m66(0.0, 1e-8)


def moments(r):
    live = ~np.isnan(r[:, 0])
    x = r[live]
    m = x.mean(axis=0)
    d = x - m
    sig = np.sqrt((d * d).mean(axis=0))
    pairs = [(0, 1), (2, 3), (0, 5), (1, 5), (2, 4), (3, 4)]
    cross = np.array([(d[:, a] * d[:, b]).mean() for a, b in pairs])
    return m, sig, cross, int(live.sum())


def equilibrium(A, LT, path, batch=0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ring = LT.dba_ring()
    m66 = entrance_m66(A, O, ring)
    r0 = LT.matched_bunch_particles(PROCS * EQ_PER, m66, seed=EQ_SEED + batch)
    jobs = [(2000 + 100 * batch + k, path, r0[k * EQ_PER:(k + 1) * EQ_PER].copy()) for k in range(PROCS)]
    with mp.get_context("spawn").Pool(PROCS) as pool:
        parts = pool.map(worker_eq, jobs)
    snaps = np.concatenate(parts, axis=1)  # [snapshot, particle, 6]
    mom = [moments(s) for s in snaps]
    turns = EQ_EVERY * (1 + np.arange(len(snaps)))
    name = "qe_equilibrium.npz" if batch == 0 else f"qe_equilibrium_b{batch}.npz"
    np.savez_compressed(os.path.join(HERE, name),
                        mean=np.array([m[0] for m in mom]), sigma=np.array([m[1] for m in mom]),
                        cross=np.array([m[2] for m in mom]), nlive=np.array([m[3] for m in mom]),
                        turns=turns, m66=m66, seed=np.array([EQ_SEED + batch]), n=np.array([PROCS * EQ_PER]))
    sig = np.array([m[1] for m in mom])
    print("turns", turns, "\nsigma\n", sig, "\nlive", [m[3] for m in mom])


def main():
    sys.path.insert(0, ROOT)
    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, LT.dba_ring())
    if len(sys.argv) > 1 and sys.argv[1] == "equilibrium":
        equilibrium(A, LT, path, int(sys.argv[2]) if len(sys.argv) > 2 else 0)
        os.unlink(path)
        return
    with mp.get_context("spawn").Pool(PROCS) as pool:
        parts = pool.map(worker, [(1000 + k, path) for k in range(PROCS)])
    os.unlink(path)
    r = np.concatenate(parts)
    m, sig, cross, nl = moments(r)
    np.savez_compressed(os.path.join(HERE, "qe_moments.npz"), mean=m, sigma=sig, cross=cross,
                        nlive=np.array([nl]), n=np.array([PROCS * PER]), turns=np.array([TURNS]))
    print("mean", m, "\nsigma", sig, "\ncross", cross, "\nlive", nl)


if __name__ == "__main__":
    main()
