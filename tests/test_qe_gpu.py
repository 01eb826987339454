"""Quantum excitation (RADQE) against the reference, statistically.

The engine draws its normal deviates from a counter-based Philox stream, the reference from
rand(); only the statistics can agree.  Every particle starts at the origin of the 18-cell DBA
(radiation + QE, cavity on), so after 200 turns the spread is produced by the excitation alone.
The reference's moments over 16,384 particles are a fixture (tests/golden/qe_moments.npz, from
make_qe_golden.py); the engine tracks 262,144.  Bar: rms sizes within 2 %; means within four
combined standard errors; the x-delta correlation within 0.02; nobody lost; no vertical motion.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def moments(r):
    live = ~np.isnan(r[:, 0])
    x = r[live]
    m = x.mean(axis=0)
    d = x - m
    return m, np.sqrt((d * d).mean(axis=0)), (d[:, 0] * d[:, 5]).mean(), int(live.sum())


def test_quantum_excitation_statistics(A, ctx, LT):
    ref = np.load(os.path.join(GOLDEN, "qe_moments.npz"))
    n_ref, turns = int(ref["n"][0]), int(ref["turns"][0])
    line = A.Line(ctx, LT.dba_ring())
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    line.set_seed(20240611)
    n = 262144
    r = np.zeros((n, 6))
    line.track(r, turns)
    m, sig, cx5, nlive = moments(r)
    assert nlive == n and int(ref["nlive"][0]) == n_ref
    for k in (0, 1, 4, 5):
        assert abs(sig[k] - ref["sigma"][k]) <= 0.02 * ref["sigma"][k], (k, sig[k], ref["sigma"][k])
        se = np.sqrt(ref["sigma"][k] ** 2 / n_ref + sig[k] ** 2 / n)
        assert abs(m[k] - ref["mean"][k]) <= 4 * se, (k, m[k], ref["mean"][k], se)
    rho, rho_ref = cx5 / (sig[0] * sig[5]), ref["cross"][2] / (ref["sigma"][0] * ref["sigma"][5])
    assert abs(rho - rho_ref) <= 0.02, (rho, rho_ref)
    assert np.all(r[:, 2:4] == 0.0)

    # the same run without excitation has no spread at all: the test measures the excitation
    line.set_flags(rad=A.RAD_RAD, cavity=1)
    q = np.zeros((1024, 6))
    line.track(q, turns)
    assert np.all(q.max(axis=0) == q.min(axis=0))


def test_quantum_excitation_is_reproducible_and_seeded(A, ctx, LT):
    """Counter-based deviates: the same seed gives the same bits, another seed other bits."""
    line = A.Line(ctx, LT.dba_ring())
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    runs = []
    for seed in (7, 7, 8):
        line.set_seed(seed)
        r = np.zeros((4096, 6))
        line.track(r, 20)
        runs.append(r)
    assert np.array_equal(runs[0], runs[1])
    assert not np.array_equal(runs[0], runs[2])


def pooled(files, snap):
    """Mean and the second moments <xx>, <x'x'>, <xx'>, <x d>, <x' d>, <zz>, <dd> of several
    independent reference batches pooled at snapshot `snap`."""
    ns = [float(f["nlive"][snap]) for f in files]
    N = sum(ns)
    mu = sum(n * f["mean"][snap] for n, f in zip(ns, files)) / N

    def cov(a, b, f):
        if a == b:
            return f["sigma"][snap][a] ** 2
        pairs = [(0, 1), (2, 3), (0, 5), (1, 5), (2, 4), (3, 4)]
        return f["cross"][snap][pairs.index((a, b))]

    def pool(a, b):
        return sum(n * (cov(a, b, f) + (f["mean"][snap][a] - mu[a]) * (f["mean"][snap][b] - mu[b]))
                   for n, f in zip(ns, files)) / N
    return {k: pool(*k) for k in [(0, 0), (1, 1), (0, 1), (0, 5), (1, 5), (4, 4), (5, 5)]}, N


def emittance_x(c):
    """Horizontal emittance with the dispersive (delta-correlated) part of x and x' removed."""
    dd = c[(5, 5)]
    xx = c[(0, 0)] - c[(0, 5)] ** 2 / dd
    pp = c[(1, 1)] - c[(1, 5)] ** 2 / dd
    xp = c[(0, 1)] - c[(0, 5)] * c[(1, 5)] / dd
    return np.sqrt(xx * pp - xp * xp)


def test_quantum_excitation_equilibrium(A, ctx, LT):
    """Equilibrium emittance and bunch length after 10,000 turns (about three transverse damping
    times) of RADQE tracking from the matched Gaussian bunch (sigma_z 3 mm, sigma_delta 1e-3,
    10 nm / 10 pm), against the reference's moments pooled over its independent batches
    (tests/golden/qe_equilibrium*.npz): horizontal emittance, bunch length and energy spread within
    2 %.  The engine tracks 131,072 particles drawn from the same distribution."""
    import glob
    files = [np.load(p) for p in sorted(glob.glob(os.path.join(GOLDEN, "qe_equilibrium*.npz")))]
    turns = files[0]["turns"]
    ref, n_ref = pooled(files, len(turns) - 1)
    n = 131072
    r = LT.matched_bunch_particles(n, files[0]["m66"], seed=777)
    line = A.Line(ctx, LT.dba_ring())
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    line.set_seed(97531)
    line.track(r, int(turns[-1]))
    live = ~np.isnan(r[:, 0])
    assert live.all()
    d = r - r.mean(axis=0)
    mine = {(a, b): float((d[:, a] * d[:, b]).mean()) for (a, b) in ref}
    for name, g, w in (("emittance_x", emittance_x(mine), emittance_x(ref)),
                       ("sigma_z", np.sqrt(mine[(4, 4)]), np.sqrt(ref[(4, 4)])),
                       ("sigma_delta", np.sqrt(mine[(5, 5)]), np.sqrt(ref[(5, 5)]))):
        assert abs(g - w) <= 0.02 * w, (name, g, w, n_ref)


@pytest.mark.parametrize("mode", ["lump", "lump_qe"])
def test_syncrad_lumped_modes_statistics(A, ctx, LT, mode):
    """ASyncRad's random modes (accel.cpp:1806-1854), reached as the reference's deck reaches them
    through the radiation flag (aline.cpp:273-289): LUMP (damping and excitation) and LUMP_QE
    (excitation alone), on the 4D DBA with one 0.2 m SyncRad element, every particle from the
    origin for 300 turns.  The reference's moments over 16,384 particles (pooled single-threaded
    srand runs, tests/golden/syncrad_lump.npz from make_syncrad_golden.py) against the engine's
    over 262,144: rms sizes within 2 % in x, x', y, y', z and delta; means within four combined
    standard errors; nobody lost.  LUMP_DAMP alone is deterministic and an element case of
    golden.npz."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_syncrad_golden as S
    ref = np.load(os.path.join(GOLDEN, "syncrad_lump.npz"))
    n_ref, turns = int(ref["n"][0]), int(ref["turns"][0])
    line = A.Line(ctx, S.ring(A, LT))
    line.set_flags(rad=A.RAD_LUMP if mode == "lump" else A.RAD_LUMP_QE, cavity=0)
    line.set_seed(777 if mode == "lump" else 778)
    n = 262144
    r = np.zeros((n, 6))
    line.track(r, turns)
    live = ~np.isnan(r[:, 0])
    assert live.all() and int(ref[f"{mode}_nlive"][0]) == n_ref
    m = r.mean(axis=0)
    d = r - m
    sig = np.sqrt((d * d).mean(axis=0))
    rs, rm = ref[f"{mode}_sigma"], ref[f"{mode}_mean"]
    for k in range(6):
        assert rs[k] > 0
        assert abs(sig[k] - rs[k]) <= 0.02 * rs[k], (mode, k, sig[k], rs[k])
        se = np.sqrt(rs[k] ** 2 / n_ref + sig[k] ** 2 / n)
        assert abs(m[k] - rm[k]) <= 4 * se, (mode, k, m[k], rm[k], se)
