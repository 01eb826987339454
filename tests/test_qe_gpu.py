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
    line = A.Line(ctx, LT.config2_ring())
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
    line = A.Line(ctx, LT.config2_ring())
    line.set_flags(rad=A.RAD_RADQE, cavity=1)
    runs = []
    for seed in (7, 7, 8):
        line.set_seed(seed)
        r = np.zeros((4096, 6))
        line.track(r, 20)
        runs.append(r)
    assert np.array_equal(runs[0], runs[1])
    assert not np.array_equal(runs[0], runs[2])
