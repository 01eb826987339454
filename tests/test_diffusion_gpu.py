"""Tune diffusion and tracked tunes (ALine::trackDiffusion, aline.cpp:716-779; ALine::tracktune,
aline.cpp:1159-1186) through the C ABI, against the reference's own results
(tests/golden/diffusion.npz, made by make_diffusion_golden.py with the reference library).

The ring is the 4D DBA, which has no transcendental on its path, so the exact mode (the
reference's operation order) tracks turn-by-turn records bit for bit equal to the reference's,
and the comparison isolates the analysis: NAFF on identical records (this NAFF agrees with the
reference's to its 3e-8 refinement tolerance), the half-record split, the diffusion formula
and the lost-point convention.  Bars: lost points (NaN) where the reference loses them; tunes
within 1e-7; dif within 0.01 where the reference's tune change is well above the NAFF
tolerance (dif > -19), otherwise both at the noise floor (dif < -17.5); the returned sum is -3
per lost point plus the kept points' dif, as the reference's; tracktune within 1e-7.  The fused mode (FMA, merged drifts) is held to
the same tunes within 1e-6 on the regular points.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def DG():
    return dict(np.load(os.path.join(GOLDEN, "diffusion.npz")))


def test_track_diffusion_against_reference(A, ctx, LT, DG):
    line = A.Line(ctx, LT.dba_4d_ring())
    nturn = int(DG["nturn"][0])
    nux, nuy, dif, tot = line.track_diffusion(nturn, DG["x0"], DG["y0"], mode=A.MODE_EXACT)
    lost_ref = np.isnan(DG["dif"])
    assert np.array_equal(np.isnan(dif), lost_ref)
    assert lost_ref.any() and (~lost_ref).sum() >= 20
    k = ~lost_ref
    assert np.max(np.abs(nux[k] - DG["nux"][k])) < 1e-7
    assert np.max(np.abs(nuy[k] - DG["nuy"][k])) < 1e-7
    big = k & (DG["dif"] > -19)
    small = k & ~big
    assert big.sum() >= 8 and small.sum() >= 4
    assert np.max(np.abs(dif[big] - DG["dif"][big])) < 1e-2, (dif[big], DG["dif"][big])
    assert np.all(dif[small] < -17.5)
    floor = -4 * np.log(1024.0)
    assert np.all(dif[k] >= floor) and np.any(dif[k] == floor)
    # the sum: -3 per lost point plus the kept points' dif
    assert abs(tot - (-3.0 * lost_ref.sum() + dif[k].sum())) < 1e-9

    # the fused mode: the same tunes on the regular points
    nf, mf, df, _ = line.track_diffusion(nturn, DG["x0"], DG["y0"], mode=A.MODE_FUSED)
    reg = k & (DG["dif"] < -19)
    assert np.max(np.abs(nf[reg] - DG["nux"][reg])) < 1e-6
    assert np.max(np.abs(mf[reg] - DG["nuy"][reg])) < 1e-6


def test_track_tune_against_reference(A, ctx, LT, DG):
    line = A.Line(ctx, LT.dba_4d_ring())
    nturn = int(DG["nturn"][0])
    for (x, y), (tx, ty) in zip(DG["tune_pts"], DG["tunes"]):
        gx, gy = line.track_tune(nturn, float(x), float(y), mode=A.MODE_EXACT)
        assert abs(gx - tx) < 1e-7 and abs(gy - ty) < 1e-7, ((x, y), (gx, gy), (tx, ty))
