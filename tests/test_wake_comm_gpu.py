"""The longitudinal wake of a bunch spread over GPUs, on the one GPU a test gets.

With a communicator, every wake element runs in stages with NCCL exchanges in between: the
bunch's z range and live count (min / max / sum), then its bin counts (sum), after which the bin
geometry is recomputed from the exchanged values.  A one-rank communicator exchanges with itself,
so the staged path must reproduce the single-GPU wake bit for bit: the same kernels, the same
formulas, and NCCL inside the captured tracking graphs.  Runs over several ranks need several GPUs;
they take the same code path with real peers.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ring_with_wake(A, LT):
    ring = LT.dba_ring()
    return ring[:-1] + [LT.longwake_elem()] + ring[-1:]  # wake before the aperture


def test_one_rank_exchange_reproduces_local_wake(A, LT):
    rng = np.random.default_rng(12)
    n = 20000
    r0 = np.zeros((n, 6))
    r0[:, 0] = rng.normal(0, 2e-4, n)
    r0[:, 2] = rng.normal(0, 2e-5, n)
    r0[:, 4] = rng.normal(0, 3e-3, n)
    r0[:, 5] = rng.normal(0, 1e-3, n)
    out = []
    for with_comm in (False, True):
        ctx = A.Context(0)
        if with_comm:
            ctx.set_comm(A.nccl_unique_id(), 1, 0)
        line = A.Line(ctx, ring_with_wake(A, LT))
        r = r0.copy()
        lt = np.empty(n, dtype=np.int32)
        line.track(r, 30, loss=lt)
        out.append((r, lt))
        line.close()
        ctx.close()
    (a, la), (b, lb) = out
    assert np.array_equal(la, lb)
    assert np.array_equal(a, b, equal_nan=True)
    # the wake did act: the same ring without it ends elsewhere
    ctx = A.Context(0)
    line = A.Line(ctx, LT.dba_ring())
    c = r0.copy()
    line.track(c, 30)
    assert not np.array_equal(a, c, equal_nan=True)


def test_one_rank_exchange_reproduces_local_transverse_wake(A):
    """The fused mode's sorted transverse wake with a communicator: each rank's entries (z, x, y)
    all-gathered between the stages, the live count all-reduced, the slot count and the particle
    total exchanged at the start of the run.  With one rank the gathered list is the rank's own,
    so the result must equal the local wake bit for bit, lost particles included."""
    rng = np.random.default_rng(13)
    n = 5000
    r0 = np.zeros((n, 6))
    r0[:, 0] = rng.normal(0, 1e-3, n)
    r0[:, 2] = rng.normal(0, 5e-4, n)
    r0[:, 4] = rng.normal(0, 3e-3, n)
    r0[:, 5] = rng.normal(0, 1e-3, n)
    r0[7, 0] = np.nan
    tw = A.elem(A.TRANSWAKE, "TW", 0.4, f=[3000, 2.0, 50.0, 10.0, 1.5, 40.0, 12.0, 2.0], flags=1)
    elems = [A.elem(A.DRIFT, "D", 0.3), tw, A.elem(A.DRIFT, "D", 0.2)]
    out = []
    for with_comm in (False, True):
        ctx = A.Context(0)
        if with_comm:
            ctx.set_comm(A.nccl_unique_id(), 1, 0)
        line = A.Line(ctx, elems)
        r = r0.copy()
        line.track(r, 3, mode=A.MODE_FUSED)
        out.append(r)
        if with_comm:
            # the plain mode's pair sum runs within the rank: allowed with one rank
            p = r0.copy()
            line.track(p, 1, mode=A.MODE_PLAIN)
        line.close()
        ctx.close()
    a, b = out
    assert np.array_equal(a, b, equal_nan=True)
    assert not np.array_equal(a[:, 1], r0[:, 1])


def test_one_rank_exchange_reproduces_local_beam_moments(A):
    """accel_beam_stat on a context with a communicator gives the moments of the whole bunch: the
    first pass's sums and live count, then the centred second moments, summed over the ranks
    between the passes.  With one rank the sums are the rank's own, so the moments must equal the
    local ones bit for bit, lost particles left out."""
    rng = np.random.default_rng(14)
    n = 30000
    r = rng.normal(0, 1e-3, (n, 6))
    r[::97, 0] = np.nan
    out = []
    for with_comm in (False, True):
        ctx = A.Context(0)
        if with_comm:
            ctx.set_comm(A.nccl_unique_id(), 1, 0)
        out.append(ctx.beam_stat(r.copy()))
        ctx.close()
    (m0, s0, c0, n0), (m1, s1, c1, n1) = out
    assert n0 == n1 == n - len(range(0, n, 97))
    assert np.array_equal(m0, m1) and np.array_equal(s0, s1) and np.array_equal(c0, c1)
