"""Size-independent properties at the benchmark's full size, and edge cases.

Every particle is tracked on its own, with no sum or exchange across particles, so its result
cannot depend on which other particles share a launch, how the live list is compacted, or how the
turns are cut into segments.  The full batched job of the benchmark (256 error-seeded DBA copies,
337,976 particles) therefore has to agree bit for bit with the same copies tracked one at a time.
The oracle cannot track that many particles in test time; this property covers the full size,
and the parity tests cover the arithmetic against the oracle at smaller sizes.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_full_batched_job_equals_copies_tracked_alone(A, ctx):
    torch = pytest.importorskip("torch")
    sys.path.insert(0, ROOT)
    import bench
    rings, off, aos, _ = bench.workload(256, 0)
    nturn = 60
    lines = [A.Line(ctx, r) for r in rings]
    st = torch.tensor(np.ascontiguousarray(aos.T), device="cuda", dtype=torch.float64).contiguous()
    loss = torch.empty(int(off[-1]), device="cuda", dtype=torch.int32)
    A.track_batched(lines, off, st, nturn, loss=loss)
    torch.cuda.synchronize()
    got = st.cpu().numpy().T
    got_loss = loss.cpu().numpy()
    assert int(off[-1]) == 337976
    for k in (0, 1, 97, 200, 255):
        r = aos[off[k]:off[k + 1]].copy()
        lt = np.empty(len(r), dtype=np.int32)
        lines[k].track(r, nturn, loss=lt)
        assert np.array_equal(lt, got_loss[off[k]:off[k + 1]]), k
        assert np.array_equal(r, got[off[k]:off[k + 1]], equal_nan=True), k
    assert (got_loss >= 0).any() and (got_loss < 0).any()  # both fates occur in this job


def test_edge_cases(A, ctx, LT):
    line = A.Line(ctx, LT.dba_ring())
    rng = np.random.default_rng(4)
    r0 = np.zeros((64, 6))
    r0[:, 0] = rng.uniform(-0.02, 0.02, 64)
    r0[:, 2] = rng.uniform(0.0, 0.01, 64)

    # nothing to do: no particles, no turns, an empty element range
    empty = np.zeros((0, 6))
    line.track(empty, 10)
    for kw in ({"nturn": 0}, {"nturn": 5, "st": 7, "ed": 7}):
        r = r0.copy()
        lt = np.full(64, 123, dtype=np.int32)
        line.track(r, loss=lt, **kw)
        assert np.array_equal(r, r0) and np.all(lt == -1)

    # a particle lost before the call keeps its state and reports turn 0; the others are tracked
    # exactly as without it
    r = r0.copy()
    r[5, 0], r[5, 4] = np.nan, 3.0
    lt = np.empty(64, dtype=np.int32)
    line.track(r, 40, loss=lt)
    keep = np.arange(64) != 5
    ref = np.ascontiguousarray(r0[keep])
    lt_ref = np.empty(63, dtype=np.int32)
    line.track(ref, 40, loss=lt_ref)
    assert np.isnan(r[5, 0]) and r[5, 4] == 3.0 and lt[5] == 0
    assert np.array_equal(r[keep], ref, equal_nan=True) and np.array_equal(lt[keep], lt_ref)

    # one particle alone equals the same particle inside a group
    one = r0[9:10].copy()
    line.track(one, 40)
    grp = r0.copy()
    line.track(grp, 40)
    assert np.array_equal(one[0], grp[9], equal_nan=True)
