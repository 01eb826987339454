"""accel_beam_stat_noalloc against accel_beam_stat on the same device arrays.

accel_beam_stat_noalloc is for callers that cannot let a library allocate device memory (memory
reserved up front by a pool or another framework, sampling loops that a cudaMalloc/cudaFree
synchronisation would stall): its partial sums live in a fixed per-device array.

Two calls in a row (AoS, then SoA with a different N and lost particles), each compared with the
allocating entry point within 1e-12 relative (both sum in fixed orders, but different ones); the
second also checks that free device memory did not move.  Then a call on a non-default stream,
an all-lost beam (NaN moments and a zero count, as accel_beam_stat and the reference give), and
an oversized request, which must come back ACCEL_E_TOO_LARGE without launching anything.  The file
name sorts last so that it runs after every other test, and it builds all of its own state, so
it also passes alone.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def beam(n, seed, lost_frac):
    rng = np.random.default_rng(seed)
    r = rng.normal(size=(n, 6)) * np.array([1e-3, 1e-4, 5e-4, 5e-5, 3e-3, 1e-3])
    r += np.array([2e-5, -1e-6, 0.0, 3e-7, 1e-4, -2e-4])
    r[:, 1] += 0.3 * r[:, 0]  # some <xx'> correlation
    lost = rng.random(n) < lost_frac
    r[lost, 0] = np.nan
    return r


def check(A, ctx, torch, r_host, layout, stream=None):
    n = r_host.shape[0]
    dev = torch.from_numpy(r_host if layout == A.LAYOUT_AOS else np.ascontiguousarray(r_host.T)).cuda()
    out = torch.full((19,), -1.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    A.beam_stat_noalloc(dev, out, layout=layout, n=n, stream=None if stream is None else stream.cuda_stream)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    got = out.cpu().numpy()
    mean, sig, cross, nlive = ctx.beam_stat(dev, layout=layout, n=n)
    want = np.concatenate([mean, sig, cross, [nlive]])
    pairs = [(0, 1), (2, 3), (0, 5), (1, 5), (2, 4), (3, 4)]  # the cross moments' coordinates
    scale = np.concatenate([sig, sig, [sig[a] * sig[b] for a, b in pairs], [1.0]])
    assert got[18] == nlive
    assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(np.abs(want), scale)), (got, want)
    return free0, free1


def test_noalloc_matches_allocating_entry_point(A, ctx):
    torch = pytest.importorskip("torch")
    # first call (does the one-time set-up)
    check(A, ctx, torch, beam(100_003, 1, 0.0), A.LAYOUT_AOS)
    # second call in a row: other size, other layout, lost particles; no device memory taken
    free0, free1 = check(A, ctx, torch, beam(37_001, 2, 0.1), A.LAYOUT_SOA)
    assert free1 == free0
    # on a stream of the caller's own
    side = torch.cuda.Stream()
    check(A, ctx, torch, beam(5_000, 3, 0.3), A.LAYOUT_AOS, stream=side)


def test_noalloc_all_lost(A, ctx):
    """Every particle lost: NaN moments and a zero count, as the allocating entry point gives."""
    torch = pytest.importorskip("torch")
    r = beam(3_000, 4, 0.0)
    r[:, 0] = np.nan
    dev = torch.from_numpy(r).cuda()
    out = torch.zeros(19, dtype=torch.float64, device="cuda")
    A.beam_stat_noalloc(dev, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    mean, sig, cross, nlive = ctx.beam_stat(dev)
    assert got[18] == 0 and nlive == 0
    assert np.all(np.isnan(got[:18]))
    assert np.all(np.isnan(np.concatenate([mean, sig, cross])))


def test_noalloc_wrapper_rejects_bad_buffers(A):
    """The Python wrapper refuses, before any call, buffers the C entry point would overrun."""
    torch = pytest.importorskip("torch")
    r = torch.zeros(60, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        A.beam_stat_noalloc(r, torch.zeros(19, dtype=torch.float32, device="cuda"))
    with pytest.raises(ValueError):
        A.beam_stat_noalloc(r, torch.zeros(18, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        A.beam_stat_noalloc(r, torch.zeros(19, dtype=torch.float64))
    with pytest.raises(ValueError):
        A.beam_stat_noalloc(r, torch.zeros(19, dtype=torch.float64, device="cuda"), n=11)


def test_noalloc_rejects_oversized_request(A):
    torch = pytest.importorskip("torch")
    small = torch.zeros(6, dtype=torch.float64, device="cuda")
    out = torch.zeros(19, dtype=torch.float64, device="cuda")
    import ctypes as C
    fn = A.lib().accel_beam_stat_noalloc  # called directly: the wrapper infers N from the tensor
    st = fn(C.c_void_p(small.data_ptr()), A.LAYOUT_AOS, 4194304 + 1, C.c_void_p(out.data_ptr()), None)
    assert st == A.E_TOO_LARGE
    assert b"exceeds" in A.lib().accel_last_error()
    torch.cuda.synchronize()
    assert float(out.abs().sum()) == 0.0  # nothing was written
