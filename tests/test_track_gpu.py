"""GPU parity: the engine's kernels, through the C-ABI, against the reference's golden outputs and
the CPU oracle on the same seeded inputs.

Tolerances (FP64):
  plain kernel (reference operation order, no FMA): bit-identical for every element whose map has
      no per-particle transcendental; within 1e-14 relative where CUDA's sin/cos/sinh/cosh/exp
      enter (linear Quad and Bend, Cavity, TransWake);
  fused kernel (FMA, merged drifts, effective Horner order): within 1e-12 relative after one turn
      and 1e-9 after 1,000 turns on regular orbits;
  loss turns: identical, except at grid points on the chaotic aperture boundary (fate sensitive to
      a 1e-12 perturbation, or within one grid step of the opposite fate), where an ulp of
      difference (CUDA's sin in the cavity, FMA) legitimately changes the turn a particle is lost.
"Relative" is per coordinate, scaled by that coordinate's RMS over the live particles.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import Sensitivity, check_loss_turns, rel_err, rel_err_each, same_bits

pytestmark = pytest.mark.gpu

TRANSCENDENTAL = {"quad_f", "quad_d", "bend", "bend_neg", "cavity", "transwake"}


def _flags(line, A, name):
    if name == "cavity":
        line.set_flags(cavity=1)
    if name == "bendm_rad":
        line.set_flags(rad=1)
    if name == "transwake":
        line.set_flags(wake=1)
    if name == "syncrad_damp":
        line.set_flags(rad=A.RAD_LUMP_DAMP)


MODES = {"plain": 1, "exact": 2, "fused": 0}  # A.MODE_PLAIN / MODE_EXACT / MODE_FUSED


@pytest.mark.parametrize("mode", ["plain", "exact", "fused"])
def test_elements_against_reference(A, ctx, G, MG, mode):
    m = MODES[mode]
    for name, elems in MG.element_cases().items():
        line = A.Line(ctx, elems)
        _flags(line, A, name)
        r = G["elem_in"].copy()
        line.track(r, 1, mode=m)
        ref = G[f"elem_{name}"]
        if mode != "fused" and name not in TRANSCENDENTAL:
            assert same_bits(r, ref), name
        elif mode != "fused":
            assert rel_err(r, ref) < 1e-14, name
        else:
            assert rel_err(r, ref) < 1e-12, (name, rel_err(r, ref))
        assert np.array_equal(np.isnan(r[:, 0]), np.isnan(ref[:, 0])), name


@pytest.mark.parametrize("mode", ["plain", "exact"])
def test_plain_fodo_bit_exact(A, ctx, G, LT, mode):
    line = A.Line(ctx, LT.fodo_ring())
    for turns, key in ((1, "fodo_t1"), (100, "fodo_t100")):
        r = G["fodo_in"].copy()
        line.track(r, turns, mode=MODES[mode])
        assert same_bits(r, G[key]), key


def _exact_vs_plain(A, lines, off, aos, nturn):
    """Track the same particles in plain and in exact mode (batched over `lines`); return both
    final states and loss turns.  Each run restarts the lines' QE sequences (set_seed), which
    every tracking call otherwise advances."""
    import torch
    out = []
    for m in (A.MODE_PLAIN, A.MODE_EXACT):
        for k, l in enumerate(lines):
            l.set_seed(4242 + k)
        soa = torch.tensor(aos.T.copy(), device="cuda", dtype=torch.float64).contiguous()
        loss = torch.empty(len(aos), device="cuda", dtype=torch.int32)
        A.track_batched(lines, off, soa, nturn, loss=loss, mode=m)
        torch.cuda.synchronize()
        out.append((soa.cpu().numpy().T.copy(), loss.cpu().numpy()))
    return out


def test_exact_mode_is_the_plain_kernel_bit_for_bit(A, ctx, G, LT):
    """The exact mode keeps the state in registers over 16-turn launches but does the plain
    kernel's arithmetic: coordinates, aperture codes and loss turns equal bit for bit, with
    radiation and RF (the DA grid of the DBA, 200 turns, particles lost all along), with quantum
    excitation (the same counter-based normals), over error-seeded copies in one batch, and on a
    line whose longitudinal wake splits every turn into ranges."""
    base = LT.dba_ring()
    # radiation + RF, losses
    line = A.Line(ctx, base)
    g = G["dba_grid_in"]
    (rp, lp), (re, le) = _exact_vs_plain(A, [line], np.array([0, len(g)]), g, 200)
    assert same_bits(re, rp) and np.array_equal(le, lp) and (lp >= 0).any() and (lp < 0).any()
    # quantum excitation
    qline = A.Line(ctx, base)
    qline.set_flags(rad=A.RAD_RADQE)
    r0 = LT.matched_bunch_particles(2048, line.m66(), seed=3)
    (rp, lp), (re, le) = _exact_vs_plain(A, [qline], np.array([0, 2048]), r0, 40)
    assert same_bits(re, rp) and np.array_equal(le, lp)
    # error copies, one batch
    rings = [LT.error_copy(base, k) for k in (0, 1, 7)]
    grids = [G["c3_0_in"], G["c3_1_in"], LT.da_grid(7, 3)]
    off = np.zeros(4, dtype=np.int64)
    off[1:] = np.cumsum([x.shape[0] for x in grids])
    (rp, lp), (re, le) = _exact_vs_plain(A, [A.Line(ctx, r) for r in rings], off, np.concatenate(grids), 100)
    assert same_bits(re, rp) and np.array_equal(le, lp)
    # a wake element every turn
    wline = A.Line(ctx, base + [LT.longwake_elem()])
    wline.set_flags(wake=1)
    (rp, lp), (re, le) = _exact_vs_plain(A, [wline], np.array([0, 2048]), r0, 20)
    assert same_bits(re, rp) and np.array_equal(le, lp)


def test_fused_fodo_tolerance(A, ctx, G, LT):
    line = A.Line(ctx, LT.fodo_ring())
    r = G["fodo_in"].copy()
    line.track(r, 1)
    assert rel_err(r, G["fodo_t1"]) < 1e-12
    r = G["fodo_in"].copy()
    line.track(r, 100)
    assert rel_err(r, G["fodo_t100"]) < 1e-10


def test_fused_fodo_1000_turns(A, ctx, O, LT):
    """The 32-cell FODO (uniform x in +-5 mm, y in +-2 mm), 1,000 turns: fused GPU vs the oracle."""
    ring = LT.fodo_ring()
    p = LT.fodo_particles()[:256].copy()
    ref = p.copy()
    lt_ref = O.port_track(ring, ref, 1000, nthreads=8)
    line = A.Line(ctx, ring)
    r = p.copy()
    lt = np.empty(len(r), dtype=np.int32)
    line.track(r, 1000, loss=lt)
    assert np.array_equal(lt, lt_ref)
    assert rel_err(r, ref) < 1e-9


@pytest.mark.parametrize("mode", ["plain", "fused"])
def test_dba_grid_loss_turns(A, ctx, O, G, LT, mode):
    """The 18-cell DBA (radiation + cavity on): loss turns of a DA grid against the reference."""
    m = A.MODE_PLAIN if mode == "plain" else A.MODE_FUSED
    ring = LT.dba_ring()
    sv = Sensitivity(O, ring, G["dba_grid_in"], 200, 13, 7)
    ref_lt = sv.lt
    assert np.array_equal(ref_lt, G["dba_grid_loss"])  # the oracle is the reference here
    line = A.Line(ctx, ring)
    r = G["dba_grid_in"].copy()
    lt = np.empty(len(r), dtype=np.int32)
    line.track(r, 200, loss=lt, mode=m)
    check_loss_turns(lt, ref_lt, sv.boundary)
    assert sv.regular.sum() >= 10
    err = rel_err_each(r[sv.regular], G["dba_grid_out"][sv.regular], sv.scale)
    assert np.max(err) < 1e-9, np.max(err)
    # lost particles carry the reference's aperture code in z and NaN in x
    # (a particle that overflows to NaN before reaching the aperture carries NaN there instead)
    same_loss = (lt >= 0) & (lt == ref_lt) & ~sv.boundary
    assert np.all(np.isnan(r[lt >= 0, 0]))
    assert np.array_equal(r[same_loss, 4], G["dba_grid_out"][same_loss, 4], equal_nan=True)


@pytest.mark.parametrize("mode", ["plain", "fused"])
def test_batched_error_copies(A, ctx, O, G, LT, mode):
    """Error-seeded copies of the DBA with uneven grids tracked in one batched launch."""
    import torch
    m = A.MODE_PLAIN if mode == "plain" else A.MODE_FUSED
    base = LT.dba_ring()
    rings = [LT.error_copy(base, k) for k in (0, 1, 7)]
    shapes = [(9, 5), (9, 5), (7, 3)]
    grids = [G["c3_0_in"], G["c3_1_in"], LT.da_grid(7, 3)]
    lines = [A.Line(ctx, r) for r in rings]
    off = np.zeros(len(grids) + 1, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    aos = np.concatenate(grids)
    soa = torch.tensor(aos.T.copy(), device="cuda", dtype=torch.float64).contiguous()
    loss = torch.empty(len(aos), device="cuda", dtype=torch.int32)
    A.track_batched(lines, off, soa, 100, loss=loss, mode=m)
    torch.cuda.synchronize()
    out = soa.cpu().numpy().T.copy()
    lt = loss.cpu().numpy()
    for k in range(3):
        s = slice(off[k], off[k + 1])
        sv = Sensitivity(O, rings[k], grids[k], 100, *shapes[k])
        if k < 2:
            assert np.array_equal(sv.lt, G[f"c3_{k}_loss"])
        check_loss_turns(lt[s], sv.lt, sv.boundary, max_frac=0.3)
        if sv.regular.any():
            err = rel_err_each(out[s][sv.regular], sv.final[sv.regular], sv.scale)
            assert np.max(err) < 1e-9, (k, np.max(err))


def test_m66_fd_matches_getm66_and_exact_is_close(A, ctx, G, LT):
    line = A.Line(ctx, LT.fodo_ring())
    fd = line.m66(method=1, delta=1e-8)
    assert same_bits(fd, G["fodo_m66"])  # the FD path is the reference's getm66 on the GPU
    ex = line.m66(method=0)
    assert np.max(np.abs(ex - fd)) < 1e-6 * max(1.0, np.max(np.abs(fd)))
    # exact map is symplectic: M^T J M = J in the transverse 4x4 block
    J = np.zeros((4, 4))
    J[0, 1] = J[2, 3] = 1
    J[1, 0] = J[3, 2] = -1
    m4 = ex[:4, :4]
    assert np.max(np.abs(m4.T @ J @ m4 - J)) < 1e-12


def test_setrfphase_matches_reference(A, ctx, G, LT):
    """ALine::setrfphase on the GPU (plain kernel, radiation on): the reference's phase, bit for bit."""
    line = A.Line(ctx, A.read_lattice(f"{LT.GOLDEN_DIR}/dba18.lat"))
    assert line.setrfphase() == G["dba_phis"][0]


def test_range_pass_and_layouts(A, ctx, O, G, LT):
    """pass(r, N, st, ed) on a sub-range, AoS and SoA, host and device pointers."""
    import torch
    ring = LT.fodo_ring()
    line = A.Line(ctx, ring)
    p = G["fodo_in"].copy()
    ref = p.copy()
    O.port_pass_line(ring, ref, 17, 211)
    r = p.copy()
    line.track(r, 1, st=17, ed=211, mode=A.MODE_PLAIN)
    assert same_bits(r, ref)
    soa = np.ascontiguousarray(p.T)
    line.track(soa, 1, st=17, ed=211, mode=A.MODE_PLAIN, layout=A.LAYOUT_SOA, n=len(p))
    assert same_bits(soa.T, ref)
    dev = torch.tensor(p, device="cuda")
    line.track(dev, 1, st=17, ed=211, mode=A.MODE_PLAIN)
    torch.cuda.synchronize()
    assert same_bits(dev.cpu().numpy(), ref)


@pytest.mark.parametrize("mode", ["fused", "exact"])
def test_range_pass_other_modes(A, ctx, O, G, LT, mode):
    """pass(r, N, st, ed) in the fused and exact modes: a sub-range against the reference's
    pass_line (1e-12 fused, bit for bit exact), and a turn tracked as two ranges equal to the
    turn in one call (each element's arithmetic does not depend on where a call starts)."""
    ring = LT.fodo_ring()
    line = A.Line(ctx, ring)
    p = G["fodo_in"].copy()
    ref = p.copy()
    O.port_pass_line(ring, ref, 17, 211)
    r = p.copy()
    line.track(r, 1, st=17, ed=211, mode=MODES[mode])
    if mode == "exact":
        assert same_bits(r, ref)
    else:
        assert rel_err(r, ref) < 1e-12
    whole, split = p.copy(), p.copy()
    line.track(whole, 1, mode=MODES[mode])
    line.track(split, 1, st=0, ed=123, mode=MODES[mode])
    line.track(split, 1, st=123, ed=len(ring), mode=MODES[mode])
    assert same_bits(split, whole)


def test_beam_stat_matches_calc_beam_stat(A, ctx, O, G):
    r = G["dba_grid_out"].copy()
    mean, sig, cross, nl = ctx.beam_stat(r)
    m2, s2, c2, n2 = O.port_beam_stat(r)
    assert nl == n2
    assert np.allclose(mean, m2, rtol=1e-12, atol=1e-18)
    assert np.allclose(sig, s2, rtol=1e-12, atol=1e-18)
    assert np.allclose(cross, c2, rtol=1e-10, atol=1e-20)


def test_longwake_against_oracle(A, ctx, O, LT):
    rng = np.random.default_rng(11)
    n = 4096
    r = np.zeros((n, 6))
    r[:, 0] = rng.normal(0, 1e-4, n)
    r[:, 4] = rng.normal(0, 3e-3, n)
    r[:, 5] = rng.normal(0, 1e-3, n)
    r[::97, 0] = np.nan  # a few lost particles are skipped
    elems = [LT.longwake_elem()]
    ref = r.copy()
    O.port_track(elems, ref, 1, loss=False)
    line = A.Line(ctx, elems)
    out = r.copy()
    line.track(out, 1)
    assert np.array_equal(np.isnan(out[:, 0]), np.isnan(ref[:, 0]))
    d_ref, d = ref[:, 5] - r[:, 5], out[:, 5] - r[:, 5]
    live = ~np.isnan(r[:, 0])
    assert np.max(np.abs(d[live] - d_ref[live])) < 1e-12 * np.max(np.abs(d_ref[live]))
    assert np.max(np.abs(d_ref[live])) > 0


@pytest.mark.parametrize("spread", ["bunch", "long"])
def test_transverse_wake_sorted_sum_matches_pair_sum(A, ctx, spread):
    """The fused mode's O(N log N) transverse wake (z-sorted prefix sums of the factorised
    resonator wake) against the plain mode's pair sum, the reference's order of operations:
    16,384 particles, a tenth of them sharing their z with another (equal z are each other's
    sources), one lost before the wake.  'long' spreads z over 10 m, beyond the factorisation's
    exponent range, where each particle takes the pair sum over the sorted list."""
    rng = np.random.default_rng(21)
    n = 16384
    r = np.zeros((n, 6))
    r[:, 0] = rng.normal(0, 1e-3, n)
    r[:, 2] = rng.normal(0, 5e-4, n)
    r[:, 4] = rng.normal(0, 3e-3, n) if spread == "bunch" else rng.uniform(-5, 5, n)
    r[:, 5] = rng.normal(0, 1e-3, n)
    r[1::10, 4] = r[0::10, 4][: len(r[1::10])]
    r[5, 0] = np.nan
    tw = A.elem(A.TRANSWAKE, "TW", 0.5, f=[3000, 2.0, 50.0, 10.0, 1.5, 40.0, 12.0, 2.0], flags=1)
    line = A.Line(ctx, [A.elem(A.DRIFT, "D", 0.3), tw, A.elem(A.DRIFT, "D", 0.2)])
    a, b, c = r.copy(), r.copy(), r.copy()
    line.track(a, 1, mode=A.MODE_PLAIN)
    n0 = ctx.transwake_pair_passes()
    line.track(b, 1, mode=A.MODE_FUSED)
    line.track(c, 1, mode=A.MODE_FUSED)
    # the long bunch takes the pair-sum fallback, once per pass, and the counter says so
    assert ctx.transwake_pair_passes() - n0 == (2 if spread == "long" else 0)
    assert np.array_equal(b, c, equal_nan=True)  # the scan adds in a fixed order: reproducible
    live = ~np.isnan(r[:, 0])
    assert np.array_equal(np.isnan(a[:, 0]), np.isnan(b[:, 0]))
    for k in (1, 3):
        kick = np.abs(a[live, k] - r[live, k])
        assert kick.max() > 0
        assert np.max(np.abs(b[live, k] - a[live, k])) < 1e-10 * kick.max(), k


def test_transverse_wake_ring_fused_matches_plain(A, ctx, LT):
    """The sorted transverse wake inside the 4D DBA ring over 100 turns: the fused mode (fast maps,
    z-sorted prefix sums, the order in z changing from turn to turn) against the plain mode (the
    reference's operation order and pair sum) at the 1000-turn regular-orbit tolerance; and the
    wake does act (the same ring without it ends elsewhere)."""
    ring = LT.dba_4d_ring()
    m = A.Line(ctx, ring).m66()
    tw = A.elem(A.TRANSWAKE, "TW", 0.0, f=[3000, 2.0, 5000.0, 10.0, 1.5, 4000.0, 12.0, 2.0], flags=1)
    r0 = LT.matched_bunch_particles(2048, m, seed=9)
    line = A.Line(ctx, ring + [tw])
    a, b, c = r0.copy(), r0.copy(), r0.copy()
    line.track(a, 100, mode=A.MODE_PLAIN)
    line.track(b, 100, mode=A.MODE_FUSED)
    A.Line(ctx, ring).track(c, 100, mode=A.MODE_FUSED)
    assert not np.isnan(a[:, 0]).any() and not np.isnan(b[:, 0]).any()
    assert rel_err(b, a) < 1e-9
    assert rel_err(c, a) > 1e-6


def test_errors_are_statuses(A, ctx):
    r = np.zeros((4, 6))
    with pytest.raises(A.AccelError) as ei:  # a WigTable that names no kick table
        A.Line(ctx, [A.elem(A.WIGTABLE, "W", 1.0)]).track(r, 1)
    assert ei.value.status == A.E_INVALID
    line2 = A.Line(ctx, [A.elem(A.DRIFT, "D", 1.0)])
    with pytest.raises(A.AccelError) as ei:
        line2.track(r, 1, st=0, ed=5)
    assert ei.value.status == A.E_INVALID


def test_device_memory_limit_fails_cleanly(A, LT):
    """Out of memory, simulated by the library's device-memory budget: tracking on a new context
    needs new buffers, the budget refuses them, the call returns E_NOMEM with the particles
    untouched, and with the budget lifted the same call tracks exactly as an unconstrained one."""
    rng = np.random.default_rng(3)
    r0 = np.zeros((3000, 6))
    r0[:, 0] = rng.uniform(-2e-3, 2e-3, 3000)
    r0[:, 2] = rng.uniform(-1e-3, 1e-3, 3000)
    ref = r0.copy()
    A.Line(A.Context(0), LT.fodo_ring()).track(ref, 20)
    c2 = A.Context(0)
    line = A.Line(c2, LT.fodo_ring())
    held = A.device_memory_held()
    try:
        A.set_device_memory_limit(held)  # no new buffer fits
        r = r0.copy()
        with pytest.raises(A.AccelError) as ei:
            line.track(r, 20)
        assert ei.value.status == A.E_NOMEM and "limit" in str(ei.value)
        assert np.array_equal(r, r0)
        assert A.device_memory_held() == held
    finally:
        A.set_device_memory_limit(None)
    r = r0.copy()
    line.track(r, 20)
    assert np.array_equal(np.isnan(r[:, 0]), np.isnan(ref[:, 0]))
    assert rel_err(r, ref) < 1e-13
    assert A.device_memory_held() > held


def test_autotune_and_launch_count(A, ctx, LT):
    import torch
    base = LT.dba_ring()
    rings = [LT.error_copy(base, k) for k in range(3)]
    grids = [LT.da_grid(11, 5), LT.da_grid(13, 7), LT.da_grid(9, 9)]
    lines = [A.Line(ctx, r) for r in rings]
    off = np.zeros(4, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    aos = np.concatenate(grids)
    soa0 = torch.tensor(aos.T.copy(), device="cuda").contiguous()
    ctx.set_tile(0, 16, 0)
    a = soa0.clone()
    la = torch.empty(len(aos), device="cuda", dtype=torch.int32)
    n0 = ctx.launch_count()
    A.track_batched(lines, off, a, 50, loss=la)
    torch.cuda.synchronize()
    assert ctx.launch_count() > n0
    ctx.set_tile(0, 0, -1)
    tile = A.autotune(lines, off, soa0)
    assert tile[0] in (64, 128, 256) and tile[1] > 0
    b = soa0.clone()
    lb = torch.empty(len(aos), device="cuda", dtype=torch.int32)
    A.track_batched(lines, off, b, 50, loss=lb)
    torch.cuda.synchronize()
    assert torch.equal(la, lb)
    assert rel_err(a.cpu().numpy().T, b.cpu().numpy().T) < 1e-13


@pytest.mark.parametrize("mode", ["plain", "fused"])
def test_wigtable_against_reference(A, ctx, mode):
    """WigTable (thin, sliced, and an uneven grid with y descending; particles inside and outside
    the grid) against the reference's pass (tests/golden/wigtable.npz, make_wigtable_golden.py).
    The map has no transcendental, so the plain kernel agrees bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_wigtable_golden as W
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wigtable.npz"))
    m = A.MODE_PLAIN if mode == "plain" else A.MODE_FUSED
    for name, spec in W.tables().items():
        line = A.Line(ctx, W.elems(A, name, spec))
        r = g["elem_in"].copy()
        line.track(r, 1, mode=m)
        ref = g[f"elem_{name}"]
        if mode == "plain":
            assert np.array_equal(r, ref), (name, rel_err(r, ref))
        else:
            assert rel_err(r, ref) < 1e-12, (name, rel_err(r, ref))
        # the exact tangent map against the reference's difference map, at a point inside a cell
        at = np.array([0.0013, 1e-4, 0.0021, -1e-4, 0.0, 5e-4])
        ex, fd = line.m66_at(at, method=0), line.m66_at(at, method=1, delta=1e-9)
        assert np.all(np.isfinite(ex)) and np.max(np.abs(ex - fd)) < 1e-6 * np.max(np.abs(fd)), name


@pytest.mark.parametrize("mode", ["plain", "fused"])
def test_crab_rfmult_wiggler_against_reference(A, ctx, mode):
    """CrabCav, RFMult and IdealWig (both planes, and with radiation) against the reference's
    passes (tests/golden/elements_extra.npz, make_elem_extra_golden.py).  These maps call sin,
    cos, atan2 and sqrt, so the plain kernel agrees to 1e-14 rather than bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_elem_extra_golden as X
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "elements_extra.npz"))
    m = A.MODE_PLAIN if mode == "plain" else A.MODE_FUSED
    for name, elems in X.cases(A).items():
        line = A.Line(ctx, elems)
        r = g["elem_in"].copy()
        line.track(r, 1, mode=m)
        ref = g[f"elem_{name}"]
        tol = 1e-14 if mode == "plain" else 1e-12
        assert rel_err(r, ref) < tol, (name, rel_err(r, ref))
        if name != "idealwig_rad":  # the exact tangent map against the reference's difference map
            ex, fd = line.m66(method=0), line.m66(method=1, delta=1e-8)
            assert np.all(np.isfinite(ex)) and np.max(np.abs(ex - fd)) < 1e-6 * np.max(np.abs(fd)), name


def test_staged_wait_that_runs_out_is_a_status(A, ctx, LT):
    """The staged schedule waits for each block's shared-memory copy with a bounded number of
    probes.  A wait that runs out (forced here: a first wait of zero probes) sets the error word;
    the block then waits, bounded again, for its copy in flight and leaves, and the call returns
    ACCEL_E_TIMEOUT instead of results.  The context stays usable: with the default limit the
    next call tracks as the default schedule does, bit for bit."""
    import torch
    base = LT.dba_ring()
    lines = [A.Line(ctx, LT.error_copy(base, k)) for k in (0, 1)]
    grids = [LT.da_grid(11, 5), LT.da_grid(9, 7)]
    off = np.zeros(3, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    aos = np.concatenate(grids)

    def run(tile):
        ctx.set_tile(0, 8, tile)
        soa = torch.tensor(aos.T.copy(), device="cuda").contiguous()
        loss = torch.empty(len(aos), device="cuda", dtype=torch.int32)
        A.track_batched(lines, off, soa, 16, loss=loss)
        torch.cuda.synchronize()
        return soa.cpu().numpy(), loss.cpu().numpy()

    try:
        ctx.set_stage_wait(-1)
        with pytest.raises(A.AccelError) as err:
            run(200)
        assert err.value.status == A.E_TIMEOUT
        ctx.set_stage_wait(0)
        a, la = run(200)
        b, lb = run(0)
    finally:
        ctx.set_stage_wait(0)
        ctx.set_tile(0, 0, -1)
    assert np.array_equal(la, lb)
    assert same_bits(a, b)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_staged_schedule_equals_fused(A, ctx, LT, variant):
    """The instance-staged schedule (each block stages one instance's element hot lines in shared
    memory with a bulk copy) runs the fused kernel's arithmetic: over error-seeded copies in one
    batch, with radiation, quantum excitation and the cavity, it gives the same coordinates and
    loss turns bit for bit as the default schedule, including at tasks that straddle two
    instances (their lanes read the other instance's records from global memory)."""
    import torch
    base = LT.dba_ring()
    rings = [LT.error_copy(base, k) for k in (0, 1, 7, 9)]
    lines = [A.Line(ctx, r) for r in rings]
    for l in lines:
        l.set_flags(rad=A.RAD_RADQE)
    grids = [LT.da_grid(11, 5), LT.da_grid(13, 7), LT.da_grid(9, 9), LT.da_grid(17, 3)]
    off = np.zeros(5, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    aos = np.concatenate(grids)
    out = []
    for tile in (0, 200 + variant):
        ctx.set_tile(0, 8, tile)
        for k, l in enumerate(lines):
            l.set_seed(99 + k)
        soa = torch.tensor(aos.T.copy(), device="cuda").contiguous()
        loss = torch.empty(len(aos), device="cuda", dtype=torch.int32)
        A.track_batched(lines, off, soa, 60, loss=loss)
        torch.cuda.synchronize()
        out.append((soa.cpu().numpy(), loss.cpu().numpy()))
    ctx.set_tile(0, 0, -1)
    (a, la), (b, lb) = out
    assert (la >= 0).any() and (la < 0).any()
    assert np.array_equal(la, lb)
    assert same_bits(a, b)
