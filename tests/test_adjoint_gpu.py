"""The adjoint pair on the GPU: gradients of L = sum over surviving particles of (x^2 + y^2) after
n turns, with respect to the initial coordinates and multipole strengths, against central finite
differences of the CPU oracle, and the one-turn Jacobian from six adjoint seeds against the exact
tangent map.  Tolerance: 1e-6 relative.  The differences are Richardson-extrapolated central
differences: steps of 1e-6 of a coordinate's spread; for a strength, the first step in 1e-2 ..
3e-6 at which the estimate has converged (a sextupole needs about 1e-3, a quadrupole about 1e-5)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def loss_of(O, ring, r0, nturn):
    r = r0.copy()
    O.port_track(ring, r, nturn, loss=False, nthreads=8)
    live = ~np.isnan(r[:, 0])
    return float(np.sum(r[live, 0] ** 2 + r[live, 2] ** 2))


def grad_final(rf):
    g = np.zeros_like(rf)
    live = ~np.isnan(rf[:, 0])
    g[live, 0] = 2 * rf[live, 0]
    g[live, 2] = 2 * rf[live, 2]
    return g


def small_particles(n, seed=1):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 6))
    r[:, 0] = rng.normal(0, 1e-3, n)
    r[:, 1] = rng.normal(0, 5e-5, n)
    r[:, 2] = rng.normal(0, 5e-4, n)
    r[:, 3] = rng.normal(0, 5e-5, n)
    return r


def richardson(f, h):
    """Central difference extrapolated from steps h and h/2: truncation error O(h^4)."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def converged_difference(f, steps=(1e-2, 1e-3, 1e-4, 3e-5, 1e-5, 3e-6)):
    """The first Richardson estimate that agrees with the one at a third of its step to 3e-7
    relative (a fifth of the test's tolerance): large steps are truncation-limited where the multi-turn map is tune-sensitive
    (quadrupoles), tiny ones round-off-limited where the gradient is a small sum of cancelling
    terms (sextupoles)."""
    for h in steps:
        a, b = richardson(f, h), richardson(f, h / 3)
        if abs(a - b) <= 3e-7 * max(abs(b), 1e-30):
            return a
    raise AssertionError(f"finite differences did not converge: {a} vs {b}")


def ring_and_params(A, LT, ringname):
    """The test rings: the FODO and the 4D DBA with two parameters on one element (the tape's
    dual-number path), the DBA with its cavity on and radiation off (synchrotron motion: the
    explicit tape's units that read z and change delta), the 4D DBA with one parameter per
    element (the explicit tape alone), and a FODO whose quadrupoles are thick linear Quad
    elements with a corrector and a matrix (element kinds the tape takes on dual numbers, and a
    Quad K parameter)."""
    if ringname == "fodo":
        ring, nturn, every = LT.fodo_ring(), 24, 8
    elif ringname == "dba4d":
        ring, nturn, every = LT.dba_4d_ring(), 40, 16  # 40 = 2 x 16 + 8: a short last segment
    elif ringname == "dba6d":
        ring, nturn, every = LT.dba_ring(), 40, 16
        for d in ring:
            if d.type == A.BENDMPOLE:
                d.flags = A.RAD_OFF
            if d.type == A.CAVITY:
                d.f[2] = 0.0  # without radiation the synchronous phase is 0
    elif ringname == "dba4d_single":
        ring, nturn, every = LT.dba_4d_ring(), 40, 16
    else:  # "fodo_quad"
        ring, nturn, every = [], 24, 8
        for d in LT.fodo_ring():
            if d.type == A.STRMPOLE and d.poly_b[2] == 0 and d.poly_b[1] != 0 and d.len > 0:
                ring.append(A.elem(A.QUAD, d.name, d.len, f=[d.poly_b[1]]))
            else:
                ring.append(d)
        ring.insert(3, A.elem(A.CORRECTOR, "C", 0.1, f=[2e-5, -1e-5]))
        m = np.eye(6)
        m[0, 1], m[2, 3] = 0.05, 0.05  # a short drift in x and y
        ring.insert(7, A.elem(A.MATRIX, "M", 0.0, mat=m.ravel()))
    sx = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.poly_b[2] != 0][:3]
    if ringname == "fodo_quad":
        qx = [i for i, d in enumerate(ring) if d.type == A.QUAD][:2]
        params = [(i, A.F_POLYNOMB, 2) for i in sx] + [(i, A.F_K, 0) for i in qx]
    elif ringname == "dba4d_single":
        qx = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.poly_b[2] == 0 and d.poly_b[1] != 0][:2]
        params = [(i, A.F_POLYNOMB, 2) for i in sx] + [(i, A.F_POLYNOMB, 1) for i in qx]
    else:
        qx = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.poly_b[2] == 0 and d.poly_b[1] != 0][:2]
        params = [(i, A.F_POLYNOMB, 2) for i in sx] + [(i, A.F_POLYNOMB, 1) for i in qx] + [(sx[0], A.F_POLYNOMA, 1)]
    return ring, nturn, every, params


@pytest.mark.parametrize("ringname", ["fodo", "dba4d", "dba6d", "dba4d_single", "fodo_quad"])
def test_adjoint_against_finite_differences(A, ctx, O, LT, ringname):
    ring, nturn, every, params = ring_and_params(A, LT, ringname)
    n = 32
    r0 = small_particles(n)
    line = A.Line(ctx, ring)
    adj = A.Adjoint(line, n, nturn, every, params)
    rf = adj.forward(r0)
    ref = r0.copy()
    O.port_track(ring, ref, nturn, loss=False)
    scale = np.sqrt(np.mean(ref ** 2, axis=0)) + 1e-30
    # the adjoint's forward is the reference map (FMA-contracted, so not bit-identical)
    assert np.max(np.abs(rf - ref) / scale) < 1e-10
    dr0, dp = adj.backward(grad_final(rf))
    h = 1e-6
    # initial coordinates: particles are independent, so perturb one particle at a time
    for p in (0, 7, 19):
        for k in range(4):
            def f(dv, p=p, k=k):
                a = r0.copy()
                a[p, k] += dv * scale[k] / scale[0]  # step relative to the coordinate's scale
                return loss_of(O, ring, a, nturn)
            fd = richardson(f, h) * scale[0] / scale[k]
            assert abs(dr0[p, k] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(dr0[:, k]))), (p, k, dr0[p, k], fd)
    # parameters
    for j, (e, fld, idx) in enumerate(params):
        def f(dv, e=e, fld=fld, idx=idx):
            rr = [d.copy() for d in ring]
            arr = rr[e].f if fld == A.F_K else (rr[e].poly_b if fld == A.F_POLYNOMB else rr[e].poly_a)
            arr[idx] += dv
            return loss_of(O, rr, r0, nturn)
        fd = converged_difference(f)
        assert abs(dp[j] - fd) <= 1e-6 * max(abs(fd), 1e-9), (j, dp[j], fd)


def test_tape_budget_paths_agree(A, ctx, LT):
    """The three ways of the reverse pass give one gradient: every turn start kept by the forward
    (the default here); checkpoint segments recomputed, with Jacobian tapes one turn at a time (a
    budget below the run's turn starts but above one turn's Jacobians); and the turn-by-turn
    reversal (a budget below one turn's Jacobians).  The first two take the same arithmetic for
    the coordinates (bit-identical dL/dr0) and group the parameter sums by chunk (round-off), the
    third another order of the arithmetic."""
    ring, _, _, params = ring_and_params(A, LT, "dba4d_single")  # five one-parameter elements
    nturn, every, n = 64, 16, 32
    r0 = small_particles(n)
    turn_starts = 48 * n * nturn                                # 98,304 bytes
    per_turn = 8 * 32 * (36 * (len(params) + 1) + 6 * len(params))  # 62,976 bytes
    assert per_turn < 80000 < turn_starts and 30000 < per_turn

    def grad(budget):
        A.set_adjoint_tape_budget(budget)
        try:
            adj = A.Adjoint(A.Line(ctx, ring), n, nturn, every, params)
            rf = adj.forward(r0)
            return adj.backward(grad_final(rf))
        finally:
            A.set_adjoint_tape_budget(None)

    d0, p0 = grad(None)
    d1, p1 = grad(80000)
    d2, p2 = grad(30000)
    assert np.array_equal(d1, d0)
    assert np.max(np.abs(p1 - p0)) < 1e-13 * np.max(np.abs(p0))
    # the turn-by-turn reversal rounds in another order; over 64 turns the map's growth makes
    # that a few 1e-10 of the largest component
    assert np.max(np.abs(d2 - d0)) < 1e-8 * np.max(np.abs(d0))
    assert np.max(np.abs(p2 - p0)) < 1e-8 * np.max(np.abs(p0))


def test_z_rows_taped_again_for_a_z_seed(A, ctx, LT):
    """On a line where no element reads z (the 4D DBA), the forward writes the unit Jacobians
    without their z rows, which a seed with zero z components multiplies by zero; a seed with a z
    component has the tapes written again with them, from the kept turn starts, before its sweep.
    The gradient is linear in the seed across the two kinds of tape, the z-free gradient is the
    same bit for bit before and after the second taping, and the z part equals the one of the
    checkpointed path (tapes chunk by chunk in the reverse pass)."""
    ring = LT.dba_4d_ring()
    pairs = LT.sextupole_pairs(ring)
    elems = sorted({i for p in pairs for i in p})[:6]
    params = [(i, A.F_POLYNOMB, 2) for i in elems]
    n, nturn, every = 64, 64, 16
    r0 = LT.gaussian_4d_particles(n, seed=3)
    adj = A.Adjoint(A.Line(ctx, ring), n, nturn, every, params)
    rf = adj.forward(r0)
    assert not np.isnan(rf[:, 0]).any()
    g = np.zeros_like(rf)
    g[:, 0], g[:, 2] = 2 * rf[:, 0], 2 * rf[:, 2]
    gz = np.zeros_like(rf)
    gz[:, 4] = np.random.default_rng(5).normal(size=n)
    d0, p0 = adj.backward(g)
    dz, pz = adj.backward(gz)
    d1, p1 = adj.backward(g)
    df, pf = adj.backward(g + gz)
    adj.close()
    assert np.array_equal(d0, d1) and np.array_equal(p0, p1)
    assert np.max(np.abs(dz)) > 0
    assert np.max(np.abs(df - d0 - dz)) < 1e-12 * np.max(np.abs(df))
    assert np.max(np.abs(pf - p0 - pz)) < 1e-12 * np.max(np.abs(pf))
    # 170,000 bytes: above one turn's tapes (147,456), below the run's turn starts (196,608)
    A.set_adjoint_tape_budget(170000)
    try:
        adj_c = A.Adjoint(A.Line(ctx, ring), n, nturn, every, params)
        adj_c.forward(r0)
        dzc, pzc = adj_c.backward(gz)
        adj_c.close()
    finally:
        A.set_adjoint_tape_budget(None)
    assert np.max(np.abs(dzc - dz)) < 1e-13 * np.max(np.abs(dz))
    assert np.max(np.abs(pzc - pz)) < 1e-12 * np.max(np.abs(pz))


def test_adjoint_one_turn_jacobian_is_exact(A, ctx, LT):
    """Six particles at the closed orbit (the origin of the 4D ring), seeded with unit adjoints:
    row i of the one-turn matrix is dL/dr0 of particle i for L = r_final[i]."""
    ring = LT.dba_4d_ring()
    line = A.Line(ctx, ring)
    r0 = np.zeros((6, 6))
    adj = A.Adjoint(line, 6, 1, 1, [])
    adj.forward(r0)
    rows, _ = adj.backward(np.eye(6))
    m_tan = line.m66(method=0)
    m_fd = line.m66(method=1, delta=1e-8)
    assert np.max(np.abs(rows - m_tan)) < 1e-12 * np.max(np.abs(m_tan))
    assert np.max(np.abs(rows - m_fd)) < 1e-6 * np.max(np.abs(m_fd))


def test_adjoint_rejects_radiation_and_bad_params(A, ctx, LT):
    ring = LT.dba_ring()  # radiation on
    line = A.Line(ctx, ring)
    with pytest.raises(A.AccelError) as ei:
        A.Adjoint(line, 4, 2, 1, [])
    assert ei.value.status == A.E_UNSUPPORTED
    line4 = A.Line(ctx, LT.dba_4d_ring())
    drift = [i for i, d in enumerate(LT.dba_4d_ring()) if d.type == A.DRIFT][0]
    with pytest.raises(A.AccelError) as ei:
        A.Adjoint(line4, 4, 2, 1, [(drift, A.F_POLYNOMB, 2)])
    assert ei.value.status == A.E_UNSUPPORTED


def test_handles_released_in_any_order(A, ctx, LT):
    """Context, line and adjoint destroyed parent-first through the C-ABI: each parent stays alive
    until its last child is gone, so the children still work and nothing is freed twice."""
    import ctypes as C
    L = A.lib()
    c = C.c_void_p()
    assert L.accel_ctx_create(0, C.byref(c)) == 0
    ring = LT.dba_4d_ring()
    arr = (A.ElemDesc * len(ring))(*ring)
    ln = C.c_void_p()
    assert L.accel_line_create(c, arr, len(ring), C.byref(ln)) == 0
    adj = C.c_void_p()
    z = np.zeros(1, dtype=np.int32)
    assert L.accel_adjoint_create(ln, 4, 2, 1, C.c_void_p(z.ctypes.data), C.c_void_p(z.ctypes.data),
                                  C.c_void_p(z.ctypes.data), 0, C.byref(adj)) == 0
    assert L.accel_ctx_destroy(c) == 0
    r = np.zeros((4, 6))
    r[:, 0] = 1e-4
    assert L.accel_line_destroy(ln) == 0
    out = np.empty_like(r)
    assert L.accel_adjoint_forward(adj, C.c_void_p(r.ctypes.data), C.c_void_p(out.ctypes.data)) == 0
    assert np.all(np.isfinite(out)) and np.any(out != r)
    assert L.accel_adjoint_destroy(adj) == 0


def test_autograd_function_over_the_adjoint_pair(A, ctx, LT):
    """A torch.autograd.Function whose forward and backward are the C-ABI pair: loss.backward()
    on a torch expression of the tracked coordinates returns the adjoint's gradients with respect
    to the initial coordinates and the sextupole strengths."""
    torch = pytest.importorskip("torch")
    ring = LT.dba_4d_ring()
    sx = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.poly_b[2] != 0][:4]
    line = A.Line(ctx, ring)
    n, nturn = 64, 32
    adj = A.Adjoint(line, n, nturn, 8, [(i, A.F_POLYNOMB, 2) for i in sx])

    class Track(torch.autograd.Function):
        @staticmethod
        def forward(fctx, r0, k2):
            # k2 carries the strengths the line already holds; it is the leaf for their gradient
            return torch.from_numpy(adj.forward(r0.detach().numpy()))

        @staticmethod
        def backward(fctx, g):
            dr0, dp = adj.backward(g.detach().contiguous().numpy())
            return torch.from_numpy(dr0), torch.from_numpy(dp)

    r0 = torch.tensor(small_particles(n, seed=3), dtype=torch.float64, requires_grad=True)
    k2 = torch.tensor([ring[i].poly_b[2] for i in sx], dtype=torch.float64, requires_grad=True)
    rf = Track.apply(r0, k2)
    loss = (rf[:, 0] ** 2 + rf[:, 2] ** 2).sum()
    loss.backward()
    rf2 = adj.forward(r0.detach().numpy())
    dr0, dp = adj.backward(grad_final(rf2))
    assert np.array_equal(rf.detach().numpy(), rf2)
    assert np.allclose(r0.grad.numpy(), dr0, rtol=1e-14, atol=0)
    assert np.allclose(k2.grad.numpy(), dp, rtol=1e-14, atol=0)


def test_gradient_4096_particles_512_turns(A, ctx, LT):
    """The gradient at the stated size: 4,096 Gaussian particles (seed 1) through 512 turns of the
    4D DBA, checkpoints every 64 turns, with respect to every particle's initial coordinates and
    the 36 sextupole knobs (the 72 sextupoles in mirror pairs).

    (a) Against central differences taken on the GPU's exact mode (the reference's operation
    order), every difference of the job tracked in one batched call, per particle (particles are
    independent), each derivative Richardson-extrapolated at two step sizes (knobs 3e-6 and 1e-6,
    coordinates 1e-7 and 5e-8 of the spread), over the quiet particles (a 1e-12 nudge grows at
    most 10-fold; about half the bunch) whose two estimates agree to 1e-7: the 36 knob gradients
    of their summed loss and their dL/dr0 in x, x', y, y' and delta within 1e-4 relative.  That is
    the accuracy of a difference over 512 turns, not of the adjoint (measured 2e-5 here).
    (b) Without differences over the run, against forward-mode derivatives along each particle's
    own exact-mode trajectory (products of the exact one-turn tangent maps; knob terms from
    one-turn differences) for the 8 most sensitive orbits short of chaos (nudge growth up to 1e4)
    and 8 quiet ones: dL/dr0 of each particle within 3e-10 x max(growth, 10) relative (rounding
    differences of the fused maps grow with the orbit's sensitivity; measured below 7e-11 x
    growth), the knob gradients of the 16 within 1e-6 (measured 5e-8)."""
    import bench
    ring = LT.dba_4d_ring()
    line = A.Line(ctx, ring)
    pairs = LT.sextupole_pairs(ring)
    assert len(pairs) == 36
    elems = sorted({i for p in pairs for i in p})
    params = [(i, A.F_POLYNOMB, 2) for i in elems]
    r0 = LT.gaussian_4d_particles(4096, seed=1)
    adj = A.Adjoint(line, 4096, 512, 64, params)
    rf = adj.forward(r0)
    assert not np.isnan(rf[:, 0]).any()
    res = bench.adjoint_fd_check(A, LT, ctx, adj, r0, 512, pairs, elems)
    growth = res.pop("growth")
    assert res["particles_checked"] >= 2000, res
    assert res["knob_max_rel_err"] < 1e-4, res
    assert res["coord_max_rel_err"] < 1e-4, res["coord"]
    pick = bench.tangent_picks(growth, 8, 8)
    assert np.max(growth[pick]) > 1e3
    tc = bench.adjoint_tangent_check(A, LT, ctx, adj, r0, 512, pick, pairs, elems, growth=growth)
    adj.close()
    bar = 3e-10 * np.maximum(growth[pick], 10.0)
    assert np.all(np.array(tc["coord_rel_err"]) < bar), (tc["coord_rel_err"], list(growth[pick]))
    assert tc["knob_max_rel_err"] < 1e-6, tc
