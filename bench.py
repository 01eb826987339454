#!/usr/bin/env python
"""Benchmark: FP64 particle-turns/s of the batched uneven-DA workload on B200.

Workload (one "step"): 256 error-seeded copies of the 18-cell DBA ring (quad gradient errors
1e-3, 30 um offsets as feed-down), each with its own DA grid of 21x11 .. 81x41 points over
x in [-25, 25] mm, y in [0, 12] mm, radiation damping and the RF cavity on, tracked for 1,000
turns in one batched launch sequence.  Particle-turns counts every turn a particle is tracked
(a particle lost in turn t contributes t + 1).  Inputs are synthetic (seeded numpy), resident in
HBM; the 16 MB state is smaller than L2, so a 256 MiB buffer is rewritten between steps.

`python bench.py --gpus N --steps K --warmup W` prints one JSON line (rank 0).  Under torchrun
each rank tracks its own 256 copies (seeds offset by rank): weak scaling, no collective on the
data path; timing is the max over ranks.  `--impl reference` times the reference's own CPU code
(oracle/_ref, OpenMP over all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-turns/s (FP64) fused-batched vs plain GPU at 1e-9; adjoint grads/s"
UNIT = "particle-turns/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--copies", type=int, default=256)
    ap.add_argument("--turns", type=int, default=1000)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-kernel comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (gradient) leg")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="only the adjoint leg, printed as its own JSON line (profiling runs)")
    ap.add_argument("--no-fd-check", action="store_true",
                    help="skip the adjoint's finite-difference check (profiling runs)")
    ap.add_argument("--adjoint-turns", type=int, default=512,
                    help="turns of the adjoint leg (fewer: a small case for profiling; the tapes "
                         "take about 100 MB per turn)")
    ap.add_argument("--wake-only", action="store_true",
                    help="time the bunch workload with its per-turn wake (2^20 particles) and exit")
    ap.add_argument("--wake-turns", type=int, default=200)
    ap.add_argument("--no-wake", action="store_true",
                    help="skip the bunch-wake and transverse-wake legs of the default line")
    ap.add_argument("--transwake-only", action="store_true",
                    help="time the transverse wake (sorted prefix sum against the pair sum) and exit")
    ap.add_argument("--ref-seconds", type=float, default=8.0,
                    help="CPU seconds of reference tracking per step of --impl reference")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--small", action="store_true",
                    help="profiling case: 16 copies, 20 turns, one step (for ncu)")
    ap.add_argument("--variant", type=int, default=-1, help="force a fused-kernel variant (skips autotuning)")
    ap.add_argument("--seg", type=int, default=0, help="force turns per segment")
    ap.add_argument("--engine-only", action="store_true",
                    help="only the fused engine timing: no plain, e2e, CPU legs (profiling runs)")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload_shape(copies: int, rank: int):
    """(per-copy grid sizes, particle offsets, AoS particles) of the batched DA workload; pure
    numpy, no engine library."""
    LT = importlib.import_module("accel-plus_b200.lattices")
    sizes = LT.copy_grid_sizes(copies, seed=12345 + rank)
    grids = [LT.da_grid(nx, ny) for nx, ny in sizes]
    off = np.zeros(copies + 1, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    return sizes, off, np.concatenate(grids, axis=0)


def workload(copies: int, rank: int):
    LT = importlib.import_module("accel-plus_b200.lattices")
    base = LT.dba_ring()
    sizes, off, aos = workload_shape(copies, rank)
    rings = [LT.error_copy(base, rank * copies + k) for k in range(copies)]
    return rings, off, aos, sizes


def tracked_turns(loss: np.ndarray, nturn: int) -> np.ndarray:
    return np.where(loss < 0, nturn, loss + 1).astype(np.int64)


def reference_copies(sizes, count: int = 8) -> list[int]:
    """`count` copies spread over the grid-size range: the copies at evenly spaced quantiles of
    the particle count, smallest and largest included."""
    n = np.array([nx * ny for nx, ny in sizes])
    order = np.argsort(n, kind="stable")
    q = np.linspace(0, len(n) - 1, min(count, len(n)))
    return sorted({int(order[int(round(x))]) for x in q})


def cpu_reference_rate(sizes, off, aos, rank: int = 0, turns_goal: float = 15.0, count: int = 8,
                       job_turns: int = 1000):
    """Time the reference library (oracle/_ref) — or, when it is absent, the C restatement — on
    `count` copies of the workload spread over its grid sizes, each on its full grid, OpenMP
    over all host threads, for a number of turns calibrated to take about `turns_goal` seconds
    in all.  The reference reads each copy's lattice file, written in pure Python
    (lattices.error_copy_text), so this process maps no library of the engine.  The sample's
    particle-turns/s stand for the whole job (every copy, every turn): an extrapolation.  Returns
    a dict."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    LT = importlib.import_module("accel-plus_b200.lattices")
    threads = os.cpu_count() or 1
    kind = "reference" if O.ref_available() else "port"
    copies = len(sizes)
    picks = reference_copies(sizes, count)
    if kind == "port":  # the C restatement takes descriptors (the engine's host-only reader)
        base = LT.dba_ring()

    def run(k, nturn):
        r = aos[off[k]:off[k + 1]].copy()
        seed = rank * copies + k
        if kind == "reference":
            fd, path = tempfile.mkstemp(suffix=".lat")
            with os.fdopen(fd, "w") as f:
                f.write(LT.error_copy_text(seed))
            ref = O.RefLine(path)
            os.unlink(path)
            ref.set_flags(rad=1, cavity=1)
            t = time.perf_counter()
            lt = ref.track_loss(r, nturn, threads=threads)
            dt = time.perf_counter() - t
        else:
            ring = LT.error_copy(base, seed)
            t = time.perf_counter()
            lt = O.port_track(ring, r, nturn, nthreads=threads)
            dt = time.perf_counter() - t
        return int(tracked_turns(lt, nturn).sum()), dt

    pt, dt = run(picks[0], 2)  # calibration
    rate0 = pt / max(dt, 1e-6)
    nsample = int(sum(off[k + 1] - off[k] for k in picks))
    nturn = int(max(5, min(200, turns_goal * rate0 / max(1, nsample))))
    tot_pt, tot_dt = 0, 0.0
    for k in picks:
        p, d = run(k, nturn)
        tot_pt += p
        tot_dt += d
    return {"value": tot_pt / tot_dt, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"extrapolated: {len(picks)} of the {copies} error-seeded copies spread over "
                      f"the grid sizes (copies {picks}, their full DA grids, {nsample} particles) x "
                      f"{nturn} of the {job_turns} turns, radiation + cavity on; the sample's rate "
                      f"stands for the whole job",
            "seconds": round(tot_dt, 3)}


def fp64_model_flops(LT, rings, off, loss, nturn):
    per = np.array([LT.flops_per_turn(r) for r in rings])
    turns = tracked_turns(loss, nturn)
    inst = np.repeat(np.arange(len(rings)), np.diff(off))
    return float(np.sum(per[inst] * turns))


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sizes, off, aos = workload_shape(args.copies, 0)
    vals = []
    for _ in range(max(1, args.warmup // 3)):
        cpu_reference_rate(sizes, off, aos, turns_goal=0.4 * args.ref_seconds, job_turns=args.turns)
    per_step = []
    for _ in range(args.steps):
        b = cpu_reference_rate(sizes, off, aos, turns_goal=args.ref_seconds, job_turns=args.turns)
        vals.append(b["value"])
        per_step.append(b)
    v = statistics.median(vals)
    b = per_step[-1]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * b["seconds"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_dict(args, off, aos),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": b["cores"], "kind": b["kind"],
                         "sample": b["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "process_maps_engine_library": maps_engine_library(),
        "native_so_loaded": repo_libraries_mapped(),
    }
    print(json.dumps(line), flush=True)


def repo_libraries_mapped() -> list[str]:
    """The shared libraries under this repository that this process has mapped, relative to it
    (/proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so")}
    except OSError:
        return []
    root = os.path.realpath(ROOT)
    return sorted(os.path.relpath(os.path.realpath(p), root) for p in paths
                  if os.path.realpath(p).startswith(root + os.sep))


def maps_engine_library() -> bool:
    """Whether this process has the engine's shared library mapped (/proc/self/maps)."""
    return any("libaccelgpu" in p for p in repo_libraries_mapped())


def config_dict(args, off, aos):
    return {"workload": f"batched uneven DA: {args.copies} error-seeded copies of the 18-cell DBA "
                        f"(3 GeV, radiation + RF on), grids 21x11..81x41 over x +-25 mm, y 0..12 mm, "
                        f"{args.turns} turns per step",
            "instances": args.copies, "particles": int(off[-1]), "turns": args.turns,
            "l2": "flushed between steps (256 MiB rewrite); state 6 x 8 B x particles < L2",
            "seeds": "copy k of rank r: error seed r*copies+k; grid sizes default_rng(12345+r)"}


def adjoint_leg(A, LT, ctx, steps: int = 3, ranks=None, check: bool = True, nturn: int = 512) -> dict:
    """Gradient of L = sum over particles of (x^2 + y^2) after nturn (512) turns of the 4D DBA (no cavity,
    radiation off), 4,096 Gaussian particles (seed 1), with respect to the 6 x 4,096 initial
    coordinates and the 36 sextupole knobs (mirror pairs of the 72 sextupoles), checkpointed every
    64 turns.  Under torchrun each rank takes its own 4,096 particles (seed 1 + rank) and the knob
    gradients of all ranks are summed with one all-reduce; times are the max over ranks.  The adjoint pair and the tracking it is compared with are synchronous host calls on
    the context's stream, so wall-clock time around them is device time plus microseconds.
    Finite-difference cost, in tracks of the same 4,096 particles for 512 turns, each priced at
    the faster of the tracker and the adjoint's forward pass without taping: naive central
    differences per scalar
    input 2 x (6 x 4096 + 36); batched over the independent particles (one coordinate of every
    particle at once) 2 x (6 + 36)."""
    ring = LT.dba_4d_ring()
    line = A.Line(ctx, ring)
    pairs = LT.sextupole_pairs(ring)
    elems = sorted({i for p in pairs for i in p})
    params = [(i, A.F_POLYNOMB, 2) for i in elems]
    n, every = 4096, 64
    rank = ranks.rank if ranks else 0
    r0 = LT.gaussian_4d_particles(n, seed=1 + rank)
    adj = A.Adjoint(line, n, nturn, every, params)

    def gradient():
        rf = adj.forward(r0)
        g = np.zeros_like(rf)
        live = ~np.isnan(rf[:, 0])
        g[live, 0], g[live, 2] = 2 * rf[live, 0], 2 * rf[live, 2]
        dr0, dp = adj.backward(g)
        return rf, dr0, dp

    gradient()
    t = time.perf_counter()
    t_fwd = 0.0
    for _ in range(steps):
        t1 = time.perf_counter()
        adj.forward(r0)
        t_fwd += time.perf_counter() - t1
        rf, dr0, dp = gradient()
    t_all = time.perf_counter() - t
    t_adj = (t_all - t_fwd) / steps
    t_fwd /= steps
    # the forward alone (what one finite-difference track costs): an adjoint whose tape budget
    # holds the turn starts but no Jacobians runs its forward without taping
    A.set_adjoint_tape_budget(int(8 * 6 * n * nturn * 1.01))
    adj_f = A.Adjoint(line, n, nturn, every, params)
    A.set_adjoint_tape_budget(None)
    adj_f.forward(r0)
    t = time.perf_counter()
    for _ in range(steps):
        adj_f.forward(r0)
    t_fwd_alone = (time.perf_counter() - t) / steps
    adj_f.close()
    r = r0.copy()
    line.track(r, nturn)
    t = time.perf_counter()
    for _ in range(steps):
        r = r0.copy()
        line.track(r, nturn)
    t_track = (time.perf_counter() - t) / steps
    # a finite-difference track costs the fastest forward available for this job: the tracker
    # (untuned for so few particles) or the adjoint's own forward pass over the same turns
    if ranks:
        t_adj, t_fwd, t_track = ranks.max(t_adj), ranks.max(t_fwd), ranks.max(t_track)
        t_fwd_alone = ranks.max(t_fwd_alone)
    t_fd = min(t_track, t_fwd_alone)
    knob = {e: j for j, e in enumerate(elems)}
    dknob_local = np.array([dp[knob[a]] + dp[knob[b]] for a, b in pairs])
    dknob = ranks.sum_array(dknob_local) if ranks else dknob_local
    # the gradient at this size against finite differences (this rank's particles)
    fd_check = tangent = None
    if check:
        fd_check = adjoint_fd_check(A, LT, ctx, adj, r0, nturn, pairs, elems)
        growth = fd_check.pop("growth")
        # checked without differences over the run: the most sensitive orbits short of chaos and
        # quiet ones
        tangent = adjoint_tangent_check(A, LT, ctx, adj, r0, nturn, tangent_picks(growth, 4, 4),
                                        pairs, elems, growth=growth)
    n_in = 6 * n + len(pairs)
    naive, batched = 2 * n_in, 2 * (6 + len(pairs))
    adj.close()
    line.close()
    return {"workload": f"4D DBA, 4096 particles, {nturn} turns, checkpoints every 64, 36 sextupole knobs",
            "gradients_per_s": 1.0 / t_adj, "gradient_components_per_s": n_in / t_adj,
            "ms_per_gradient": 1e3 * t_adj, "ms_forward": 1e3 * t_fwd, "ms_backward": 1e3 * (t_adj - t_fwd),
            "ms_forward_alone": 1e3 * t_fwd_alone,
            "forward_note": "ms_forward includes the Jacobian tapes written behind the forward on a "
                            "second stream; ms_forward_alone is the forward without taping",
            "ms_per_track": 1e3 * t_track,
            "fd_tracks_naive": naive, "fd_tracks_batched": batched,
            "ms_per_fd_track": 1e3 * t_fd,
            "fd_cost_ratio_naive": naive * t_fd / t_adj,
            "fd_cost_ratio_batched": batched * t_fd / t_adj,
            "survivors": int((~np.isnan(rf[:, 0])).sum()),
            "knob_gradient_norm": float(np.linalg.norm(dknob)),
            "fd_check": fd_check, "tangent_check": tangent,
            "timing": "wall clock around synchronous C-ABI calls, mean of %d" % steps}


def adjoint_fd_check(A, LT, ctx, adj, r0, nturn, pairs, elems, knob_steps=(3e-6, 1e-6),
                     coord_step=1e-7, coords=(0, 1, 2, 3, 5), quiet=10.0, tol_conv=1e-7) -> dict:
    """The adjoint's gradient of L = sum over particles of (x^2 + y^2) against central finite
    differences taken on the GPU in the exact mode (the reference's operation order, bit for bit
    the plain kernel), every difference of the job tracked together in one batched call.

    Particles are independent, so every difference is taken per particle: each copy of the bunch
    moves one knob (a sextupole pair) or one coordinate of every particle, and each particle's own
    loss l = x^2 + y^2 gives its derivative, Richardson-extrapolated (steps +-h, +-h/2; error
    O(h^4)) at two step sizes (knobs 3e-6 and 1e-6; coordinates h = 1e-7 of the spread relative to
    x's, 1e-7 for delta, and h/2).  Over 512 turns a difference is trustworthy only on an orbit
    that does not amplify small changes much: the same call tracks the bunch with x and y nudged
    by 1e-12 (relative), and the check covers the quiet particles, whose nudge grows at most
    `quiet`-fold (half of the Gaussian bunch; a few particles of its tails amplify it more than
    1e7-fold) and whose two estimates agree to tol_conv for every knob and coordinate; the adjoint
    is run with its seed dL/dr_final restricted to them (it is linear in the seed).
    Relative error of a knob: |adjoint - fd| / |fd|; of a coordinate entry: |adjoint - fd| /
    max(|fd|, 1e-3 x the largest |adjoint| of that coordinate), the bar of the smaller tests.
    Differences over 512 turns are themselves good to about 1e-5 relative at best (steps small
    enough to stay linear meet the rounding of the run): against the exact forward-mode
    derivatives of adjoint_tangent_check, the exact mode's and the fused mode's differences are
    off by 1e-6 to 1e-4 on the same particles where the adjoint agrees to 1e-7 or better.  The
    tight check of the gradient is adjoint_tangent_check; this one shows it at the full size
    against the only derivative the reference itself can give, its own tracking differenced."""
    import torch
    n = len(r0)
    ring = LT.dba_4d_ring()
    scale = np.sqrt(np.mean(r0 ** 2, axis=0))
    nudged = r0.copy()
    nudged[:, 0] *= 1 + 1e-12
    nudged[:, 2] *= 1 + 1e-12
    rings, particles, tags = [ring, ring], [r0, nudged], [("base",), ("nudged",)]
    for j, (ea, eb) in enumerate(pairs):
        for h in knob_steps:
            for dv in (h, -h, h / 2, -h / 2):
                rr = [d.copy() for d in ring]
                rr[ea].poly_b[2] += dv
                rr[eb].poly_b[2] += dv
                rings.append(rr)
                particles.append(r0)
                tags.append(("knob", j, h, dv))
    cstep = {}
    for k in coords:
        cstep[k] = coord_step * (scale[k] / scale[0] if scale[k] > 0 else 1.0)
        for h in (cstep[k], cstep[k] / 2):
            for dv in (h, -h, h / 2, -h / 2):
                a = r0.copy()
                a[:, k] += dv
                rings.append(ring)
                particles.append(a)
                tags.append(("coord", k, h, dv))
    lines = [A.Line(ctx, rr) for rr in rings]
    off = np.arange(len(lines) + 1, dtype=np.int64) * n
    soa = torch.tensor(np.ascontiguousarray(np.concatenate(particles).T), device="cuda",
                       dtype=torch.float64).contiguous()
    torch.cuda.synchronize()
    t = time.perf_counter()
    A.track_batched(lines, off, soa, nturn, mode=A.MODE_EXACT)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t
    for l in lines:
        l.close()
    out = soa.cpu().numpy().reshape(6, -1, n)
    with np.errstate(invalid="ignore"):
        lp = np.where(np.isnan(out[0]), 0.0, out[0] ** 2 + out[2] ** 2)  # [copy, particle]
    growth = nudge_growth(out[:, 0, :].T, out[:, 1, :].T)
    f = {tg: lp[i] for i, tg in enumerate(tags)}

    def rich(key, h):
        d1 = (f[key(h)] - f[key(-h)]) / (2 * h)
        d2 = (f[key(h / 2)] - f[key(-h / 2)]) / h
        return (4 * d2 - d1) / 3

    def converged(e1, e2):
        ref = np.abs(e2) + 1e-3 * np.max(np.abs(e2))
        return np.abs(e1 - e2) <= tol_conv * ref

    ok = np.isfinite(growth) & (growth <= quiet)
    kfd = np.zeros((len(pairs), n))
    for j in range(len(pairs)):
        e = [rich(lambda dv, j=j, h=h: ("knob", j, h, dv), h) for h in knob_steps]
        kfd[j] = e[-1]
        ok &= converged(e[0], e[1])
    cfd = {}
    for k in coords:
        e = [rich(lambda dv, k=k, h=h: ("coord", k, h, dv), h) for h in (cstep[k], cstep[k] / 2)]
        cfd[k] = e[-1]
        ok &= converged(e[0], e[1])
    dr0, dknob = masked_gradient(adj, r0, ok, pairs, elems)
    knob_fd = kfd[:, ok].sum(axis=1)
    knob_rel = np.abs(dknob - knob_fd) / np.abs(knob_fd)
    coord = {}
    for k in coords:
        floor = 1e-3 * np.max(np.abs(dr0[ok, k]))
        rel = np.where(ok, np.abs(dr0[:, k] - cfd[k]) / np.maximum(np.abs(cfd[k]), floor), 0.0)
        w = int(np.argmax(rel))
        coord[str(k)] = {"max_rel_err": float(rel[w]), "worst_particle": w,
                         "adjoint": float(dr0[w, k]), "fd": float(cfd[k][w])}
    return {"fd_mode": "exact (the reference's operation order), all differences in one batched call",
            "particles_checked": int(ok.sum()), "particles": n,
            "checked": f"the quiet particles: a 1e-12 nudge grows at most {quiet:g}-fold over {nturn} turns "
                       f"and the differences at two steps agree to {tol_conv:g}",
            "knobs": len(pairs), "knob_steps": list(knob_steps), "knob_max_rel_err": float(np.max(knob_rel)),
            "coord_steps": "1e-7 and 5e-8 of each coordinate's spread relative to x's",
            "coords_checked_per_particle": [int(k) for k in coords],
            "coord_max_rel_err": max(c["max_rel_err"] for c in coord.values()),
            "coord": coord, "growth": growth, "instances": len(lines), "seconds": round(secs, 2)}


def nudge_growth(base: np.ndarray, nudged: np.ndarray) -> np.ndarray:
    """How many times a 1e-12 relative nudge of x and y has grown by the end: the largest over the
    coordinates of |difference| / RMS, over 1e-12 (inf for a particle lost in either run)."""
    sc = np.sqrt(np.nanmean(base ** 2, axis=0))
    sc[sc == 0] = 1.0
    with np.errstate(invalid="ignore"):
        g = np.max(np.abs(nudged - base) / sc, axis=1) / 1e-12
    g[~np.isfinite(g)] = np.inf
    return g


def masked_gradient(adj, r0, mask, pairs, elems):
    """dL/dr0 and the knob gradients of L summed over the particles in `mask` (the adjoint's seed
    dL/dr_final is 2x, 2y there and zero elsewhere)."""
    rf = adj.forward(r0)
    g = np.zeros_like(rf)
    live = mask & ~np.isnan(rf[:, 0])
    g[live, 0], g[live, 2] = 2 * rf[live, 0], 2 * rf[live, 2]
    dr0, dp = adj.backward(g)
    knob = {e: j for j, e in enumerate(elems)}
    return dr0, np.array([dp[knob[a]] + dp[knob[b]] for a, b in pairs])


def tangent_picks(growth: np.ndarray, n_sensitive: int, n_quiet: int, seed: int = 0) -> np.ndarray:
    """Particles for adjoint_tangent_check: the n_sensitive whose 1e-12 nudge grows most while
    staying at most 1e4-fold (the most sensitive orbits short of chaos), and n_quiet drawn (seeded)
    from those whose nudge grows at most 10-fold."""
    order = np.argsort(np.where(growth <= 1e4, growth, -1.0))
    sens = order[-n_sensitive:]
    quiet = np.setdiff1d(np.nonzero(growth <= 10)[0], sens)
    q = np.random.default_rng(seed).choice(quiet, min(n_quiet, len(quiet)), replace=False)
    return np.sort(np.concatenate([sens, q]))


def adjoint_tangent_check(A, LT, ctx, adj, r0, nturn, pick, pairs, elems, hk=1e-3,
                          growth=None, detail=False) -> dict:
    """The gradient for the particles `pick` by forward-mode accumulation along each particle's
    own exact-mode trajectory, with no difference taken across more than one turn:
      coordinates: J = product over the turns of the exact one-turn tangent map about r_t
        (accel_m66_at, method 0: dual numbers through the literal element maps), dL/dr0 = J^T g;
      knobs: v_k <- M_t v_k + b_{t,k}, where b_{t,k} is the one-turn map's derivative with respect
        to knob k at r_t (central differences of one turn at +-hk, +-hk/2, Richardson-extrapolated;
        one turn amplifies nothing), dL/dk = g . v_k;
    with g = dl/dr_final = (2x, 0, 2y, 0, 0, 0).  Against the adjoint (reverse mode through the
    fused maps) this holds for particles of any sensitivity short of chaos, where differences over
    the whole run no longer converge.  Relative errors: dL/dr0 per particle, the largest
    |adjoint - tangent| over the coordinates over the largest |tangent|; the knobs, over the
    particles together, the largest |adjoint - tangent| over the largest |tangent|."""
    ring = LT.dba_4d_ring()
    line = A.Line(ctx, ring)
    kr = []
    for ea, eb in pairs:
        for dv in (hk, -hk, hk / 2, -hk / 2):
            rr = [d.copy() for d in ring]
            rr[ea].poly_b[2] += dv
            rr[eb].poly_b[2] += dv
            kr.append(rr)
    klines = [A.Line(ctx, rr) for rr in kr]
    m, nk = len(pick), len(pairs)
    off = np.arange(len(klines) + 1, dtype=np.int64) * m
    r = np.ascontiguousarray(r0[pick])
    J = np.tile(np.eye(6), (m, 1, 1))
    V = np.zeros((m, nk, 6))
    for _ in range(nturn):
        soa = np.ascontiguousarray(np.tile(r, (len(klines), 1)).T)
        A.track_batched(klines, off, soa, 1, mode=A.MODE_EXACT)
        out = soa.T.reshape(nk, 4, m, 6)
        d1 = (out[:, 0] - out[:, 1]) / (2 * hk)
        d2 = (out[:, 2] - out[:, 3]) / hk
        b = (4 * d2 - d1) / 3
        for q in range(m):
            M = line.m66_at(r[q], method=0)
            J[q] = M @ J[q]
            V[q] = V[q] @ M.T + b[:, q, :]
        line.track(r, 1, mode=A.MODE_EXACT)
    for l in klines:
        l.close()
    line.close()
    g = np.zeros((m, 6))
    g[:, 0], g[:, 2] = 2 * r[:, 0], 2 * r[:, 2]
    tangent = np.einsum("qij,qi->qj", J, g)
    tknob = np.einsum("qkj,qj->k", V, g)
    mask = np.zeros(len(r0), dtype=bool)
    mask[pick] = True
    dr0, dknob = masked_gradient(adj, r0, mask, pairs, elems)
    err = np.max(np.abs(dr0[pick] - tangent), axis=1) / np.max(np.abs(tangent), axis=1)
    kerr = np.max(np.abs(dknob - tknob)) / np.max(np.abs(tknob))
    res = {} if not detail else {"dr0": tangent.tolist(),
                                 "knob_each": np.einsum("qkj,qj->qk", V, g).tolist()}
    if growth is not None:
        gp = np.maximum(growth[pick], 10.0)
        res |= {"growth": [float(x) for x in growth[pick]],
                "coord_err_per_growth_max": float(np.max(err / gp))}
    return res | {"particles": [int(p) for p in pick], "coord_max_rel_err": float(np.max(err)),
            "coord_rel_err": [float(e) for e in err], "knob_max_rel_err": float(kerr),
            "method": "forward mode along each particle's exact-mode trajectory: exact one-turn "
                      f"tangent maps; knob terms from one-turn differences (+-{hk:g}, Richardson)"}


def parity_on_classified_copies(off, fused_soa, fused_loss, plain_soa=None, plain_loss=None):
    """The timed fused run checked on the copies whose reference outputs and per-particle
    classification are committed (tests/golden/config_golden.npz: four copies of this workload,
    1,000 turns, by the reference library): loss turns where the fate is certain (off the
    boundary and not chaotic); every survivor of certain fate against its own spread (its error
    over `amp`, what a 1e-12 nudge of its start grows to in the reference; the parity tests bar
    50 for the fused mode); regular survivors (amp < 1e-10) within 1e-9 of the reference and of
    the plain kernel; and the DA area beside the reference's and its own spread under a 1e-12
    nudge."""
    path = os.path.join(ROOT, "tests", "golden", "config_golden.npz")
    if not os.path.exists(path):
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_config_golden as MC
    cg = np.load(path)
    picks = [int(k) for k in cg["c3_copies"]]
    tot = {"regular": 0, "reg_ref": 0, "reg_plain": 0, "checked": 0, "lt_ok": 0, "worst": 0.0,
           "surv": 0, "spread": 0.0}
    areas = []
    for k in picks:
        s = slice(int(off[k]), int(off[k + 1]))
        ref, lt_ref = cg[f"c3_{k}_out"], cg[f"c3_{k}_loss"]
        amp, sc = cg[f"c3_{k}_amp"], cg[f"c3_{k}_scale"]
        unc = MC.fate_uncertain(cg[f"c3_{k}_boundary"], amp)
        surv = (lt_ref < 0) & ~unc
        reg = surv & (amp < MC.REGULAR_AMP)
        r, lt = fused_soa[:, s].T, fused_loss[s]
        with np.errstate(invalid="ignore"):
            err = np.max(np.abs(r - ref) / sc, axis=1)
        err[np.isnan(err)] = np.inf
        tot["checked"] += int((~unc).sum())
        tot["lt_ok"] += int(((lt == lt_ref) & ~unc).sum())
        tot["surv"] += int(surv.sum())
        if surv.any():
            tot["spread"] = max(tot["spread"], float(np.max(err[surv] / np.maximum(amp[surv], 1e-12))))
        tot["regular"] += int(reg.sum())
        tot["reg_ref"] += int((err[reg] < 1e-9).sum())
        if reg.any():
            tot["worst"] = max(tot["worst"], float(err[reg].max()))
        if plain_soa is not None:
            with np.errstate(invalid="ignore"):
                ep = np.max(np.abs(r - plain_soa[:, s].T) / sc, axis=1)
            tot["reg_plain"] += int((ep[reg] < 1e-9).sum())
        nx, ny = (int(v) for v in cg[f"c3_{k}_shape"])
        cell = (0.05 / (nx - 1)) * (0.012 / (ny - 1))
        a_ref = MC.grid_area(lt_ref, nx, ny)
        areas.append({"copy": k, "fused_cells_from_reference": round((MC.grid_area(lt, nx, ny) - a_ref) / cell, 1),
                      "reference_nudged_cells": [round((a - a_ref) / cell, 1) for a in cg[f"c3_{k}_pert_area"]]})
    return {"copies": picks, "turns": 1000, "particles_with_certain_fate": tot["checked"],
            "loss_turns_equal_where_fate_certain": tot["lt_ok"] / max(1, tot["checked"]),
            "survivors_with_certain_fate": tot["surv"],
            "max_error_over_reference_spread": tot["spread"],
            "regular_survivors": tot["regular"],
            "regular_within_1e-9_of_reference": tot["reg_ref"] / max(1, tot["regular"]),
            "regular_within_1e-9_of_plain": (tot["reg_plain"] / max(1, tot["regular"]))
            if plain_soa is not None else None,
            "worst_regular_rel_err": tot["worst"], "da_area": areas,
            "classification": "tests/golden/config_golden.npz: the reference re-tracked with x, y "
                              "moved by +-1e-12; fate uncertain on the boundary or where the nudge "
                              "grows past 1e-3 of the beam RMS; regular: the nudge grows below 1e-10"}


class Ranks:
    """One process per GPU, as torchrun starts them (RANK / LOCAL_RANK / WORLD_SIZE, rendezvous on
    MASTER_ADDR).  Every rank takes the same collective steps in the same order; a single process
    (WORLD_SIZE unset or 1) needs no process group.  `backend` is "nccl" for the GPU run and
    "gloo" for CPU tests of this plumbing."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 600):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dev = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if self.world > 1:
            from datetime import timedelta
            kw = {"device_id": self.dev} if backend == "nccl" else {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], device=self.dev, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX)

    def sum_array(self, a: np.ndarray) -> np.ndarray:
        """Element-wise sum over ranks of a float64 array (one all-reduce)."""
        if self.world == 1:
            return np.asarray(a, dtype=np.float64)
        t = self.torch.tensor(np.asarray(a, dtype=np.float64), device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM)

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def engine_arm(args):
    import torch

    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.small:
        args.copies, args.turns, args.steps, args.warmup = 16, 20, 1, 1
        args.no_plain = args.no_cpu = args.no_e2e = args.no_adjoint = args.no_wake = True
    if args.engine_only:
        args.no_plain = args.no_cpu = args.no_e2e = args.no_adjoint = args.no_wake = True

    rings, off, aos, sizes = workload(args.copies, rank)
    ntot = int(off[-1])
    ctx = A.Context(local)
    lines = [A.Line(ctx, r) for r in rings]
    soa0 = torch.tensor(np.ascontiguousarray(aos.T), device=dev, dtype=torch.float64).contiguous()
    state = torch.empty_like(soa0)
    loss = torch.empty(ntot, device=dev, dtype=torch.int32)
    flush = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)
    stream = torch.cuda.current_stream().cuda_stream

    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum

    def step(mode=A.MODE_FUSED, k=0):
        flush.fill_(float(k))
        state.copy_(soa0)
        A.track_batched(lines, off, state, args.turns, loss=loss, mode=mode, stream=stream)

    tile = None
    if args.variant >= 0 or args.seg > 0:
        ctx.set_tile(0, max(0, args.seg), args.variant)
        tile = ctx.get_tile()
    elif not args.no_autotune:
        tile = A.autotune(lines, off, soa0)
    for k in range(args.warmup):
        step(k=k)
    torch.cuda.synchronize()
    pt_step = float(tracked_turns(loss.cpu().numpy(), args.turns).sum())

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    n0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for k in range(args.steps):
        step(k=k)
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - n0
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms / args.steps
    total_pt = sum_over_ranks(pt_step)
    value = total_pt / (ms_step / 1e3)
    loss_np = loss.cpu().numpy()
    fused_np = state.cpu().numpy()

    # ---- roofline of the dominant kernel: one profiled step with events around each launch ----
    peak, probe_mhz = ctx.fp64_peak_clocked()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz")
    peak_theory = sms * 64 * 2 * mhz * 1e6 / 1e12 if mhz else None
    ctx.profile(True)
    step(k=0)
    fused_ms, fused_n, call_ms = ctx.profile_read()
    ctx.profile(False)
    flops = fp64_model_flops(LT, rings, off, loss_np, args.turns)
    achieved = flops / (fused_ms / 1e3) / 1e12 if fused_ms > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "fused_track_c3_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get("bytes_per_launch_full")
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": "k_fused (persistent FP64 tracker)",
                "launches": fused_n, "kernel_ms_per_step": fused_ms, "step_ms_profiled": call_ms,
                "model_flops_per_step": flops,
                "peak_source": "measured in this run: FP64 FMA-chain probe (accel_fp64_peak_clocked, "
                               "best of three 9 ms runs at full occupancy, with the SM clock it "
                               "ran at); MEASURED_PEAKS.json carries no FP64 figure",
                "peak_theoretical": peak_theory, "frac_theoretical": (achieved / peak_theory)
                if achieved and peak_theory else None,
                "peak_theoretical_basis": "SMs x 64 FP64 FMA per clock x 2 flops x the median SM "
                                          "clock sampled in the timed region",
                "probe_sm_mhz": probe_mhz,
                "probe_fma_per_clk_per_sm": (peak * 1e12 / 2 / sms / (probe_mhz * 1e6))
                if probe_mhz else None,
                "flops_model": "add/sub/mul/div = 1 at the effective multipole order "
                               "(StrMPole slice 52+3(8m+4), BendMPole slice 4*46+3(90+7m) with "
                               "radiation, drift 14)"}

    # ---- the plain per-element kernel on the same workload ----
    plain = None
    if not args.no_plain:
        step(mode=A.MODE_PLAIN)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        step(mode=A.MODE_PLAIN)
        p1.record()
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1))
        lp = loss.cpu().numpy()
        sp = state.cpu().numpy()
        pt_plain = sum_over_ranks(float(tracked_turns(lp, args.turns).sum()))
        diff = lp != loss_np
        plain = {"value": pt_plain / (pms / 1e3), "ms_per_step": pms,
                 "fused_over_plain": value / (pt_plain / (pms / 1e3)),
                 "loss_turn_mismatches": int(diff.sum()),
                 "mismatch_note": "particles whose loss turn differs between the two kernels; the "
                                  "parity tests confine such differences to the chaotic aperture edge",
                 "survival_mismatches": int(((lp < 0) != (loss_np < 0)).sum())}
        # the exact mode: the plain kernel's arithmetic with the state in registers over turns
        step(mode=A.MODE_EXACT)
        torch.cuda.synchronize()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x0.record()
        step(mode=A.MODE_EXACT)
        x1.record()
        torch.cuda.synchronize()
        xms = max_over_ranks(x0.elapsed_time(x1))
        lx = loss.cpu().numpy()
        sx = state.cpu().numpy()
        pt_exact = sum_over_ranks(float(tracked_turns(lx, args.turns).sum()))
        same = bool(np.array_equal(lx, lp) and np.array_equal(sx.view(np.int64), sp.view(np.int64)))
        plain["exact"] = {"value": pt_exact / (xms / 1e3), "ms_per_step": xms,
                          "exact_over_plain": (pt_exact / (xms / 1e3)) / (pt_plain / (pms / 1e3)),
                          "bit_identical_to_plain": same}

    # ---- parity of the timed run on the copies the reference's outputs are committed for ----
    parity = None
    if rank == 0 and args.copies == 256 and args.turns == 1000:
        parity = parity_on_classified_copies(off, fused_np, loss_np, None if plain is None else sp,
                                             None if plain is None else lp)

    # ---- end to end through the C-ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        # the user's call: page-locked host arrays handed straight to accel_track_batched, which
        # copies them in, tracks, copies the state and loss turns back and returns when done
        h_in = torch.tensor(np.ascontiguousarray(aos.T), dtype=torch.float64).pin_memory()
        h_state = torch.empty_like(h_in).pin_memory()
        h_loss = torch.empty(ntot, dtype=torch.int32).pin_memory()

        def e2e_step(k):
            flush.fill_(float(k))
            h_state.copy_(h_in)  # this step's input (the call tracks in place)
            A.track_batched(lines, off, h_state, args.turns, loss=h_loss, stream=stream)

        e2e_step(0)
        torch.cuda.synchronize()
        same = bool(np.array_equal(h_loss.numpy(), loss_np))
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            e2e_step(k)
        e1.record()
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1)) / args.steps
        e2e = {"value": total_pt / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h_in.numel() * 8),
               "d2h_bytes_per_step": int(h_state.numel() * 8 + h_loss.numel() * 4),
               "loss_turns_equal_device_run": same,
               "ms_per_step": ems,
               "path": "host pointers through accel_track_batched (C-ABI): page-locked SoA state "
                       "and loss turns, copied in and out inside the call"}

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(A, LT, ctx, ranks=ranks, check=not args.no_fd_check, nturn=args.adjoint_turns)

    # the collective workloads: a 2^20-particle bunch with its per-turn longitudinal wake, and the
    # transverse wake's sorted sum against the pair sum (each rank on its own GPU)
    wake = transwake = None
    if not args.no_wake:
        wake = wake_leg(A, LT, ctx, nturn=args.wake_turns)
        transwake = transwake_leg(A, ctx)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_rate(sizes, off, aos, job_turns=args.turns)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args, off, aos), "roofline": roofline, "cpu_baseline": cpu,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "plain": plain,
            "parity": parity, "adjoint": adjoint, "bunch_wake": wake, "transverse_wake": transwake,
            "tile": {"block": tile[0], "seg_turns": tile[1], "variant": tile[2] % 100,
                     "sched": ["atomic chunks per warp", "contiguous range per block",
                               "instance-staged blocks (element hot lines in shared memory)"][tile[2] // 100]}
                    if tile else None,
            "particle_turns_per_step": total_pt,
            "survivors": int((loss_np < 0).sum()),
        }
        print(json.dumps(line), flush=True)
    for l in lines:
        l.close()
    ctx.close()
    ranks.close()


def wake_leg(A, LT, ctx, nturn: int = 200, n: int = 1 << 20) -> dict:
    """The bunch workload with its collective step: the DBA with radiation and quantum excitation,
    the cavity on, and a broadband longitudinal resonator wake (Rs 1 kOhm, Q 1, fr 10 GHz, 256
    bins) applied once per turn to 2^20 particles drawn from the matched Gaussian (sigma_z 3 mm,
    sigma_delta 1e-3, 10 nm / 10 pm).  The state stays on the device (SoA); timed with CUDA events
    on the launching stream after a warm-up, over `nturn` turns of the 10,000 the full run takes."""
    import torch
    ring = LT.dba_ring()
    m = A.Line(ctx, ring).m66()
    wring = ring + [LT.longwake_elem()]
    line = A.Line(ctx, wring)
    line.set_flags(rad=A.RAD_RADQE, cavity=1, wake=1)
    line.set_seed(2024)
    r = LT.matched_bunch_particles(n, m, seed=5)
    st = torch.tensor(np.ascontiguousarray(r.T), device="cuda", dtype=torch.float64).contiguous()
    s = torch.cuda.current_stream()
    line.track(st, 5, layout=A.LAYOUT_SOA, stream=s.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    line.track(st, nturn, layout=A.LAYOUT_SOA, stream=s.cuda_stream)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    x = st.cpu().numpy()
    live = ~np.isnan(x[0])
    return {"workload": "18-cell DBA, radiation + quantum excitation + RF, longitudinal broadband "
                        "wake once per turn (256 bins), matched Gaussian bunch",
            "particles": n, "turns": nturn, "ms_per_turn": ms / nturn,
            "particle_turns_per_s": n * nturn / (ms / 1e3),
            "live": int(live.sum()), "sigma_z_m": float(np.std(x[4, live])),
            "sigma_delta": float(np.std(x[5, live])),
            "timing": "CUDA events on the launching stream, state resident on the device"}


def transwake_leg(A, ctx, sizes=(65536, 1 << 20), pair_n: int = 65536) -> dict:
    """The transverse resonator wake (ATransWake: 3 GeV, Ne 2, Wx 50 / fRx 10 GHz / Qx 1.5,
    Wy 40 / fRy 12 GHz / Qy 2, 0.5 m) between two drifts, on a Gaussian bunch (x 1 mm, y 0.5 mm,
    z 3 mm, delta 1e-3): the fused mode's z-sorted prefix sum at each size, the plain mode's pair
    sum (the reference's O(N^2) order of operations) at `pair_n`, and their agreement after one
    pass there.  CUDA events on the launching stream, state resident on the device (SoA)."""
    import torch
    tw = A.elem(A.TRANSWAKE, "TW", 0.5, f=[3000, 2.0, 50.0, 10.0, 1.5, 40.0, 12.0, 2.0], flags=1)
    line = A.Line(ctx, [A.elem(A.DRIFT, "D", 0.3), tw, A.elem(A.DRIFT, "D", 0.2)])
    s = torch.cuda.current_stream()

    def bunch(n):
        rng = np.random.default_rng(3)
        r = np.zeros((6, n))
        r[0] = rng.normal(0, 1e-3, n)
        r[2] = rng.normal(0, 5e-4, n)
        r[4] = rng.normal(0, 3e-3, n)
        r[5] = rng.normal(0, 1e-3, n)
        return torch.tensor(r, device="cuda", dtype=torch.float64).contiguous()

    def timed(st, mode, turns):
        line.track(st, 3, layout=A.LAYOUT_SOA, mode=mode, stream=s.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        line.track(st, turns, layout=A.LAYOUT_SOA, mode=mode, stream=s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / turns

    out = {"workload": "transverse resonator wake between two drifts, Gaussian bunch", "sorted": {}}
    for n in sizes:
        out["sorted"][str(n)] = {"ms_per_pass": timed(bunch(n), A.MODE_FUSED, 20)}
    out["pair"] = {str(pair_n): {"ms_per_pass": timed(bunch(pair_n), A.MODE_PLAIN, 3)}}
    r0 = bunch(pair_n)
    a, b = r0.clone(), r0.clone()
    line.track(a, 1, layout=A.LAYOUT_SOA, mode=A.MODE_PLAIN, stream=s.cuda_stream)
    line.track(b, 1, layout=A.LAYOUT_SOA, mode=A.MODE_FUSED, stream=s.cuda_stream)
    torch.cuda.synchronize()
    kick = (a[1] - r0[1]).abs().max().item()
    out["sorted_vs_pair_rel"] = (b[1] - a[1]).abs().max().item() / kick
    out["timing"] = "CUDA events on the launching stream, 20 passes (sorted) / 3 (pair) after 3 warm-up"
    return out


def transwake_only():
    A = importlib.import_module("accel-plus_b200")
    ctx = A.Context(0)
    print(json.dumps({"transwake": transwake_leg(A, ctx)}), flush=True)
    ctx.close()


def wake_only(turns: int, variant: int = -1):
    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    ctx = A.Context(0)
    if variant >= 0:
        ctx.set_tile(0, 0, variant)
    out = wake_leg(A, LT, ctx, nturn=turns)
    out["tile"] = ctx.get_tile()
    print(json.dumps({"wake": out}), flush=True)
    ctx.close()


def adjoint_only(check: bool = True, nturn: int = 512):
    A = importlib.import_module("accel-plus_b200")
    LT = importlib.import_module("accel-plus_b200.lattices")
    ctx = A.Context(0)
    print(json.dumps({"adjoint": adjoint_leg(A, LT, ctx, check=check, nturn=nturn)}), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.adjoint_only:
        adjoint_only(check=not args.no_fd_check, nturn=args.adjoint_turns)
        return
    if args.wake_only:
        wake_only(args.wake_turns, args.variant)
        return
    if args.transwake_only:
        transwake_only()
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
