"""Reference outputs of the tracking workloads at their stated sizes, with each particle's
sensitivity classified, so the GPU parity tests compare against the reference without
re-tracking anything on the CPU.

Run where the reference sources exist (oracle/Makefile compiles them into
oracle/_ref/libaccel_ref.so):

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_config_golden.py

Cases (every input is regenerated from its seed by accel-plus_b200/lattices.py):
  c1      the 32-cell FODO (fodo32.lat), 1,024 particles x uniform in +-5 mm, y in +-2 mm
          (default_rng(0)), 1,000 turns, radiation, cavity and wake off
  c2      the 18-cell DBA with radiation and RF on (dba_ring), a 101 x 51 grid over x in
          [-25, 25] mm, y in [0, 12] mm, 1,024 turns
  c3_<k>  error-seeded copy k of that DBA (error_copy(base, k)) on its full grid from
          copy_grid_sizes(256, 12345)[k], 1,000 turns; four copies spanning the grid-size range

Each case is tracked by the reference's ALine::pass one turn at a time with the per-turn NaN
scan of trackDA (aline.cpp:646-659), OpenMP over all host threads (bit-identical to one thread
without quantum excitation), and then twice more with x and y perturbed by +-1e-12 (relative,
plus 1e-15 m absolute).  Stored per case:
  <case>_out       final AoS state (N x 6)
  <case>_loss      loss turn per particle (-1 = survived)
  <case>_boundary  fate changes under the perturbation, or (grids) a grid neighbour's fate
                   differs: the chaotic aperture boundary, where either fate is accepted
  <case>_amp       how far the perturbed runs are from the unperturbed one at the end of the
                   last turn the particle survives (the final turn for survivors): the largest
                   over both signs and the six coordinates of |difference| / RMS (inf when a
                   perturbed run loses the particle in another turn).  A lost particle with a
                   large amp was on a chaotic orbit before its loss, and its loss turn is fragile
  <case>_regular   survives, off the boundary, and amp < REGULAR_AMP (1e-10: the nudge grows at
                   most 100-fold)
  <case>_scale     that RMS per coordinate over the surviving particles
  <case>_pert_area (grids) the DA area of the two perturbed runs, for the area tolerance
  c3_copies        the copy indices; <case>_shape (nx, ny) for grids
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

A = importlib.import_module("accel-plus_b200")
LT = importlib.import_module("accel-plus_b200.lattices")
import oracle as O  # noqa: E402

EPS = 1e-12
OUT = os.path.join(HERE, "config_golden.npz")
# A particle whose end state (or state before its loss) moves by more than this fraction of the
# beam RMS under the 1e-12 nudge, a billion-fold amplification, is on a chaotic orbit: its fate
# over the run is decided at the rounding level, and in this lattice even two reference runs 1e-12
# apart may keep it alive in both while ending O(1) apart.
CHAOTIC_AMP = 1e-3
# a regular orbit: the 1e-12 nudge grows at most 100-fold by the end
REGULAR_AMP = 1e-10


def fate_uncertain(boundary, amp):
    """The particles whose fate or loss turn a rounding-level difference may change: the
    boundary found by the perturbed runs and the grid neighbours, plus the chaotic orbits."""
    return boundary | (amp > CHAOTIC_AMP)


def ref_line(elems, rad: int, cavity: int):
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, elems)
    line = O.RefLine(path)
    os.unlink(path)
    line.set_flags(rad=rad, cavity=cavity)
    return line


def perturbed(r0: np.ndarray, sgn: float) -> np.ndarray:
    g = r0.copy()
    for k in (0, 2):
        g[:, k] = g[:, k] * (1 + sgn * EPS) + sgn * EPS * 1e-3
    return g


def rms_scale(r: np.ndarray) -> np.ndarray:
    live = ~np.isnan(r[:, 0])
    sc = np.sqrt(np.mean(r[live] ** 2, axis=0)) if live.any() else np.ones(6)
    sc[sc == 0] = 1.0
    return sc


def grid_area(loss: np.ndarray, nx: int, ny: int, x0=-0.025, x1=0.025, y0=0.0, y1=0.012) -> float:
    """DA area of a Cartesian grid by trackDA's triangle fan (aline.cpp:675-708): in each column
    the boundary point is the first lost point going up from y0 (the top point when none is
    lost), and the fan from the origin over the columns' boundary points, in order of angle,
    sums 0.5 r1 r2 sin(dphi)."""
    surv = (loss < 0).reshape(ny, nx)
    xs = np.linspace(x0, x1, nx)
    ys = np.linspace(y0, y1, ny)
    rx, ry = np.empty(nx), np.empty(nx)
    for i in range(nx):
        lost = np.nonzero(~surv[:, i])[0]
        rx[i] = xs[i]
        ry[i] = ys[lost[0]] if len(lost) else ys[-1]
    order = np.argsort(np.arctan2(ry, rx))
    rx, ry = rx[order], ry[order]
    s = 0.0
    for i in range(1, nx):
        rd1 = np.hypot(rx[i - 1], ry[i - 1])
        rd2 = np.hypot(rx[i], ry[i])
        dphi = np.arctan2(ry[i], rx[i]) - np.arctan2(ry[i - 1], rx[i - 1])
        s += 0.5 * rd1 * rd2 * np.sin(dphi)
    return float(s)


def classify(line, r0: np.ndarray, nturn: int, threads: int, shape=None) -> dict:
    t0 = time.perf_counter()
    out = r0.copy()
    last = np.empty_like(r0)
    lt = line.track_loss(out, nturn, threads=threads, last=last)
    sc = rms_scale(out)
    sens = np.zeros(len(r0), dtype=bool)
    amp = np.zeros(len(r0))
    areas = []
    for sgn in (1.0, -1.0):
        g = perturbed(r0, sgn)
        gl = np.empty_like(r0)
        lg = line.track_loss(g, nturn, threads=threads, last=gl)
        sens |= lg != lt
        with np.errstate(invalid="ignore"):
            d = np.max(np.abs(gl - last) / sc, axis=1)
        d[np.isnan(d) | (lg != lt)] = np.inf
        amp = np.maximum(amp, d)
        if shape:
            areas.append(grid_area(lg, *shape))
    boundary = sens.copy()
    if shape:
        nx, ny = shape
        fate = (lt < 0).reshape(ny, nx)
        near = np.zeros_like(fate)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ys = slice(max(0, dy), ny + min(0, dy))
                yd = slice(max(0, -dy), ny + min(0, -dy))
                xs = slice(max(0, dx), nx + min(0, dx))
                xd = slice(max(0, -dx), nx + min(0, -dx))
                near[yd, xd] |= fate[ys, xs] != fate[yd, xd]
        boundary |= near.ravel()
    regular = (lt < 0) & ~boundary & (amp < REGULAR_AMP)
    res = {"out": out, "loss": lt.astype(np.int32), "boundary": boundary, "regular": regular,
           "scale": sc, "amp": amp}
    if shape:
        res["shape"] = np.array(shape, dtype=np.int32)
        res["pert_area"] = np.array(areas)
    print(f"  N={len(r0)} turns={nturn}: survivors {int((lt < 0).sum())}, boundary "
          f"{int(boundary.sum())}, regular {int(regular.sum())}, {time.perf_counter() - t0:.0f} s",
          flush=True)
    return res


def c3_copies(sizes) -> list[int]:
    """Four copies spanning the grid sizes: the smallest, the largest, and two near the
    first and third quartiles of the particle count."""
    n = np.array([nx * ny for nx, ny in sizes])
    order = np.argsort(n, kind="stable")
    picks = [int(order[0]), int(order[len(n) // 4]), int(order[(3 * len(n)) // 4]), int(order[-1])]
    return sorted(set(picks))


def main():
    threads = os.cpu_count() or 1
    only = set(sys.argv[1:])
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}

    def store(prefix, res):
        for k, v in res.items():
            out[f"{prefix}_{k}"] = v
        np.savez_compressed(OUT, **out)

    if not only or "c1" in only:
        print("c1: FODO, 1024 particles, 1000 turns", flush=True)
        line = ref_line(LT.fodo_ring(), rad=0, cavity=0)
        store("c1", classify(line, LT.fodo_particles(), 1000, threads))
    if not only or "c2" in only:
        print("c2: DBA, 101 x 51 grid, 1024 turns", flush=True)
        line = ref_line(LT.dba_ring(), rad=1, cavity=1)
        store("c2", classify(line, LT.da_grid(101, 51), 1024, threads, shape=(101, 51)))
    if not only or "c3" in only:
        sizes = LT.copy_grid_sizes(256, 12345)
        base = LT.dba_ring()
        picks = c3_copies(sizes)
        out["c3_copies"] = np.array(picks, dtype=np.int32)
        for k in picks:
            nx, ny = sizes[k]
            print(f"c3 copy {k}: {nx} x {ny} grid, 1000 turns", flush=True)
            line = ref_line(LT.error_copy(base, k), rad=1, cavity=1)
            store(f"c3_{k}", classify(line, LT.da_grid(nx, ny), 1000, threads, shape=(nx, ny)))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
