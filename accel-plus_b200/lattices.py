"""Synthetic rings and particle sets for the five tracking workloads.

  fodo32     32-cell FODO at 3 GeV: QF/QD StrMPole quads (0.25 m, K = +-1.2, 10 slices), 2.0 m
             drifts, BendMPole sector bends (1.0 m, 2 pi/64), 0.5 m drifts, SF/SD sextupoles
             (0.2 m).  Sextupole strengths come from the reference's correct_chrom to (1, 1).
  dba18      18-cell double-bend achromat at 3 GeV, circumference 372 c / 476 MHz: per cell two
             BendMPole bends (1.5 m, 2 pi/36), six StrMPole quads, four StrMPole sextupoles; one
             zero-length RF cavity (3.2 MV, 476 MHz, harmonic 372) at the ring start and one
             +-50 mm aperture at the ring end.
  copies     error-seeded copies of a ring: quad gradient errors N(0, 1e-3) relative, quad and
             sextupole transverse offsets N(0, 30 um) truncated at 2 sigma, written as exact
             feed-down multipoles (the reference elements carry no offset fields).
  grids      Cartesian DA grids over x in [-25, 25] mm, y in [0, 12] mm at z = delta = 0.

Everything is generated from numpy's seeded default_rng, so a workload is a pure function of
its seed.  Element descriptors are accel_elem_desc structures from the package.
"""
from __future__ import annotations

import importlib
import math
import os
from math import comb
from typing import Sequence

import numpy as np

A = importlib.import_module("accel-plus_b200")

C0 = 2.99792458e8
HARMONIC = 372
F_RF = 476e6
CIRCUMFERENCE = HARMONIC * C0 / F_RF          # 234.292... m
GOLDEN_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")

# DBA quad strengths (m^-2): a periodic-optics scan of the cell picked this working point, ring
# tunes ~ (7.18, 5.37), natural chromaticity ~ (-5.6, -10.8), M56 < 0 (stable with the reference's
# asin RF phase); corrected to chromaticity (1, 1) the sextupoles stay near 20 m^-3
DBA_KF1, DBA_KD1, DBA_KF2 = 0.525, -1.475, 0.625


def fodo32(b2_sf: float = 0.0, b2_sd: float = 0.0, ncell: int = 32) -> list:
    e = A.elem
    ang = 2 * math.pi / 64
    out = []
    for _ in range(ncell):
        out += [
            e(A.STRMPOLE, "QF", 0.25, max_npole=4, poly_b=[0, 1.2]),
            e(A.DRIFT, "D2", 2.0),
            e(A.BENDMPOLE, "B", 1.0, f=[ang, 0, 0, 3000], max_npole=1),
            e(A.DRIFT, "D05", 0.5),
            e(A.STRMPOLE, "SF", 0.2, max_npole=4, poly_b=[0, 0, b2_sf]),
            e(A.STRMPOLE, "QD", 0.25, max_npole=4, poly_b=[0, -1.2]),
            e(A.DRIFT, "D2", 2.0),
            e(A.BENDMPOLE, "B", 1.0, f=[ang, 0, 0, 3000], max_npole=1),
            e(A.DRIFT, "D05", 0.5),
            e(A.STRMPOLE, "SD", 0.2, max_npole=4, poly_b=[0, 0, b2_sd]),
        ]
    return out


def dba_cell(b2_sd: float = 0.0, b2_sf: float = 0.0, kf1=DBA_KF1, kd1=DBA_KD1, kf2=DBA_KF2) -> list:
    """One DBA cell, mirror-symmetric about its centre:
       D0 QF1 D1 B D2 SD D3 QD1 D4 SF D5 QF2 D6 | D6 QF2 D5 SF D4 QD1 D3 SD D2 B D1 QF1 D0
    The straight-section half length D0 takes what the fixed circumference leaves over."""
    e = A.elem
    ang = 2 * math.pi / 36
    dq = 0.2
    d0 = CIRCUMFERENCE / 36 - (0.4 + 1.5 + 0.2 + 0.3 + 0.2 + 0.5) - (0.4 + 0.25 + 4 * dq)
    half = [
        e(A.DRIFT, "D0", d0),
        e(A.STRMPOLE, "QF1", 0.4, max_npole=4, poly_b=[0, kf1]),
        e(A.DRIFT, "D1", 0.4),
        e(A.BENDMPOLE, "B", 1.5, f=[ang, 0, 0, 3000], max_npole=1),
        e(A.DRIFT, "D2", 0.25),
        e(A.STRMPOLE, "SD", 0.2, max_npole=4, poly_b=[0, 0, b2_sd]),
        e(A.DRIFT, "D3", dq),
        e(A.STRMPOLE, "QD1", 0.3, max_npole=4, poly_b=[0, kd1]),
        e(A.DRIFT, "D4", dq),
        e(A.STRMPOLE, "SF", 0.2, max_npole=4, poly_b=[0, 0, b2_sf]),
        e(A.DRIFT, "D5", dq),
        e(A.STRMPOLE, "QF2", 0.5, max_npole=4, poly_b=[0, kf2]),
        e(A.DRIFT, "D6", dq),
    ]
    # the sextupole pairs of a cell share family names, so the reference's correct_chrom moves
    # all SD and all SF together; the adjoint's 36 knobs are the per-cell pairs
    return half + [d.copy() for d in half[::-1]]


def dba18(b2_sd: float = 0.0, b2_sf: float = 0.0, voltage_mv: float = 3.2, phis: float = 0.0,
          cavity: bool = True, aperture: bool = True) -> list:
    e = A.elem
    out = []
    if cavity:
        f = HARMONIC * C0 / ring_length(dba_cell() * 18)
        out.append(e(A.CAVITY, "RF", 0.0, f=[voltage_mv, f, phis, 3000]))
    for _ in range(18):
        out += dba_cell(b2_sd, b2_sf)
    if aperture:
        out.append(e(A.APERTURE, "AP", 0.0, f=[-0.05, 0.05, -0.05, 0.05]))
    return out


def ring_length(elems: Sequence) -> float:
    return float(sum(d.len for d in elems))


# ---- committed lattices (chromaticity corrected by the reference, see tests/golden) ----------
def load_golden(name: str) -> list:
    path = os.path.join(GOLDEN_DIR, name)
    return A.read_lattice(path)


def fodo_ring() -> list:
    return load_golden("fodo32.lat")


def dba_ring() -> list:
    """DBA with the RF phase from setrfphase; radiation (classical) and cavity on."""
    ring = load_golden("dba18.lat")
    for d in ring:
        if d.type == A.BENDMPOLE:
            d.flags = A.RAD_RAD
        if d.type == A.CAVITY:
            d.flags = 1
    return ring


def dba_4d_ring() -> list:
    """The 18-cell DBA without its cavity, radiation off (4D)."""
    ring = [d for d in load_golden("dba18.lat") if d.type != A.CAVITY]
    for d in ring:
        if d.type == A.BENDMPOLE:
            d.flags = A.RAD_OFF
    return ring


def sextupole_pairs(ring: Sequence) -> list[tuple[int, int]]:
    """36 knobs: per cell, the SD pair and the SF pair (mirror images within the cell)."""
    sd = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.name == "SD"]
    sf = [i for i, d in enumerate(ring) if d.type == A.STRMPOLE and d.name == "SF"]
    pairs = []
    for c in range(len(sd) // 2):
        pairs.append((sd[2 * c], sd[2 * c + 1]))
        pairs.append((sf[2 * c], sf[2 * c + 1]))
    return pairs


# ---- error seeds as feed-down ---------------------------------------------------------------
def feed_down(a: np.ndarray, b: np.ndarray, dx: float, dy: float) -> tuple[np.ndarray, np.ndarray]:
    """Multipoles of an element displaced by (dx, dy), expressed in the undisplaced frame.

    The field sum_n (B_n + i A_n)(x + i y)^n seen at (x - dx, y - dy) equals
    sum_k c'_k (x + i y)^k with c'_k = sum_{n>=k} C(n, k) c_n (-(dx + i dy))^(n-k).
    Drifts commute with a transverse translation, so tracking the lab-frame particle through
    these coefficients is the displaced element exactly (up to rounding).
    """
    c = b.astype(complex) + 1j * a.astype(complex)
    w = -(dx + 1j * dy)
    out = np.zeros_like(c)
    for k in range(len(c)):
        out[k] = sum(comb(n, k) * c[n] * w ** (n - k) for n in range(k, len(c)))
    return out.imag.copy(), out.real.copy()


def _strmpole_errors(rng, a: np.ndarray, b: np.ndarray, dk_rel: float, sigma_off: float):
    """The errors of one StrMPole, drawn from `rng` in a fixed order: a gradient error when the
    element is a pure quadrupole, then the x and y offsets (each redrawn until inside 2 sigma);
    returns the feed-down (poly_a, poly_b) over MAX_MPOLE orders."""
    b = b.copy()
    is_quad = b[1] != 0 and not np.any(b[2:]) and not np.any(a)
    if is_quad:
        b[1] *= 1.0 + rng.normal(0.0, dk_rel)
    offs = []
    for _ in range(2):
        v = rng.normal(0.0, sigma_off)
        while abs(v) > 2 * sigma_off:
            v = rng.normal(0.0, sigma_off)
        offs.append(v)
    return feed_down(a, b, offs[0], offs[1])


def error_copy(base: Sequence, seed: int, dk_rel: float = 1e-3, sigma_off: float = 30e-6) -> list:
    """One error-seeded copy: quads get dK/K ~ N(0, dk_rel), quads and sextupoles get offsets
    N(0, sigma_off) truncated at 2 sigma (redrawn until inside), all from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for d in base:
        d = d.copy()
        if d.type == A.STRMPOLE:
            b = np.array(d.poly_b[:], dtype=np.float64)
            a = np.array(d.poly_a[:], dtype=np.float64)
            a2, b2 = _strmpole_errors(rng, a, b, dk_rel, sigma_off)
            for i in range(A.MAX_MPOLE):
                d.poly_a[i] = float(a2[i])
                d.poly_b[i] = float(b2[i])
        out.append(d)
    return out


def error_copy_text(seed: int, base_text: str | None = None, dk_rel: float = 1e-3,
                    sigma_off: float = 30e-6) -> str:
    """The lattice file of error_copy(dba_ring(), seed), made from the text of dba18.lat in
    pure Python (no engine library): the same draws in the same order, each StrMPole's two
    coefficient lines rewritten with 17 significant digits, every other line kept.  The result
    equals accel_lattice_write of the descriptor copy, character for character (the lattice
    format carries no radiation or cavity flags)."""
    if base_text is None:
        with open(os.path.join(GOLDEN_DIR, "dba18.lat")) as f:
            base_text = f.read()
    rng = np.random.default_rng(seed)
    lines = base_text.split("\n")
    out = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        head = ln.split()
        out.append(ln)
        i += 1
        if len(head) >= 5 and head[1] == ":" and head[2] == "StrMPole":
            npole = int(head[4])
            b = np.zeros(A.MAX_MPOLE)
            a = np.zeros(A.MAX_MPOLE)
            b[:npole] = [float(x) for x in lines[i].split()]
            a[:npole] = [float(x) for x in lines[i + 1].split()]
            a2, b2 = _strmpole_errors(rng, a, b, dk_rel, sigma_off)
            for arr in (b2, a2):
                out.append("\t\t\t" + "".join("%.17g\t" % float(arr[k]) for k in range(npole)))
            i += 2
    return "\n".join(out)


# ---- particle sets --------------------------------------------------------------------------
def da_grid(nx: int, ny: int, x0=-0.025, x1=0.025, y0=0.0, y1=0.012) -> np.ndarray:
    """nx x ny grid (x fastest) of AoS particles, z = delta = 0."""
    xs = np.linspace(x0, x1, nx)
    ys = np.linspace(y0, y1, ny)
    r = np.zeros((ny, nx, 6))
    r[:, :, 0] = xs[None, :]
    r[:, :, 2] = ys[:, None]
    return r.reshape(-1, 6).copy()


def fodo_particles(n: int = 1024, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 6))
    r[:, 0] = rng.uniform(-5e-3, 5e-3, n)
    r[:, 2] = rng.uniform(-2e-3, 2e-3, n)
    return r


def copy_grid_sizes(ncopy: int = 256, seed: int = 12345) -> list[tuple[int, int]]:
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(21, 82)), int(rng.integers(11, 42))) for _ in range(ncopy)]


def batched_da_workload(ncopy: int = 256, seed: int = 12345):
    """(rings, part_off, AoS particles) for the batched uneven-DA workload."""
    base = dba_ring()
    sizes = copy_grid_sizes(ncopy, seed)
    rings = [error_copy(base, k) for k in range(ncopy)]
    grids = [da_grid(nx, ny) for nx, ny in sizes]
    off = np.zeros(ncopy + 1, dtype=np.int64)
    off[1:] = np.cumsum([g.shape[0] for g in grids])
    return rings, off, np.concatenate(grids, axis=0)


def gaussian_4d_particles(n: int = 4096, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 6))
    r[:, 0] = rng.normal(0, 1e-3, n)
    r[:, 1] = rng.normal(0, 50e-6, n)
    r[:, 2] = rng.normal(0, 0.5e-3, n)
    r[:, 3] = rng.normal(0, 50e-6, n)
    return r


def twiss_from_m66(m: np.ndarray):
    """Periodic (beta, alpha) in x and y from a one-turn matrix (ALine::calctwiss, aline.cpp:1092)."""
    out = []
    for k in (0, 2):
        cmu = 0.5 * (m[k, k] + m[k + 1, k + 1])
        mu = math.acos(cmu)
        s = math.sin(mu)
        if m[k, k + 1] < 0:
            s = -s
        out.append((m[k, k + 1] / s, (m[k, k] - m[k + 1, k + 1]) / (2 * s)))
    return out


def matched_bunch_particles(n: int, m66: np.ndarray, seed: int = 5, ex=10e-9, ey=10e-12, sz=3e-3,
                      sd=1e-3) -> np.ndarray:
    """Gaussian bunch matched to the ring-entrance Twiss of m66."""
    rng = np.random.default_rng(seed)
    (bx, ax), (by, ay) = twiss_from_m66(m66)
    r = np.zeros((n, 6))
    for k, (b, a, e) in ((0, (bx, ax, ex)), (2, (by, ay, ey))):
        u = rng.normal(0, 1, n)
        v = rng.normal(0, 1, n)
        r[:, k] = math.sqrt(e * b) * u
        r[:, k + 1] = math.sqrt(e / b) * (v - a * u)
    r[:, 4] = rng.normal(0, sz, n)
    r[:, 5] = rng.normal(0, sd, n)
    return r


def longwake_elem(energy_mev=3000.0, charge_nc=1.0, rs=1e3, fr=10e9, q=1.0, nbins=256):
    return A.elem(A.LONGWAKE, "WAKE", 0.0, f=[energy_mev, charge_nc, rs, fr, q, nbins], flags=1)


def flops_per_turn(ring: Sequence) -> float:
    """Algorithmic flops per particle-turn (add/sub/mul/div = 1) at the effective multipole order:
    StrMPole slice 52 + 3 (8 m + 4); BendMPole slice 4*46 + 3 (44 + 7 m) (radiation: 90 + 7 m per
    kick); drift 14; quad 60; bend 98; cavity 6 (+28 with length)."""
    f = 0.0
    for d in ring:
        t = d.type
        if t == A.DRIFT:
            f += 14
        elif t == A.STRMPOLE:
            m = max([i for i in range(A.MAX_MPOLE) if d.poly_a[i] != 0 or d.poly_b[i] != 0] or [0])
            f += (8 * m + 6) if d.len == 0 else d.nslice * (52 + 3 * (8 * m + 4))
        elif t == A.BENDMPOLE:
            m = max([i for i in range(d.max_npole) if d.poly_b[i] != 0] or [0])
            kick = (90 + 7 * m) if d.flags >= 1 else (44 + 7 * m)
            f += (d.nslice * (2 * 46 + kick) if d.flags == 2 else d.nslice * (4 * 46 + 3 * kick)) + 8
        elif t == A.QUAD:
            f += 60
        elif t == A.BEND:
            f += 98
        elif t == A.CAVITY:
            f += 6 + (28 if d.len else 0)
        elif t in (A.CORRECTOR, A.SYNCRAD, A.LONGWAKE):
            f += 6 + (28 if d.len else 0)
        elif t == A.MATRIX:
            f += 66 + (28 if d.len else 0)
        elif t == A.APERTURE:
            f += 14 if d.len else 0
    return f
