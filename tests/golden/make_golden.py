"""Generate the committed golden fixtures from the reference Accel+ library itself.

Run in a container where the reference sources exist (oracle/Makefile compiles them into
oracle/_ref/libaccel_ref.so):

    make -C oracle all REF_SRC=<reference>/src/lib/accel && python tests/golden/make_golden.py

Writes, next to this script:
  fodo32.lat   32-cell FODO, sextupoles from the reference's correct_chrom to (1, 1), twice
  dba18.lat    18-cell DBA, RF phase from the reference's setrfphase, chromaticity (1, 1)
  golden.npz   reference outputs on small seeded inputs (every array named below)
The lattices are written with 17 significant digits, so the reference reads them back exactly.
"""
from __future__ import annotations

import importlib
import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

A = importlib.import_module("accel-plus_b200")
LT = importlib.import_module("accel-plus_b200.lattices")
import oracle as O  # noqa: E402


def ref_of(elems):
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    A.write_lattice(path, elems)
    line = O.RefLine(path)
    os.unlink(path)
    return line


def sextupole_index(elems, name):
    return [i for i, d in enumerate(elems) if d.type == A.STRMPOLE and d.name == name][0]


def make_fodo():
    base = LT.fodo32()
    r = ref_of(base)
    r.set_flags(rad=0, cavity=0)
    r.correct_chrom("SF", "SD", 1.0, 1.0)
    cx, cy = r.correct_chrom("SF", "SD", 1.0, 1.0)
    b2f = r.get_poly(sextupole_index(base, "SF"), 2)
    b2d = r.get_poly(sextupole_index(base, "SD"), 2)
    ring = LT.fodo32(b2f, b2d)
    path = os.path.join(HERE, "fodo32.lat")
    A.write_lattice(path, ring)
    chk = O.RefLine(path)
    print(f"fodo32: SF {b2f:.6f} SD {b2d:.6f} chrom ({cx:.6f}, {cy:.6f}) ref-reload chrom {chk.chrom()}")
    return path


DBA_CHROM = 1.0


def make_dba():
    base = LT.dba18()
    r = ref_of(base)
    phis = r.setrfphase()  # leaves cavities off and radiation off, as the reference does
    r.set_flags(rad=0, cavity=0)
    r.correct_chrom("SD", "SF", DBA_CHROM, DBA_CHROM)
    cx, cy = r.correct_chrom("SD", "SF", DBA_CHROM, DBA_CHROM)
    b2d = r.get_poly(sextupole_index(base, "SD"), 2)
    b2f = r.get_poly(sextupole_index(base, "SF"), 2)
    ring = LT.dba18(b2d, b2f, phis=phis)
    path = os.path.join(HERE, "dba18.lat")
    A.write_lattice(path, ring)
    chk = O.RefLine(path)
    chk.set_flags(rad=0, cavity=0)
    print(f"dba18: phis {phis:.9f} SD {b2d:.6f} SF {b2f:.6f} chrom ({cx:.6f},{cy:.6f}) "
          f"tune {chk.tune()} L={LT.ring_length(ring):.9f}")
    return path


def element_cases():
    """Single elements of every supported type, on 16 seeded particles."""
    e = A.elem
    m = np.eye(6)
    m[0, 1] = 1.1
    m[1, 0] = -0.2
    m[2, 3] = 0.7
    m[4, 5] = 0.01
    cases = {
        "drift": [e(A.DRIFT, "D", 1.3)],
        "quad_f": [e(A.QUAD, "Q", 0.4, f=[1.7])],
        "quad_d": [e(A.QUAD, "Q", 0.4, f=[-1.1])],
        "quad_0": [e(A.QUAD, "Q", 0.4, f=[0.0])],
        "bend": [e(A.BEND, "B", 1.2, f=[0.12, 0.03, 0.05, 0.2])],
        "bend_neg": [e(A.BEND, "B", 1.2, f=[0.02, 0.0, 0.0, -0.9])],
        "corrector": [e(A.CORRECTOR, "C", 0.3, f=[1e-4, -2e-4])],
        "matrix": [e(A.MATRIX, "M", 0.5, mat=m.ravel())],
        "aperture": [e(A.APERTURE, "AP", 0.8, f=[-0.003, 0.004, -0.002, 0.0025])],
        "cavity": [e(A.CAVITY, "RF", 0.3, f=[3.2, 476e6, 0.26, 3000])],
        "strm_thick": [e(A.STRMPOLE, "S", 0.3, max_npole=4, poly_b=[1e-4, 1.3, 20.0, -300.0],
                         poly_a=[2e-5, 0.01, 3.0, 0.0])],
        "strm_thin": [e(A.STRMPOLE, "T", 0.0, max_npole=5, poly_b=[0, 0.2, 4.0, 50.0, 600.0],
                        poly_a=[0, 0.05, 1.0, 0, 10.0])],
        "bendm": [e(A.BENDMPOLE, "BM", 1.1, f=[0.1, 0.02, 0.04, 3000], max_npole=3, poly_b=[0, 0.3, 5.0])],
        "bendm_rad": [e(A.BENDMPOLE, "BM", 1.1, f=[0.1, 0.02, 0.04, 3000], max_npole=3,
                        poly_b=[0, 0.3, 5.0], flags=1)],
        "syncrad_damp": [e(A.SYNCRAD, "SR", 0.2, f=[3000, 0.9, 1.3, 1.0, 2e-9, 2e-11, 1e-3, 5.0, 3.0], flags=1)],
        "transwake": [e(A.TRANSWAKE, "TW", 0.0, f=[3000, 2.0, 50.0, 10.0, 1.5, 40.0, 12.0, 2.0], flags=1)],
    }
    return cases


def element_particles(n=16, seed=7):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 6))
    r[:, 0] = rng.normal(0, 2e-3, n)
    r[:, 1] = rng.normal(0, 2e-4, n)
    r[:, 2] = rng.normal(0, 1e-3, n)
    r[:, 3] = rng.normal(0, 1e-4, n)
    r[:, 4] = rng.normal(0, 3e-3, n)
    r[:, 5] = rng.normal(0, 1e-3, n)
    return r


def main():
    O.ref().ref_set_threads(1)
    out = {}
    fodo = make_fodo()
    dba = make_dba()

    # elements
    r0 = element_particles()
    out["elem_in"] = r0
    for name, elems in element_cases().items():
        line = ref_of(elems)
        if name == "cavity":
            line.set_flags(cavity=1)
        if name == "bendm_rad":
            line.set_flags(rad=1)
        if name == "transwake":
            line.set_flags(wake=1)
        if name == "syncrad_damp":
            line.set_flags(rad=A.RAD_LUMP_DAMP)
        r = r0.copy()
        line.track(r, 1)
        out[f"elem_{name}"] = r

    # the 32-cell FODO: 64 of its 1,024 uniform particles, 1 and 100 turns; one-turn matrix
    rf = O.RefLine(fodo)
    p = LT.fodo_particles()[:64].copy()
    out["fodo_in"] = p.copy()
    r1 = p.copy()
    rf.track(r1, 1)
    out["fodo_t1"] = r1
    r100 = p.copy()
    rf.track(r100, 100)
    out["fodo_t100"] = r100
    out["fodo_m66"] = rf.m66()
    out["fodo_tune"] = np.array(rf.tune())
    out["fodo_chrom"] = np.array(rf.chrom())

    # the 18-cell DBA, radiation + cavity on, a coarse DA grid with loss turns over 200 turns
    rd = O.RefLine(dba)
    rd.set_flags(rad=0, cavity=0)
    out["dba_m66"] = rd.m66()
    out["dba_tune"] = np.array(rd.tune())
    out["dba_chrom"] = np.array(rd.chrom())
    rd.set_flags(rad=1, cavity=1)
    g = LT.da_grid(13, 7)
    out["dba_grid_in"] = g.copy()
    rg = g.copy()
    out["dba_grid_loss"] = rd.track_loss(rg, 200)
    out["dba_grid_out"] = rg
    out["dba_m66_rad"] = rd.m66()
    rp = O.RefLine(dba)
    out["dba_phis"] = np.array([rp.setrfphase()])  # on the committed (sextupole-corrected) ring

    # two error-seeded copies of the DBA (feed-down), small grids, 100 turns
    base = LT.dba_ring()
    for k in (0, 1):
        ring = LT.error_copy(base, k)
        rr = ref_of(ring)
        rr.set_flags(rad=1, cavity=1)
        gk = LT.da_grid(9, 5)
        out[f"c3_{k}_in"] = gk.copy()
        rk = gk.copy()
        out[f"c3_{k}_loss"] = rr.track_loss(rk, 100)
        out[f"c3_{k}_out"] = rk

    # reference trackDA on the DBA (rays x steps, area)
    rd2 = O.RefLine(dba)
    rd2.set_flags(rad=1, cavity=1)
    area, rx, ry = rd2.trackDA(0.03, 0.002, 0.012, 100, 7, 8)
    out["da_area"] = np.array([area])
    out["da_rx"] = rx
    out["da_ry"] = ry

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
