"""The CPU oracle, pinned: the C restatement (oracle/liboracle.so) must reproduce the reference
library's own outputs bit for bit — the committed golden vectors everywhere, and the live
reference library (oracle/_ref) where it was built."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, same_bits


def _flags(O, A, name, elems):
    if name == "cavity":
        O.port_set_flags(elems, cavity=1)
    if name == "bendm_rad":
        O.port_set_flags(elems, rad=1)
    if name == "transwake":
        O.port_set_flags(elems, wake=1)
    if name == "syncrad_damp":
        O.port_set_flags(elems, rad=A.RAD_LUMP_DAMP)


def test_port_elements_match_golden(A, O, G, MG):
    for name, elems in MG.element_cases().items():
        _flags(O, A, name, elems)
        r = G["elem_in"].copy()
        O.port_track(elems, r, 1, loss=False)
        assert same_bits(r, G[f"elem_{name}"]), name


def test_port_fodo_matches_golden(O, G, LT):
    ring = LT.fodo_ring()
    for turns, key in ((1, "fodo_t1"), (100, "fodo_t100")):
        r = G["fodo_in"].copy()
        O.port_track(ring, r, turns, loss=False)
        assert same_bits(r, G[key])
    assert same_bits(O.port_m66(ring), G["fodo_m66"])


def test_port_openmp_blocks_bit_identical(O, G, LT):
    """ALine::pass splits particles into per-thread blocks; results do not depend on it."""
    ring = LT.fodo_ring()
    r1 = G["fodo_in"].copy()
    r8 = G["fodo_in"].copy()
    O.port_track(ring, r1, 20, loss=False, nthreads=1)
    O.port_track(ring, r8, 20, loss=False, nthreads=8)
    assert same_bits(r1, r8)


def test_port_dba_loss_turns_match_golden(O, G, LT):
    ring = LT.dba_ring()
    r = G["dba_grid_in"].copy()
    lt = O.port_track(ring, r, 200)
    assert np.array_equal(lt, G["dba_grid_loss"])
    assert same_bits(r, G["dba_grid_out"])
    assert 0 < (lt >= 0).sum() < lt.size  # the grid straddles the aperture


def test_port_error_copies_match_golden(O, G, LT):
    base = LT.dba_ring()
    for k in (0, 1):
        ring = LT.error_copy(base, k)
        r = G[f"c3_{k}_in"].copy()
        lt = O.port_track(ring, r, 100)
        assert np.array_equal(lt, G[f"c3_{k}_loss"])
        assert same_bits(r, G[f"c3_{k}_out"])


def test_port_m66_dba(O, G, LT):
    ring = LT.dba_ring()
    O.port_set_flags(ring, rad=0, cavity=0)
    assert same_bits(O.port_m66(ring), G["dba_m66"])
    O.port_set_flags(ring, rad=1, cavity=1)
    assert same_bits(O.port_m66(ring), G["dba_m66_rad"])


def test_golden_lattice_properties(G):
    """The committed rings are what their builders claim: chromaticity (1, 1) from the
    reference's correct_chrom, stable tunes, a stable synchrotron motion (M56 < 0)."""
    assert np.allclose(G["fodo_chrom"], [1, 1], atol=1e-3)
    assert np.allclose(G["dba_chrom"], [1, 1], atol=2e-3)
    for key in ("fodo_m66", "dba_m66"):
        m = G[key]
        assert abs(m[0, 0] + m[1, 1]) < 2 and abs(m[2, 2] + m[3, 3]) < 2
    assert G["dba_m66"][4, 5] < 0
    ev = np.abs(np.linalg.eigvals(G["dba_m66_rad"]))
    assert np.all(ev < 1.0 + 1e-6)  # radiation damping: no growing mode


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference library not built here")
class TestAgainstLiveReference:
    def test_random_strmpole_and_bends(self, A, O, LT):
        rng = np.random.default_rng(3)
        for trial in range(5):
            elems = [
                A.elem(A.STRMPOLE, "S", 0.1 + rng.random(), max_npole=6, nslice=int(rng.integers(1, 12)),
                       poly_b=rng.normal(0, [1e-4, 1, 10, 100, 1e3, 1e4]),
                       poly_a=rng.normal(0, [1e-4, 0.1, 1, 10, 100, 1e3])),
                A.elem(A.DRIFT, "D", rng.random()),
                A.elem(A.BENDMPOLE, "B", 0.5 + rng.random(), f=[rng.normal(0, 0.2), 0.01, -0.02, 2500],
                       max_npole=3, nslice=int(rng.integers(1, 12)), poly_b=[0, rng.normal(0, 0.5), rng.normal(0, 5)]),
            ]
            r0 = rng.normal(0, [2e-3, 2e-4, 1e-3, 1e-4, 3e-3, 1e-3], size=(32, 6))
            path = "/tmp/_orc_rand.lat"
            A.write_lattice(path, elems)
            ref = O.RefLine(path)
            r_ref = r0.copy()
            ref.track(r_ref, 3)
            r_port = r0.copy()
            O.port_track(A.read_lattice(path), r_port, 3, loss=False)
            assert same_bits(r_port, r_ref), trial

    def test_setrfphase_and_trackDA_consistent(self, O, G, LT):
        path = f"{LT.GOLDEN_DIR}/dba18.lat"
        ref = O.RefLine(path)
        ref.set_flags(rad=1, cavity=1)
        area, rx, ry = ref.trackDA(0.03, 0.002, 0.012, 100, 7, 8)
        assert area == G["da_area"][0]
        assert same_bits(rx, G["da_rx"]) and same_bits(ry, G["da_ry"])


def test_longwake_oracle_self_consistent(A, O):
    """The new longitudinal wake: a point bunch (one bin) receives W(0)/2 q per unit charge, and
    trailing bins see the resonator wake; checked against the formula directly."""
    import ctypes as C
    nb = 8
    counts = np.zeros(nb)
    counts[5] = 1000.0
    V = np.zeros(nb)
    dz = 1e-3
    qper = 1e-9 / 1000
    O.port().orc_longwake_voltage(nb, dz, counts.ctypes.data, qper, 1e3, 10e9, 1.0, V.ctypes.data)
    wr = 2 * np.pi * 10e9
    amp = wr * 1e3 / 1.0
    assert np.isclose(V[5], 0.5 * amp * 1e-9)
    a = wr / 2
    wb = np.sqrt(wr * wr - a * a)
    tau = 2 * dz / 2.99792458e8
    w = amp * np.exp(-a * tau) * (np.cos(wb * tau) - a / wb * np.sin(wb * tau))
    assert np.isclose(V[3], w * 1e-9, rtol=1e-12)
    assert np.all(V[6:] == 0)


def test_naff_matches_reference(A):
    """The host NAFF against the reference's naff on synthetic lines (with a second harmonic and
    noise) and on FODO turn-by-turn records: the same frequency to well inside the golden-section
    tolerance (3e-8 relative)."""
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "naff.npz"))
    for x, lo, hi, nu in zip(g["records"], g["xlow"], g["xhi"], g["nu"]):
        assert abs(A.naff(x, lo, hi) - nu) <= 1e-8 * abs(nu), (A.naff(x, lo, hi), nu)


def test_port_reproduces_full_size_fixture_subset(O, LT):
    """The reference outputs committed for the full-size parity tests (config_golden.npz, made by
    the reference library) against the C restatement on a subset of the same particles: the
    FODO's first 256 particles and the whole grid of the smallest error-seeded DBA copy (24 x 11,
    radiation and cavity on), 1,000 turns each: loss turns equal and final coordinates bit for
    bit."""
    cg = np.load(os.path.join(GOLDEN, "config_golden.npz"))
    threads = os.cpu_count() or 1
    r = LT.fodo_particles()[:256].copy()
    lt = O.port_track(LT.fodo_ring(), r, 1000, nthreads=threads)
    assert np.array_equal(lt, cg["c1_loss"][:256])
    assert same_bits(r, cg["c1_out"][:256])
    k = int(cg["c3_copies"][0])
    nx, ny = (int(v) for v in cg[f"c3_{k}_shape"])
    assert nx * ny == 264
    r = LT.da_grid(nx, ny)
    lt = O.port_track(LT.error_copy(LT.dba_ring(), k), r, 1000, nthreads=threads)
    assert np.array_equal(lt, cg[f"c3_{k}_loss"])
    assert same_bits(r, cg[f"c3_{k}_out"])
