"""The C-ABI library on the host: it loads, exports every entry point the header declares, reads
and writes the reference's lattice format, and reports errors by status without a GPU."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT


def test_library_exports_every_declared_symbol(A):
    lib = A.lib()
    declared = A.exported_symbols()
    assert len(declared) >= 35
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings(A):
    for s in (A.OK, A.E_INVALID, A.E_UNSUPPORTED, A.E_CUDA, A.E_NOMEM, A.E_IO, A.E_TIMEOUT,
              A.E_NODEVICE, A.E_TOO_LARGE):
        assert A.status_string(s) and A.status_string(s) != "unknown status"


def test_lattice_roundtrip_bit_exact(A, LT, tmp_path):
    for ring in (LT.fodo_ring(), LT.dba_ring()):
        p = str(tmp_path / "x.lat")
        A.write_lattice(p, ring)
        back = A.read_lattice(p)
        assert len(back) == len(ring)
        for a, b in zip(ring, back):
            # the file carries no run-time switches (radiation, cavity on/off), only parameters
            assert (a.type, a.nslice, a.max_npole, a.len, a.name) == (b.type, b.nslice, b.max_npole, b.len, b.name)
            for f in ("f", "poly_a", "poly_b", "mat"):
                assert bytes(getattr(a, f)) == bytes(getattr(b, f)), (a.name, f)


def test_lattice_reader_grammar(A):
    text = """
    ! a comment line
    QF1  : StrMPole 0.25 3
        0 1.2 0
        0 0 0
    D1 :  Drift 2.0
    B1:   BendMPole 1.0 0.1 0.01 0.02 2
        0.0 0.5
    RF :  Cavity 0 3.2 476e6 0.26 3000
    AP :  Aperture 0 -0.05 0.05 -0.04 0.04
    M  : Matrix 0
      1 0 0 0 0 0
      0 1 0 0 0 0
      0 0 1 0 0 0
      0 0 0 1 0 0
      0 0 0 0 1 0
      0 0 0 0 0 1
    MON : Monitor 0 0 -2
    RETURN
    X : Drift 9
    """
    e = A.parse_lattice(text)
    assert [d.type_name for d in e] == ["StrMPole", "Drift", "BendMPole", "Cavity", "Aperture", "Matrix", "Monitor"]
    assert e[0].max_npole == 3 and e[0].poly_b[1] == 1.2 and e[0].nslice == 10
    assert e[2].f[0] == 0.1 and e[2].f[4] == 0.1 / 1.0 and e[2].poly_b[1] == 0.5 and e[2].f[3] == 3000
    assert e[3].flags == 1  # a Cavity is constructed on; the Lattice block switches it off
    assert list(e[4].f[:4]) == [-0.05, 0.05, -0.04, 0.04]
    assert e[6].f[0] == 1 and e[6].f[1] == 0.1  # interval clamped to 1, ratio < 0 -> 0.1


def test_lattice_reader_errors(A):
    with pytest.raises(A.AccelError) as ei:
        A.parse_lattice("Q : Quadrupole 0.3 1.0\n")
    assert ei.value.status == A.E_IO
    with pytest.raises(A.AccelError) as ei:
        A.parse_lattice("B : BendMPole 1.0 0.1 0 0 11\n 1 2 3\n")
    assert ei.value.status == A.E_IO
    with pytest.raises(A.AccelError) as ei:
        A.read_lattice("/nonexistent/lattice.lat")
    assert ei.value.status == A.E_IO


def test_wigtable_registry_and_lattice_format(A, tmp_path):
    """WigTable kick tables: registered, read back, written in the reference's layout (sizes, xl,
    yl, xkick rows, a blank line, ykick rows; accel.cpp:1247-1270) and parsed again bit-exactly."""
    xl = np.linspace(-0.02, 0.02, 5)
    yl = np.array([0.01, 0.0, -0.01])          # descending is allowed
    xk = np.arange(15.0).reshape(3, 5) * 1e-5 + 1.0 / 3.0
    yk = -np.arange(15.0).reshape(3, 5) * 1e-6
    tid = A.wigtable(xl, yl, xk, yk)
    got = A.wigtable_get(tid)
    for a, b in zip(got, (xl, yl, xk, yk)):
        assert np.array_equal(a, b)
    ring = [A.elem(A.DRIFT, "D", 1.0), A.elem(A.WIGTABLE, "WT", 1.5, nslice=4, f=[tid]),
            A.elem(A.DRIFT, "D", 0.5)]
    p = str(tmp_path / "w.lat")
    A.write_lattice(p, ring)
    lines = open(p).read().splitlines()
    assert lines[1].split() == ["WT", ":", "WigTable", "1.5", "4", "5", "3"]
    assert len(lines) == 1 + 1 + 2 + 3 + 1 + 3 + 1 and lines[7].strip() == ""
    back = A.read_lattice(p)
    assert [d.type for d in back] == [A.DRIFT, A.WIGTABLE, A.DRIFT] and back[2].len == 0.5
    assert back[1].nslice == 4 and back[1].len == 1.5 and int(back[1].f[0]) != tid
    for a, b in zip(A.wigtable_get(int(back[1].f[0])), (xl, yl, xk, yk)):
        assert np.array_equal(a, b)
    A.wigtable_destroy(tid)
    with pytest.raises(A.AccelError) as ei:
        A.wigtable_get(tid)
    assert ei.value.status == A.E_INVALID


def test_wigtable_rejects_bad_tables(A):
    ok_x, ok_y = np.linspace(-1, 1, 4), np.linspace(-1, 1, 3)
    z = np.zeros((3, 4))
    for xl, yl, zz in ((np.array([0.0]), ok_y, np.zeros((3, 1))),          # one grid point
                       (np.linspace(-1, 1, 102), ok_y, np.zeros((3, 102))),  # above MAX_WIGTAB_X
                       (ok_x, np.linspace(-1, 1, 22), np.zeros((22, 4))),    # above MAX_WIGTAB_Y
                       (np.array([0.0, 1.0, 1.0, 2.0]), ok_y, z),            # repeated point
                       (np.array([0.0, 2.0, 1.0, 3.0]), ok_y, z)):           # not monotonic
        with pytest.raises(A.AccelError) as ei:
            A.wigtable(xl, yl, zz, zz)
        assert ei.value.status == A.E_INVALID
    with pytest.raises(A.AccelError) as ei:   # a table that ends early
        A.parse_lattice("WT : WigTable 1.0 2 3 2\n 0 1 2\n 0 1\n 1 2 3\n 4 5 6\n\n 1 2 3\n")
    assert ei.value.status == A.E_IO


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference library not built here")
def test_reader_agrees_with_reference_deserialize(A, O, LT):
    """Every element's fields as the reference's own deserialize+getfield see them."""
    path = os.path.join(LT.GOLDEN_DIR, "dba18.lat")
    mine = A.read_lattice(path)
    ref = O.RefLine(path)
    assert len(ref) == len(mine)
    for i, d in enumerate(mine):
        assert ref.get_field(i, "Length") == d.len
        if d.type == A.STRMPOLE:
            for n in range(d.max_npole):
                assert ref.get_poly(i, n) == d.poly_b[n]
                assert ref.get_poly(i, n, skew=True) == d.poly_a[n]
        if d.type == A.CAVITY:
            assert ref.get_field(i, "Voltage") == d.f[0]
            assert ref.get_field(i, "Frequency") == d.f[1]
            assert ref.get_field(i, "Phis") == d.f[2]


def test_state_checkpoint_roundtrip(A, tmp_path):
    """Particle states survive a checkpoint bit for bit (lost particles' NaN and codes included),
    with and without loss turns; a foreign or truncated file is an I/O error."""
    rng = np.random.default_rng(5)
    r = rng.normal(0, 1e-3, (1000, 6))
    r[7, 0], r[7, 4] = np.nan, 3.0
    lt = rng.integers(-1, 500, 1000).astype(np.int32)
    p = str(tmp_path / "s.bin")
    A.write_state(p, r, turn=1234, loss=lt)
    r2, t2, l2 = A.read_state(p)
    assert t2 == 1234 and np.array_equal(r2.view(np.int64), r.view(np.int64)) and np.array_equal(l2, lt)
    A.write_state(p, r[:3])
    r3, t3, l3 = A.read_state(p)
    assert t3 == 0 and l3 is None and np.array_equal(r3, r[:3])
    with open(p, "r+b") as f:
        f.truncate(40)
    with pytest.raises(A.AccelError) as ei:
        A.read_state(p)
    assert ei.value.status == A.E_IO
    # a header whose particle count disagrees with the file's length (here one that would overflow
    # the byte count) is refused before anything is allocated
    A.write_state(p, r[:3])
    with open(p, "r+b") as f:
        f.seek(16)
        f.write(np.int64(2**61).tobytes())
    with pytest.raises(A.AccelError) as ei:
        A.read_state(p)
    assert ei.value.status == A.E_IO
    q = str(tmp_path / "x.txt")
    open(q, "w").write("not a state file, just text, long enough for a header\n")
    with pytest.raises(A.AccelError) as ei:
        A.read_state(q)
    assert ei.value.status == A.E_IO


def test_device_memory_limit_without_a_device(A):
    """The budget is host state: it can be set and read with no device (nothing is held)."""
    assert A.device_memory_held() >= 0
    A.set_device_memory_limit(1 << 20)
    A.set_device_memory_limit(None)
    with pytest.raises(A.AccelError) as ei:
        A._check(A.lib().accel_device_memory_held(None), "accel_device_memory_held")
    assert ei.value.status == A.E_INVALID


def test_no_device_is_an_error_not_a_fallback(A):
    if A.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(A.AccelError) as ei:
        A.Context(0)
    assert ei.value.status == A.E_NODEVICE


def test_model_flops_match_cost_formula(A, LT):
    """The flop model (StrMPole slice 52 + 3(8m + 4), BendMPole slice 4*46 + 3(44 + 7m), drift
    14) on the 32-cell FODO: 32 x [2 quads (m=1) + 2 sextupoles (m=2) + 2 bends (m=0) + 4 drifts]."""
    ring = LT.fodo_ring()
    per_cell = 2 * 10 * (52 + 3 * 12) + 2 * 10 * (52 + 3 * 20) + 2 * (10 * (184 + 3 * 44) + 8) + 4 * 14
    assert LT.flops_per_turn(ring) == 32 * per_cell


def test_nccl_unique_id_without_a_gpu(A):
    """The communicator id is made on the host (NCCL is loaded at run time); ids differ."""
    a, b = A.nccl_unique_id(), A.nccl_unique_id()
    assert len(a) == len(b) == 128 and a != b and any(a)
