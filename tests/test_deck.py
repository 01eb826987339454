"""The input-deck interpreter `accel+gpu` against the reference's own `accel+` on the same decks.

The reference's outputs are committed fixtures (tests/golden/<deck>.ref.out, written by
make_deck_golden.py).  Both programs print with six significant digits, so the comparison is line by
line: the words must be identical and every number equal within 2e-5 relative (1e-12 absolute for
values that are round-off around zero).  Dynamic- and momentum-aperture boundaries are decided by a
lost / survived verdict that may flip for a particle on the chaotic edge; there a ray radius may
differ by one scan step and the area by the one triangle it changes.
"""
from __future__ import annotations

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "accel-plus_b200", "accel+gpu")
GOLDEN = os.path.join(ROOT, "tests", "golden")
DECKS = os.path.join(ROOT, "tests", "decks")
NUM = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?")


def run_deck(name, *flags):
    out = subprocess.run([EXE, os.path.join(DECKS, name + ".in"), *flags], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if not l.startswith("#UTC")]


def split(line):
    nums = [float(m) for m in NUM.findall(line)]
    return NUM.sub("#", line).split(), nums


def close(a, b, rel=2e-5, abs_=1e-12):
    return abs(a - b) <= max(rel * max(abs(a), abs(b)), abs_)


def compare(mine, ref):
    assert len(mine) == len(ref), "\n".join(mine[-20:])
    block, step = None, None
    for lm, lr in zip(mine, ref):
        wm, nm = split(lm)
        wr, nr = split(lr)
        assert wm == wr and len(nm) == len(nr), (lm, lr)
        if lr.startswith("$$$") or lr.startswith("*****"):
            block = lr
        if lr.startswith("#") and len(nr) == 7:  # track_DA: xmin xmax ymax nray nstep nturn neg
            step = ("da", (nr[1] - nr[0]) / (nr[4] - 1))
        if lr.startswith("#") and len(nr) == 5:  # track_MA: nmoni nstep nturn dppmin dppmax
            step = ("ma", (nr[4] - nr[3]) / nr[1])
        if all(close(a, b) for a, b in zip(nm, nr)):
            continue
        if block and block.startswith("$$$DA-profile") and step and step[0] == "da":
            if lr.startswith("$$$DA"):
                assert close(nm[-1], nr[-1], rel=0.05), (lm, lr)
            else:
                rm, rr = (nm[0] ** 2 + nm[1] ** 2) ** 0.5, (nr[0] ** 2 + nr[1] ** 2) ** 0.5
                assert abs(rm - rr) <= 1.01 * step[1], (lm, lr)
            continue
        if block and block.startswith("$$$MA") and step and step[0] == "ma":
            if lr.startswith("$$$MA"):
                assert close(nm[-1], nr[-1], rel=0.2), (lm, lr)
            else:
                assert all(abs(a - b) <= 1.01 * step[1] for a, b in zip(nm, nr)), (lm, lr)
            continue
        raise AssertionError(f"numbers differ:\n mine: {lm}\n ref:  {lr}")


@pytest.mark.gpu
@pytest.mark.parametrize("deck", ["dba_deck", "fodo_deck", "ops_deck", "dist_deck"])
def test_deck_matches_reference(deck):
    with open(os.path.join(GOLDEN, deck + ".ref.out")) as f:
        ref = [l for l in f.read().splitlines() if not l.startswith("#UTC")]
    compare(run_deck(deck), ref)


@pytest.mark.gpu
def test_deck_in_exact_mode_matches_reference():
    """The DBA deck (optics, DA and MA scans, tracking) with --exact: the reference's operation
    order throughout, against the reference's own output."""
    with open(os.path.join(GOLDEN, "dba_deck.ref.out")) as f:
        ref = [l for l in f.read().splitlines() if not l.startswith("#UTC")]
    compare(run_deck("dba_deck", "--exact"), ref)


@pytest.mark.gpu
def test_exact_corrections_reach_their_targets():
    """correct_tune / correct_chrom with EXACT (an extension of the reference's commands): Newton
    iterations on tunes and chromaticities from exact one-turn tangent maps land on the targets
    to the printed six digits, where the reference's fit (one step of a difference-based
    response) leaves a residual; the following print_tune shows the corrected tunes."""
    out = run_deck("engine_only/correct_exact")  # no reference output: EXACT is this engine's
    tunes = [l for l in out if l.startswith("corrected tunes:")]
    chrom = [l for l in out if l.startswith("corrected chromaticities:")]
    assert len(tunes) == 1 and len(chrom) == 1
    t = [float(x) for x in NUM.findall(tunes[0])]
    c = [float(x) for x in NUM.findall(chrom[0])]
    assert abs(t[0] - 0.19) < 2e-6 and abs(t[1] - 0.36) < 2e-6, tunes
    assert abs(c[0] - 1.0) < 2e-5 and abs(c[1] - 1.5) < 2e-5, chrom
    printed = [l for l in out if l.startswith("Tunes:")][-1]
    p = [float(x) for x in NUM.findall(printed)]
    assert abs(p[0] - 0.19) < 2e-5 and abs(p[1] - 0.36) < 2e-5, printed


@pytest.mark.gpu
def test_deck_resumes_bit_for_bit_from_a_binary_checkpoint(tmp_path):
    """Do_Track save=FILE then "Distribution : Load FILE, format=binary" (extensions of the
    reference's decks, whose text export keeps six digits): 40 + 60 turns through the checkpoint
    print the same final coordinates as 100 turns in one go."""
    ckpt = str(tmp_path / "state.bin")
    head = ("Lattice\n  file_name = tests/golden/dba18.lat, type=ERING\nEnd\nTrack\n"
            "  Distribution = Coordinate r=(1e-3, 0, 5e-4, 0, 0, 0; 2e-3, 1e-5, 1e-3, 0, 0, 1e-3; "
            "-3e-3, 2e-5, 2e-4, 0, 1e-3, -5e-4)\n")
    one = head + "  Do_Track: radiation=rad, rfcavity=on, nturn=100, printfinal=Full\nEnd\nSTOP\n"
    two = (head + f"  Do_Track: radiation=rad, rfcavity=on, nturn=40, save={ckpt}\nEnd\nTrack\n"
           f"  Distribution : Load {ckpt}, format=binary\n"
           "  Do_Track: radiation=rad, rfcavity=on, nturn=60, printfinal=Full\nEnd\nSTOP\n")
    outs = []
    for name, text in (("one", one), ("two", two)):
        deck = tmp_path / f"{name}.in"
        deck.write_text(text)
        out = subprocess.run([EXE, str(deck)], cwd=ROOT, capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        lines = out.stdout.splitlines()
        k = max(i for i, l in enumerate(lines) if l.startswith("$$$Track-Data: Full export"))
        outs.append([l.split("\t", 1)[1] for l in lines[k + 2:k + 5]])  # the coordinates, turn column dropped
    assert outs[0] == outs[1]


def test_deck_compare_accepts_reference_against_itself():
    """The comparison's own logic, on the golden outputs alone (no GPU)."""
    for deck in ("dba_deck", "fodo_deck", "ops_deck", "dist_deck"):
        with open(os.path.join(GOLDEN, deck + ".ref.out")) as f:
            ref = f.read().splitlines()
        compare(ref, ref)
        bent = list(ref)
        i = next(k for k, l in enumerate(bent) if any(float(x) != 0 for x in NUM.findall(l)))
        x = next(m for m in NUM.finditer(bent[i]) if float(m.group()) != 0)
        bent[i] = bent[i][:x.start()] + repr(1.001 * float(x.group())) + bent[i][x.end():]
        with pytest.raises(AssertionError):
            compare(bent, ref)


def test_deck_without_device_fails_loudly():
    """With no CUDA device the executable exits non-zero with the reason, and runs nothing."""
    import ctypes
    try:
        n = ctypes.c_int(0)
        ok = ctypes.CDLL("libcuda.so.1").cuInit(0) == 0 and ctypes.CDLL("libcuda.so.1").cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        ok = False
    if ok:
        pytest.skip("a CUDA device is present")
    out = subprocess.run([EXE, os.path.join(DECKS, "fodo_deck.in")], cwd=ROOT, capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 2
    assert "accel+gpu:" in out.stderr
