"""Host-side checks of the benchmark's reference arm (no GPU).

The reference arm times the reference's own CPU tracking on a sample of the batched DA workload.
Its copies' lattice files are written in pure Python (lattices.error_copy_text), so the process
that runs the reference maps no library of the engine: the text must equal the engine's own
lattice writer's output for the same copy, character for character, and a short run of the arm
must report the engine library unmapped.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import pytest

from conftest import ROOT


@pytest.mark.parametrize("seed", [0, 5, 131, 255])
def test_error_copy_text_equals_library_writer(A, LT, seed):
    fd, path = tempfile.mkstemp(suffix=".lat")
    os.close(fd)
    try:
        A.write_lattice(path, LT.error_copy(LT.dba_ring(), seed))
        with open(path) as f:
            want = f.read()
    finally:
        os.unlink(path)
    assert LT.error_copy_text(seed) == want


def test_reference_arm_maps_no_engine_library(O):
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--copies", "16", "--turns", "20",
                          "--ref-seconds", "0.5"], capture_output=True, text=True, timeout=600,
                         env={**os.environ, "OMP_NUM_THREADS": "2"})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["cpu_baseline"]["kind"] == "reference"
    assert "extrapolated" in line["cpu_baseline"]["sample"]
    assert line["process_maps_engine_library"] is False
    assert line["native_so_loaded"] == ["oracle/_ref/libaccel_ref.so"]
    assert line["value"] > 0


def test_nudge_growth_and_tangent_picks():
    """The full-size gradient check's helpers: the growth of a 1e-12 nudge relative to each
    coordinate's RMS (inf for a particle lost in either run), and the particles the forward-mode
    check takes (the most sensitive with growth up to 1e4, and quiet ones drawn with a seed)."""
    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(0)
    base = rng.normal(size=(200, 6))
    nudged = base.copy()
    nudged[:, 0] += 1e-12 * np.sqrt(np.mean(base[:, 0] ** 2)) * np.arange(200)
    nudged[7, 0] = np.nan
    g = bench.nudge_growth(base, nudged)
    assert np.isinf(g[7])
    assert np.allclose(g[[0, 1, 50]], [0.0, 1.0, 50.0], atol=1e-3)
    growth = np.concatenate([np.linspace(0, 20, 100), [5e3, 2e4, 9e3, 3e3, 1e5, np.inf]])
    pick = bench.tangent_picks(growth, 2, 3, seed=1)
    assert list(pick[-2:]) == [100, 102]            # 5e3 and 9e3: the largest up to 1e4
    quiet = [p for p in pick if p < 100]
    assert len(quiet) == 3 and all(growth[p] <= 10 for p in quiet)
    assert np.array_equal(pick, bench.tangent_picks(growth, 2, 3, seed=1))
