"""bench.py's multi-rank plumbing on CPU: two `gloo` ranks, as torchrun would start them.

Covers what the GPU run relies on without a second GPU: the max / sum reductions that turn
per-rank timings and particle counts into the job's numbers, the all-reduce of the adjoint's knob
gradients, the barrier, the per-rank workload
shards (different error seeds and grid sizes on each rank, identical on a re-run), and the
reference arm, which only rank 0 runs.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import io, json, os, sys, contextlib, types
sys.path.insert(0, os.environ["ROOT"])
import numpy as np
import bench
r = bench.Ranks("gloo", timeout_s=60)
out = {"rank": r.rank, "world": r.world}
out["max"] = r.max(float(r.rank + 1))
out["sum"] = r.sum(10.0 * (r.rank + 1))
out["sum_array"] = r.sum_array(np.arange(4.0) * (r.rank + 1)).tolist()
r.barrier()
rings, off, aos, sizes = bench.workload(4, r.rank)
rings2, off2, aos2, sizes2 = bench.workload(4, r.rank)
out["sizes"] = [list(map(int, s)) for s in sizes]
out["repeat_identical"] = bool(np.array_equal(aos, aos2) and np.array_equal(off, off2))
out["k1"] = float(rings[0][[i for i, d in enumerate(rings[0]) if d.poly_b[1] != 0][0]].poly_b[1])
out["particles"] = int(off[-1])
out["total"] = r.sum(float(off[-1]))
buf = io.StringIO()
if r.rank != 0:
    with contextlib.redirect_stdout(buf):
        bench.reference_arm(types.SimpleNamespace(copies=4, warmup=3, steps=1, gpus=r.world, turns=10))
out["ref_arm_output"] = buf.getvalue()
r.barrier()
r.close()
print("RESULT " + json.dumps(out))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    pytest.importorskip("torch")
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, ROOT=ROOT, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-3000:]
        line = [l for l in out.splitlines() if l.startswith("RESULT ")][-1]
        res.append(json.loads(line[7:]))
    r0, r1 = sorted(res, key=lambda d: d["rank"])
    for r in (r0, r1):
        assert r["world"] == 2 and r["max"] == 2.0 and r["sum"] == 30.0
        assert r["sum_array"] == [0.0, 3.0, 6.0, 9.0]
        assert r["repeat_identical"]
        assert r["total"] == r0["particles"] + r1["particles"]
    assert r0["sizes"] != r1["sizes"]          # each rank draws its own grids ...
    assert r0["k1"] != r1["k1"]                # ... and its own error seeds
    assert r1["ref_arm_output"] == ""          # only rank 0 runs and prints the reference arm
