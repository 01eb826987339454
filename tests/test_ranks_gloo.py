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


WAKE_CHILD = r"""
import json, os, sys, importlib
from datetime import timedelta
sys.path.insert(0, os.environ["ROOT"])
sys.path.insert(0, os.path.join(os.environ["ROOT"], "oracle"))
import numpy as np
import torch
import torch.distributed as dist
import oracle as O
LT = importlib.import_module("accel-plus_b200.lattices")

dist.init_process_group("gloo", timeout=timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
el = LT.longwake_elem(energy_mev=3000.0, charge_nc=2.0, rs=1e3, fr=10e9, q=1.0, nbins=256)
E, charge, Rs, fr, Q, nbins = (el.f[k] for k in range(6))
nbins = int(min(max(nbins, 1), 4096))


def staged_wake(mine):
    # the engine's exchange for a bunch spread over ranks: local z range and live count, their
    # min / max / sum over ranks, the bin geometry from those, local bin counts, their sum over
    # ranks, then the oracle's wake voltage (orc_longwake_voltage) and the kick of local particles
    live = ~np.isnan(mine[:, 0])
    z = mine[live, 4]
    zmin = torch.tensor([z.min() if len(z) else np.inf], dtype=torch.float64)
    zmax = torch.tensor([z.max() if len(z) else -np.inf], dtype=torch.float64)
    n = torch.tensor([int(live.sum())], dtype=torch.int64)
    dist.all_reduce(zmin, op=dist.ReduceOp.MIN)
    dist.all_reduce(zmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    zmin, zmax, nlive = float(zmin.item()), float(zmax.item()), int(n.item())
    if nlive == 0:
        return mine
    dz = (zmax - zmin) / nbins
    if not dz > 0:
        dz = 1e-12
    inv_dz = 1.0 / dz
    b = np.clip(((z - zmin) * inv_dz).astype(np.int64), 0, nbins - 1)
    counts = torch.tensor(np.bincount(b, minlength=nbins), dtype=torch.int64)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM)
    qper = charge * 1e-9 / nlive
    V = np.zeros(nbins)
    c = np.ascontiguousarray(counts.numpy().astype(np.float64))
    O.port().orc_longwake_voltage(nbins, dz, c.ctypes.data, qper, Rs, fr, Q, V.ctypes.data)
    inv_e = 1.0 / (E * 1e6)
    out = mine.copy()
    out[np.nonzero(live)[0], 5] = mine[live, 5] - V[b] * inv_e
    return out


rng = np.random.default_rng(17)
N = 20011
r = np.zeros((N, 6))
r[:, 0] = rng.normal(0, 1e-4, N)
r[:, 4] = rng.normal(0, 3e-3, N)
r[:, 5] = rng.normal(0, 1e-3, N)
r[::97, 0] = np.nan          # lost before the wake: skipped
r[5, 4] = r[6, 4]            # equal z on two ranks
ref = r.copy()
O.port_track([el], ref, 1, loss=False)   # the one-rank wake over the whole bunch
res = {"rank": rank}
# interleaved shards
mine = staged_wake(r[rank::world].copy())
res["interleaved_bit_exact"] = bool(np.array_equal(mine.view(np.int64), ref[rank::world].view(np.int64)))
res["kicked"] = bool(np.any(mine[:, 5] != r[rank::world, 5]))
# contiguous shards, the second holding the bunch head (largest z) and every lost particle
order = np.argsort(np.where(np.isnan(r[:, 0]), np.inf, r[:, 4]), kind="stable")
half = order[: N // 2] if rank == 0 else order[N // 2:]
mine = staged_wake(r[half].copy())
res["contiguous_bit_exact"] = bool(np.array_equal(mine.view(np.int64), ref[half].view(np.int64)))
# the bunch's moments from the two halves (accel_beam_stat with a communicator): the sums and
# live count added over the ranks, then the centred second moments with the bunch's means
mine = r[half]
live = ~np.isnan(mine[:, 0])
s1 = torch.tensor(np.append(mine[live].sum(axis=0), live.sum()), dtype=torch.float64)
dist.all_reduce(s1, op=dist.ReduceOp.SUM)
s1 = s1.numpy()
mean = s1[:6] / s1[6]
d = mine[live] - mean
s2 = torch.tensor(np.concatenate([(d * d).sum(axis=0), [(d[:, 0] * d[:, 1]).sum(), (d[:, 2] * d[:, 3]).sum(),
                  (d[:, 0] * d[:, 5]).sum(), (d[:, 1] * d[:, 5]).sum(), (d[:, 2] * d[:, 4]).sum(),
                  (d[:, 3] * d[:, 4]).sum()]]), dtype=torch.float64)
dist.all_reduce(s2, op=dist.ReduceOp.SUM)
s2 = s2.numpy()
m_ref, sig_ref, cross_ref, nl_ref = O.port_beam_stat(r)
res["moments_count"] = bool(int(s1[6]) == nl_ref)
sc = np.where(sig_ref > 0, sig_ref, 1.0)  # x', y and y' of this bunch are all zero
res["moments_rel_err"] = float(max(np.max(np.abs(mean - m_ref) / sc),
                                   np.max(np.abs(np.sqrt(s2[:6] / s1[6]) - sig_ref) / sc),
                                   np.max(np.abs(s2[6:] / s1[6] - cross_ref)) / np.max(sig_ref) ** 2))
dist.barrier()
dist.destroy_process_group()
print("RESULT " + json.dumps(res))
"""


def test_two_gloo_ranks_split_bunch_wake():
    """The longitudinal wake of a bunch split over two ranks, exchanged as the engine does it
    (z range and live count by min / max / sum, then bin counts by sum): each rank's kicked
    particles equal, bit for bit, the one-rank wake of the whole bunch (integer counts and exact
    min / max make the exchange exact).  The bunch's moments from the two halves, exchanged as
    accel_beam_stat does with a communicator (first-pass sums and count, then centred second
    moments, each summed over the ranks), equal the oracle's moments of the whole bunch to
    1e-12."""
    pytest.importorskip("torch")
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, ROOT=ROOT, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WAKE_CHILD], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-3000:]
        res.append(json.loads([l for l in out.splitlines() if l.startswith("RESULT ")][-1][7:]))
    for r in res:
        assert r["interleaved_bit_exact"] and r["contiguous_bit_exact"] and r["kicked"], r
        # the moments of the split bunch against the oracle's moments of the whole bunch: the
        # same sums in another order of additions
        assert r["moments_count"] and r["moments_rel_err"] < 1e-12, r
