"""Replica placement and the multi-rank plumbing of bench.py, on CPU.

Replicas are independent, so the only multi-GPU logic is placement (every
replica on exactly one rank, balanced by cost), the gather of per-replica
results, and the max-over-ranks / sum-over-ranks reductions of the timing.
These run here as two gloo ranks on 127.0.0.1 (no GPU)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from ftspolysol_b200 import replicas as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_replica_set_shape():
    cs = R.replica_set(64)
    assert len(cs) == 64
    grids = [c.m[0] for c in cs]
    for g in R.GRIDS:
        assert grids.count(g) == 16
    for c in cs:
        assert c.L[0] == pytest.approx(0.5 * c.m[0])
        assert len(c.species[0].monomers) in R.CHAIN_LENGTHS
    salts = sorted(c.salt["num_salt"] / c.volume for c in cs)
    assert salts[0] == pytest.approx(0.01, abs=0.005) and salts[-1] == pytest.approx(0.5, abs=0.005)
    assert len({c.init_seed for c in cs}) == 64


@pytest.mark.parametrize("ws", [1, 2, 3, 8])
def test_assign_covers_every_replica_once_and_balances(ws):
    costs = [R.cost(c) for c in R.replica_set(64)]
    parts = R.assign(costs, ws)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    # LPT bound: no rank exceeds the mean by more than the largest single job
    assert max(loads) <= sum(costs) / ws + max(costs) + 1e-6
    assert parts == R.assign(costs, ws)   # deterministic


def test_ensemble_statistics():
    """Mean and standard error over the seeds of one system; a system with a
    single replica keeps its own time average and block error."""
    cs = R.replica_set(8, seeds_per_system=2)
    keys = {i: R.system_key(c) for i, c in enumerate(cs)}
    assert len(set(keys.values())) == 4
    for i in range(0, 8, 2):
        assert keys[i] == keys[i + 1] and cs[i].init_seed != cs[i + 1].init_seed
    res = {i: {"Pi": (1.0 + i, 0.1)} for i in range(8)}
    res[8] = {"Pi": (7.0, 0.25)}
    keys[8] = "single"
    ens = R.ensemble(res, keys, ["Pi"])
    g = ens[keys[0]]
    assert g["replicas"] == 2
    assert g["Pi"][0] == pytest.approx(1.5)
    assert g["Pi"][1] == pytest.approx(0.5)       # std([1, 2], ddof=1) / sqrt(2)
    assert ens["single"] == {"replicas": 1, "Pi": (7.0, 0.25)}


WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
from ftspolysol_b200 import replicas as R
ws, rank, local = bench.dist_setup()
costs = [R.cost(c) for c in R.replica_set(16)]
mine = R.assign(costs, ws)[rank]
res = R.gather({{i: {{"rank": rank, "Pi": (float(i), 0.0)}} for i in mine}}, ws)
cs = R.replica_set(16, seeds_per_system=2)
ens = R.ensemble(res, {{i: R.system_key(c) for i, c in enumerate(cs)}}, ["Pi"])
out = {{"rank": rank, "mine": mine, "gathered": {{str(k): v for k, v in res.items()}}, "ensemble": ens,
        "max": bench.dist_max(1.5 + rank, ws), "sum": bench.dist_sum(len(mine), ws)}}
bench.barrier(ws)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps(out))
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    a, b = outs
    assert sorted(a["mine"] + b["mine"]) == list(range(16))
    assert a["gathered"] == b["gathered"] and len(a["gathered"]) == 16
    for k, v in a["gathered"].items():
        assert int(k) in (a["mine"] if v["rank"] == 0 else b["mine"])
    assert a["max"] == b["max"] == 2.5
    # the ensemble over the gathered replicas: both ranks agree, and each
    # system averages the indices of its two seeds (2j, 2j + 1)
    assert a["ensemble"] == b["ensemble"] and len(a["ensemble"]) == 8
    for g in a["ensemble"].values():
        assert g["replicas"] == 2 and (g["Pi"][0] - 0.5) % 2 == 0
    assert a["sum"] == b["sum"] == 16
