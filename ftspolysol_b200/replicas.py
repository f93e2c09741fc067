"""Replica sets and their placement on GPUs.

A replica is one independent complex-Langevin system (its own grid, chain
length, salt and seed).  Replicas share nothing, so the only multi-GPU work is
placement: `assign` spreads replicas over ranks by estimated cost (longest
processing time first), and `gather` collects per-replica results on every
rank after the run.  One process per GPU; `torch.distributed` is only used
for the gather (any backend: NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence

import numpy as np

from .cases import Case, homopolymer

GRIDS = (32, 48, 64, 96)
CHAIN_LENGTHS = (20, 32, 50)


def replica_set(n: int = 64, seed: int = 2024, dt: float = 0.005, seeds_per_system: int = 1) -> List[Case]:
    """The uneven replica sweep: n replicas, a quarter each on 32^3, 48^3,
    64^3 and 96^3 grids with box side L = 0.5 b x grid, N drawn from
    {20, 32, 50}, salt swept uniformly over 0.01-0.5 b^-3, bead density
    0.5 b^-3, v = 0.1, lB = 1, monovalent counterions, the isotropic pressure
    in the record; every replica has its own initial-field seed (its noise seed is chosen by the caller).  With
    seeds_per_system = k, consecutive groups of k replicas share one system
    (grid, N, salt) and differ only in their seeds, so that `ensemble` can
    average over them."""
    if seeds_per_system < 1 or n % seeds_per_system:
        raise ValueError("n must be a multiple of seeds_per_system")
    rng = np.random.default_rng(seed)
    salts = np.linspace(0.01, 0.5, n // seeds_per_system)
    rng.shuffle(salts)
    out = []
    for r in range(n):
        m = GRIDS[r * len(GRIDS) // n]
        if r % seeds_per_system == 0:
            N = int(rng.choice(CHAIN_LENGTHS))
            salt = float(salts[r // seeds_per_system])
        V = (0.5 * m) ** 3
        nchain = max(1, int(round(0.5 * V / N)))
        out.append(Case(name="rep%02d_%dcube_N%d" % (r, m, N), m=(m, m, m), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0],
                        xi=0.1, lB=1.0, species=[homopolymer("P", nchain, N)],
                        counterions={"number": "auto_neutralize", "valence": 1.0},
                        salt={"num_salt": int(round(salt * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                        dt=dt, isotropic_pressure=True, init_seed=1000 + r))
    return out


def system_key(case: Case) -> str:
    """Replicas with equal keys simulate the same system (seeds aside)."""
    salt = case.salt["num_salt"] if case.salt else 0
    return "%dcube_N%d_salt%d" % (case.m[0], case.species[0].N, salt)


def ensemble(results: Dict[int, dict], keys: Dict[int, str], names: Sequence[str]) -> Dict[str, dict]:
    """Ensemble statistics of time-averaged observables over the replicas of
    each system.  results[i][name] = (time average, its block standard
    error) of replica i; keys[i] names its system.  Per system and
    observable: the mean over its replicas, the standard error of that mean
    (the spread over replicas / sqrt(n) for n >= 2, else the replica's own
    block error) and n."""
    groups: Dict[str, List[int]] = {}
    for i in sorted(results):
        groups.setdefault(keys[i], []).append(i)
    out: Dict[str, dict] = {}
    for k, idx in groups.items():
        g = {"replicas": len(idx)}
        for name in names:
            vals = np.array([results[i][name][0] for i in idx], dtype=np.float64)
            errs = np.array([results[i][name][1] for i in idx], dtype=np.float64)
            mean = float(np.mean(vals))
            if len(idx) >= 2:
                se = float(np.std(vals, ddof=1) / math.sqrt(len(idx)))
            else:
                se = float(errs[0])
            g[name] = (mean, se)
        out[k] = g
    return out


def cost(case: Case) -> float:
    """Relative cost of one step: segments x grid points x log2(points)."""
    V = int(np.prod(case.m))
    N = sum(len(s.monomers) for s in case.species)
    return float(N * V * math.log2(V))


def assign(costs: Sequence[float], world_size: int) -> List[List[int]]:
    """Replica indices per rank, longest processing time first: each replica,
    in order of decreasing cost, goes to the rank with the least total so
    far (ties to the lower rank).  Deterministic, so every rank computes the
    same placement without communication."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    out: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def gather(local: Dict[int, dict], world_size: int) -> Dict[int, dict]:
    """Merges {replica index: result} dicts from all ranks (every rank gets
    the union).  world_size 1 returns the input."""
    if world_size <= 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world_size
    dist.all_gather_object(parts, local)
    merged: Dict[int, dict] = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError("replica %d reported by two ranks" % k)
            merged[k] = v
    return merged
