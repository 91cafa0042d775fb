"""The batched-ensemble workload (256 uneven warm-bubble cases) and its sharding.

Each of `n` cases is a plain warm bubble whose grid and bubble are drawn from
a seeded generator: NX from {256, 512, 1024, 2048}, NZ from {64, 96, 128},
amplitude U(1, 3) K, centre U(0.2, 0.8) of the domain, radius U(1, 3) km,
dx = dz = 200 m, dt = 1 s. Cases are independent, so `bench.py --gpus N`
splits the list over the ranks by cost (cells), with no exchange between them.
"""
from __future__ import annotations

import numpy as np

from .initial_state import VVMState, warm_bubble

NX_CHOICES = (256, 512, 1024, 2048)
NZ_CHOICES = (64, 96, 128)


def ensemble_specs(n: int = 256, seed: int = 3) -> list[dict]:
    """Seeded grid and bubble of every case."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        specs.append(dict(NX=int(rng.choice(NX_CHOICES)), NZ=int(rng.choice(NZ_CHOICES)),
                          amp=float(rng.uniform(1.0, 3.0)), xc_frac=float(rng.uniform(0.2, 0.8)),
                          radius=float(rng.uniform(1000.0, 3000.0))))
    return specs


def ensemble_state(spec: dict, dx: float = 200.0, dz: float = 200.0, dt: float = 1.0) -> VVMState:
    return warm_bubble(spec["NX"], spec["NZ"], dx, dz, dt, amp=spec["amp"], radius=spec["radius"],
                       xc_frac=spec["xc_frac"])


def shard_by_cost(costs, world: int) -> list[list[int]]:
    """Case indices of each rank: longest cases first, each to the rank with
    the least load so far (ties to the lower rank). Deterministic, so every
    rank computes the same split without communicating."""
    loads = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        r = min(range(world), key=lambda q: (loads[q], q))
        shards[r].append(i)
        loads[r] += costs[i]
    for s in shards:
        s.sort()
    return shards
