"""Host side of the batched ensemble (no counterpart in the reference, which
runs one impact per process): the seeded instance set of the ensemble
workload, the split of instances over GPUs, and the end-of-run gather of
per-instance scalars.

Instances are independent, so the split needs no data exchange while
stepping: each rank builds an Ensemble (compute.Ensemble) from its share and
steps it alone; the only collective is one gather of small per-instance
records at the end (torch.distributed, any backend).
"""
from __future__ import annotations

import math

import numpy as np

from . import ic as ic_mod


def make_specs(count: int = 64, seed: int = 0, n_min: float = 2e4, n_max: float = 5e5) -> list[dict]:
    """`count` impacts: total particle counts log-uniform in [n_min, n_max],
    impact angles uniform in 30-60 degrees, approach speeds 1.0-1.4 times the
    mutual escape speed, impactor mass ratios 0.08-0.15; equal-mass
    particles, so the impactor holds ratio / (1 + ratio) of them.  Each
    instance has its own generator seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        q = float(rng.uniform(0.08, 0.15))
        n_imp = max(1, int(round(n * q / (1.0 + q))))
        specs.append(dict(index=i, n=n, n_target=n - n_imp, n_impactor=n_imp, mass_ratio=q,
                          angle_deg=float(rng.uniform(30.0, 60.0)), speed_factor=float(rng.uniform(1.0, 1.4)),
                          seed=int(seed) * 100003 + i))
    return specs


def make_ic(spec: dict) -> dict:
    """Initial conditions of one instance (ic.make_impact)."""
    return ic_mod.make_impact(spec["n_target"], spec["n_impactor"], seed=spec["seed"],
                              mass_ratio=spec["mass_ratio"], speed_factor=spec["speed_factor"],
                              angle_deg=spec["angle_deg"])


def shard(sizes: list[int], world: int) -> list[list[int]]:
    """Split instances over `world` ranks so that the particle totals are
    balanced: largest first, each to the rank with the smallest total so far
    (ties to the lower rank).  Returns each rank's instance indices, in
    increasing order; every instance appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def gather(records: dict[int, dict], group=None) -> dict[int, dict]:
    """Every rank's per-instance records, merged by instance index (one
    all-gather of Python objects when torch.distributed is initialised with
    more than one rank; the local records otherwise)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return dict(records)
    out: list = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, dict(records), group=group)
    merged: dict[int, dict] = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"instance {k} reported by two ranks")
            merged[int(k)] = v
    return merged
