"""Host side of the batched ensemble: the seeded instance set, the split of
instances over ranks, and the end-of-run gather over a real two-rank gloo
process group (CPU only)."""
from __future__ import annotations

import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def test_specs_follow_the_workload(pkg):
    specs = pkg.ensemble.make_specs(64, seed=5)
    assert len(specs) == 64
    assert specs == pkg.ensemble.make_specs(64, seed=5)  # seeded
    n = np.array([s["n"] for s in specs])
    assert n.min() >= 2e4 and n.max() <= 5e5
    # log-uniform: the mean of log n sits near the middle of the log range
    mid = 0.5 * (math.log(2e4) + math.log(5e5))
    assert abs(np.mean(np.log(n)) - mid) < 0.35
    for s in specs:
        assert 30.0 <= s["angle_deg"] <= 60.0
        assert 1.0 <= s["speed_factor"] <= 1.4
        assert 0.08 <= s["mass_ratio"] <= 0.15
        assert s["n_target"] + s["n_impactor"] == s["n"]
        # equal-mass particles: the impactor's share is ratio / (1 + ratio)
        assert abs(s["n_impactor"] / s["n"] - s["mass_ratio"] / (1 + s["mass_ratio"])) < 1e-3
    assert len({s["seed"] for s in specs}) == 64


def test_instance_ic_is_an_impact(pkg):
    spec = pkg.ensemble.make_specs(3, seed=1, n_min=3000, n_max=3000)[0]
    ic = pkg.ensemble.make_ic(spec)
    assert ic["pos"].reshape(-1, 3).shape[0] == 3000
    m = np.asarray(ic["mass"])
    # equal-mass particles up to the rounding of the impactor's particle count
    assert np.allclose(m, m[0], rtol=2e-2)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_covers_every_instance_once_and_balances(pkg, world):
    sizes = [s["n"] for s in pkg.ensemble.make_specs(64, seed=2)]
    parts = pkg.ensemble.shard(sizes, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(sizes[i] for i in p) for p in parts]
    # greedy largest-first: no rank exceeds the mean by more than the largest instance
    assert max(loads) - min(loads) <= max(sizes)
    assert max(loads) <= sum(sizes) / world + max(sizes)


def test_shard_rejects_an_empty_world(pkg):
    with pytest.raises(ValueError):
        pkg.ensemble.shard([1, 2], 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import importlib
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    pkg = importlib.import_module("real-time-planetary-impacts-mps_b200")
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs = pkg.ensemble.make_specs(16, seed=9)
        sizes = [s["n"] for s in specs]
        mine = pkg.ensemble.shard(sizes, world)[rank]
        # stand-in for the per-instance scalars a rank reports after stepping
        records = {i: {"n": sizes[i], "rank": rank, "particle_steps": 10 * sizes[i]} for i in mine}
        merged = pkg.ensemble.gather(records)
        if rank == 0:
            import json
            with open(os.path.join(out_dir, "merged.json"), "w") as f:
                json.dump({str(k): v for k, v in merged.items()}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_over_gloo(pkg, tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    import json
    merged = {int(k): v for k, v in json.loads((tmp_path / "merged.json").read_text()).items()}
    specs = pkg.ensemble.make_specs(16, seed=9)
    sizes = [s["n"] for s in specs]
    parts = pkg.ensemble.shard(sizes, world)
    assert sorted(merged) == list(range(16))
    for i, rec in merged.items():
        assert rec["n"] == sizes[i]
        assert i in parts[rec["rank"]]
    assert sum(r["particle_steps"] for r in merged.values()) == 10 * sum(sizes)
    assert {r["rank"] for r in merged.values()} == {0, 1}
