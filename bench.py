#!/usr/bin/env python
"""Benchmark: particle-steps/s of the full SPH + FMM step at N = 1e6 on B200.

One step = GPU octree build, sort (hash, radix sort, cell ranges), gravity
(up pass, down pass, L2P + P2P), density, acceleration, kick/drift -- the
reference's Headless::step without the snapshot -- on a seeded two-body impact
of 800k + 200k particles (the 16384 + 4096 generator rescaled), leaf capacity
32, depth 7.  The state (~150 B/particle plus the 128 MiB cell table) is larger
than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one impact per GPU; the path has no data
exchange), launched by torchrun; value = all ranks' particle-steps / max time.
`--impl reference` times the reference's own kernels compiled for the host
(oracle/_ref, else the oracle restatement) on the host cores.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TARGET, N_IMPACTOR = 800_000, 200_000
LEAF, DEPTH = 32, 7
METRIC = "particle-steps/s at N=1e6, chosen vs plain form on one B200, grav err<=1e-3"
PASSES = ("tree", "sort", "gravity", "density", "acceleration", "step")
# compulsory HBM bytes per particle per pass (each array touched once)
ALGO_BYTES = {"tree": 76, "sort": 92, "gravity": 44, "density": 65, "acceleration": 88, "step": 92}
PASS_KERNELS = {
    "tree": "k_bbox, k_tree_keys, k_onesweep x3, k_children/k_emit/scan x7, k_marks, k_write, k_link",
    "sort": "k_hash_hist, k_onesweep x3, k_cells",
    "gravity": "k_up x8, k_down x8",
    "density": "k_gather, k_density",
    "acceleration": "k_acceleration",
    "step": "k_step",
}
LAUNCHES_PER_STEP = None  # filled from the pass structure below


def launches_per_step(depth: int) -> int:
    tree = 1 + 1 + 1 + 3 + 1 + depth * (1 + 4 + 1) + 1 + 1 + (depth + 1) + 4 + 4 + (depth + 1) + depth
    sort = 1 + 3 + 1
    gravity = 2 * (depth + 1)
    return tree + sort + gravity + 2 + 1 + 1


def load_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[2]) for r in self.rows if len(r) >= 10 and r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in self.rows if len(r) >= 10 and r[3].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            if len(r) < 10:
                continue
            for k, name in enumerate(names):
                if r[6 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


_T0 = time.perf_counter()


def log(msg: str):
    print(f"[bench {time.perf_counter() - _T0:8.2f}s] {msg}", file=sys.stderr, flush=True)


def make_ic(seed: int, scale: float = 1.0):
    ic_mod = importlib.import_module("real-time-planetary-impacts-mps_b200.ic")
    return ic_mod.make_impact(int(N_TARGET * scale), int(N_IMPACTOR * scale), seed=seed)


def cpu_reference(ic: dict, steps: int, warmup: int, budget_s: float | None = None) -> dict:
    """The reference's kernels on the host cores (oracle/_ref when built, else
    the oracle restatement), full N, reference CPU octree rebuilt every step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # noqa: E402 -- CPU-baseline leg only
    eos_mod = importlib.import_module("real-time-planetary-impacts-mps_b200.eos_tables")
    tabs = eos_mod.ensure_tables()
    kind = "ref" if os.path.exists(O.REF_PATH) else "oracle"
    if kind == "oracle":
        O.build()
    ef = O.aneos_load(tabs["forsterite"], 2048)
    ee = O.aneos_load(tabs["Fe85Si15"], 2048)
    st = O.OracleState(ic, ef, ee, kind=kind)
    cores = O.load("oracle").ora_get_threads() if kind == "oracle" else (os.cpu_count() or 1)

    def tree_fn(p):
        return O.tree_reference(p, LEAF, DEPTH, kind=kind)

    for _ in range(warmup):
        st.full_step(tree_fn)
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        st.full_step(tree_fn)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": st.n * done / dt, "unit": "particle-steps/s", "cores": cores,
            "kind": "reference" if kind == "ref" else "port", "steps": done, "seconds": dt,
            "sample": f"{done} full step(s) of the N={st.n} impact after {warmup} warm-up step(s), "
                      f"reference CPU octree (leaf {LEAF}) rebuilt each step, all passes"}


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    ic = make_ic(0)
    cb = cpu_reference(ic, args.steps, args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": "particle-steps/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": cb["steps"], "warmup": args.warmup,
            "ms_per_step": 1e3 * cb["seconds"] / max(cb["steps"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"two-body impact N={ic['n']} (800k+200k), leaf {LEAF}, depth {DEPTH}, "
                                   "plain form", "n_particles": int(ic["n"]), "parallelism": "replicas"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="particle count relative to 1e6 (diagnostics)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    pkg = importlib.import_module("real-time-planetary-impacts-mps_b200")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    ic = make_ic(rank, args.scale)
    log(f"ic ready: {ic['n']} particles")
    n = int(ic["n"])
    c = pkg.Compute(ic, max_children_in_leaf=LEAF, max_tree_depth=DEPTH)
    stream = torch.cuda.Stream()
    # warm-up: the first steps carry the reference's cold-start gravity (no |a| yet)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            c.step(stream)
            stream.synchronize()
            log("warm-up step done")
    stream.synchronize()
    c.synchronize()

    # the timed region replays K full steps captured into one CUDA graph
    K = args.steps
    calls = (c.updateOctreeBuffer, c.sort, c.gravitationalPass, c.densityPass, c.accelerationPass, c.stepPass)
    graph = None
    try:
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for k in range(K):
                for f in calls:
                    f(stream)
        mode = "cuda-graph"
    except Exception as exc:  # eager launches instead
        graph = None
        mode = f"eager ({type(exc).__name__})"
    stream.synchronize()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        if uuid and not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    sampler = ClockSampler(uuid)
    log(f"timing mode {mode}")
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    if graph is not None:
        with torch.cuda.stream(stream):  # replay() launches on the current stream
            graph.replay()
    else:
        with torch.cuda.stream(stream):
            for k in range(K):
                for f in calls:
                    f(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    c.synchronize()
    elapsed_ms = t_start.elapsed_time(t_end)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = world * n * K / (elapsed_ms / 1e3)
    log(f"timed region: {elapsed_ms / K:.3f} ms/step")

    # per-pass split: K more steps, eager, with an event between passes on the
    # launching stream (events inside a captured graph cannot be timed)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(PASSES) + 1)] for _ in range(K)]
    with torch.cuda.stream(stream):
        for k in range(K):
            ev[k][0].record(stream)
            for j, f in enumerate(calls):
                f(stream)
                ev[k][j + 1].record(stream)
    torch.cuda.synchronize()
    c.synchronize()
    per_pass = {p: 0.0 for p in PASSES}
    for k in range(K):
        for j, p in enumerate(PASSES):
            per_pass[p] += ev[k][j].elapsed_time(ev[k][j + 1])
    per_pass = {p: v / K for p, v in per_pass.items()}
    log("per-pass ms: " + ", ".join(f"{p} {v:.3f}" for p, v in per_pass.items()))

    # end to end through the public API: host state in, step, host state out
    import ctypes  # noqa: F401
    fields = ("pos", "vel", "u", "h", "rho")
    host = {f: torch.from_numpy(c.download(f)).pin_memory().numpy() for f in fields}
    h2d = sum(a.nbytes for a in host.values())
    d2h = h2d
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        for f in fields:
            c.upload(f, host[f])
        c.step_all(1)
        for f in fields:
            host[f][...] = c.download(f)
    c.synchronize()
    e2e_s = time.perf_counter() - t0
    log(f"e2e: {e2e_s / args.e2e_steps * 1e3:.2f} ms/step")
    e2e_times = torch.tensor([e2e_s], device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_times, op=dist.ReduceOp.MAX)
    e2e_value = world * n * args.e2e_steps / float(e2e_times.item())

    if rank == 0:
        dom = max(per_pass, key=per_pass.get)
        peaks = load_peaks()
        achieved = ALGO_BYTES[dom] * n / (per_pass[dom] / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded two-body impact generator)",
            "config": {"workload": f"two-body impact N={n} (800k+200k), leaf {LEAF}, depth {DEPTH}, plain form",
                       "form": "plain", "n_particles": n, "leaf_capacity": LEAF, "max_tree_depth": DEPTH,
                       "parallelism": f"replicas x{world}", "l2": "state larger than L2 (no flush)",
                       "timing": mode},
            "pass_ms": {p: round(v, 4) for p, v in per_pass.items()},
            "roofline": {"bound": "hbm", "kernel": f"{dom} pass ({PASS_KERNELS[dom]})", "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "peak_source": peaks["source"], "algo_bytes_per_particle": ALGO_BYTES[dom],
                         "traffic": None},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches_per_step(DEPTH) * K,
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            log("cpu baseline ...")
            cb = cpu_reference(ic, steps=1, warmup=1, budget_s=30.0)
            log(f"cpu baseline: {cb['value']:.3e} particle-steps/s on {cb['cores']} cores")
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    c.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
