#!/usr/bin/env python
"""Benchmark: particle-steps/s of the full SPH + FMM step at N = 1e6 on B200,
the chosen form against the plain form.

One step = GPU octree build, sort (hash, radix sort, cell ranges), gravity,
density, acceleration, kick/drift -- the reference's Headless::step without
the snapshot -- on a seeded two-body impact of 800k + 200k particles (the
16384 + 4096 generator rescaled), leaf capacity 32, depth 7.  The state
(~150 B/particle plus the 128 MiB cell table) is larger than the 126 MB L2,
so no flush is needed between steps.

Forms (one context each, same initial conditions):
  plain   the reference's logic (its adaptive gravity acceptance, float
          positions, plain initial h guess) -- what the parity tests pin;
  chosen  opening-angle gravity (theta, default 0.6), mixed precision (FP64
          master positions and time, Kahan sums) and the learned h seed,
          trained on the warm-up steps' density passes and refreshed every
          step (--online-iters Adam steps beside the tree, sort and gravity
          passes, inside the timed steps).
`value` is the chosen form; `chosen_over_plain` is the ratio of the two
graph-replayed step times.  The line also carries the gravity error of both
forms against an FP64 direct sum (16 384 targets), the total-energy drift of
both over `--drift-steps` further steps, and the learned seed's iteration
counts.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one impact per GPU; the path has no data
exchange), launched by torchrun; value = all ranks' particle-steps / max time.
`--ensemble M [--autotune]` times the batched ensemble of M seeded impacts
instead (N log-uniform in [2e4, 5e5]); with N > 1 the instances are split over
the ranks by particle totals and the per-instance records gathered at the end.
`--impl reference` times the reference's own kernels compiled for the host
(oracle/_ref, else the oracle restatement) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes
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
    "gravity": "plain: k_up x8, k_down x8; chosen: k_up_theta x8, k_gather_key_order, k_walk",
    "density": "k_gather, [k_mlp (learned seed)], k_tile_starts, k_density_tile, k_density_deferred",
    "acceleration": "k_tile_starts, k_acceleration_tile, k_acceleration_deferred",
    "step": "k_step",
}


def launches_per_step(depth: int, chosen: bool, online_iters: int = 0, seed: bool | None = None) -> int:
    """Kernels of one step (memsets excluded), counted from the pass structure
    (matches the ncu launch list: 116 plain, 131 chosen with 8 online Adam
    steps, at depth 7)."""
    scan = 4  # reduce, blocks, apply, total
    tree = 3 + 3 + 1 + depth * (1 + scan + 1) + 1 + 1 + (depth + 1) + 2 * scan + (depth + 1) + depth
    sort = 1 + 3 + 1 + 1                 # hash, 3 passes, cells, units
    gravity = (depth + 1) + 2 if chosen else 2 * (depth + 1)
    # gather, tile starts, tile pass, coarse starts, coarse tile pass, deferred pass
    density = 6
    if chosen if seed is None else seed:
        density += 3                     # seed inference, pair capture, targets
        if online_iters > 0:
            density += 2 + 2 * online_iters  # standardisation, gradient + Adam per step
    acceleration = 5                     # tile starts, tile pass, coarse starts, coarse pass, deferred pass
    return tree + sort + gravity + density + acceleration + 1


def load_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic() -> dict:
    """DRAM bytes per launch of the kernels captured with ncu (profiles/)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


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


def host_cores() -> dict:
    """Logical CPUs usable here and the physical core count (lscpu)."""
    logical = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    physical = None
    try:
        out = subprocess.run(["lscpu", "-p=CORE,SOCKET"], capture_output=True, text=True, timeout=10).stdout
        cores = {tuple(l.split(",")) for l in out.splitlines() if l and not l.startswith("#")}
        physical = len(cores) or None
    except Exception:
        pass
    return {"logical": logical, "physical": physical}


def set_omp_threads(n: int):
    """Threads of the OpenMP runtime the host reference library runs on."""
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass
    os.environ["OMP_NUM_THREADS"] = str(n)


def cpu_reference(ic: dict, steps: int, warmup: int, budget_s: float | None = None, threads: int | None = None) -> dict:
    """The reference's kernels on the host cores (oracle/_ref when built, else
    the oracle restatement), full N, reference CPU octree rebuilt every step."""
    if threads:
        set_omp_threads(threads)
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
    hc = host_cores()

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
    used = int(os.environ.get("OMP_NUM_THREADS", hc["logical"]))
    return {"value": st.n * done / dt, "unit": "particle-steps/s", "cores": used,
            "physical_cores": hc["physical"], "logical_cpus": hc["logical"],
            "kind": "reference" if kind == "ref" else "port", "steps": done, "seconds": dt,
            "sample": f"{done} full step(s) of the N={st.n} impact after {warmup} warm-up step(s), "
                      f"reference CPU octree (leaf {LEAF}) rebuilt each step, all passes, {used} threads"}


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
                                   "the reference's logic", "n_particles": int(ic["n"]), "parallelism": "replicas"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "physical_cores")},
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def graph_time(c, stream, K: int) -> tuple[float, str]:
    """Device time (ms) of K full steps captured into one CUDA graph."""
    import torch
    calls = (c.updateOctreeBuffer, c.sort, c.gravitationalPass, c.densityPass, c.accelerationPass, c.stepPass)
    try:
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            for _ in range(K):
                for f in calls:
                    f(stream)
        mode = "cuda-graph"
    except Exception as exc:
        graph, mode = None, f"eager ({type(exc).__name__})"
    stream.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    with torch.cuda.stream(stream):
        if graph is not None:
            graph.replay()
        else:
            for _ in range(K):
                for f in calls:
                    f(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    c.synchronize()
    del graph
    return t0.elapsed_time(t1), mode


def pass_times(c, stream, K: int, label: str) -> dict:
    """Per-pass device times (ms), eager with events between the passes; the
    launches sit in an NVTX range named `label` (for profiler filters)."""
    import torch
    calls = (c.updateOctreeBuffer, c.sort, c.gravitationalPass, c.densityPass, c.accelerationPass, c.stepPass)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(PASSES) + 1)] for _ in range(K)]
    torch.cuda.nvtx.range_push(label)
    with torch.cuda.stream(stream):
        for k in range(K):
            ev[k][0].record(stream)
            for j, f in enumerate(calls):
                f(stream)
                ev[k][j + 1].record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    c.synchronize()
    return {p: sum(ev[k][j].elapsed_time(ev[k][j + 1]) for k in range(K)) / K for j, p in enumerate(PASSES)}


def gravity_error(c, targets) -> dict:
    """Median / p99 relative acceleration error of the form's gravity pass
    against the FP64 direct sum, at the current positions."""
    ref = c.gravity_direct_f64(targets)
    c.updateOctreeBuffer()
    c.sort()
    c.gravitationalPass()
    c.synchronize()
    a = c.download("acc")[targets].astype(np.float64)
    e = np.linalg.norm(a - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)
    return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max()),
            "targets": int(targets.size), "reference": "FP64 direct sum, cubic-spline softening 0.04"}


def energy_drift(c, steps: int, chunk: int = 100) -> dict:
    log("  drift: first diagnostics")
    d0 = c.diagnostics()
    worst, done = 0.0, 0
    while done < steps:
        k = min(chunk, steps - done)
        c.step_all(k)
        done += k
        d = c.diagnostics()
        worst = max(worst, abs(d["total"] - d0["total"]) / abs(d0["total"]))
        log(f"  drift: {done} steps, |dE|/|E0| so far {worst:.3e}")
    c.synchronize()
    return {"steps": steps, "max_rel_change_total_energy": worst, "e0": d0["total"],
            "sampled_every": chunk}


def fp32_peak(lib, stream) -> float:
    """Measured FP32 FMA throughput (TFLOP/s) of this device."""
    import torch
    blocks, iters = 148 * 16, 8192
    sink = torch.zeros(blocks, dtype=torch.float32, device="cuda")
    s = ctypes.c_void_p(stream.cuda_stream)
    for _ in range(2):
        lib.sph_probe_fp32_fma(blocks, iters, ctypes.c_void_p(sink.data_ptr()), s)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(5):
        lib.sph_probe_fp32_fma(blocks, iters, ctypes.c_void_p(sink.data_ptr()), s)
    t1.record(stream)
    torch.cuda.synchronize()
    flops = 5.0 * blocks * 256 * iters * 16
    return flops / (t0.elapsed_time(t1) / 1e3) / 1e12


ENSEMBLE_METRIC = "aggregate particle-steps/s, ensemble of impacts (N log-uniform 2e4-5e5), one graph launch per step"


def run_ensemble(args, rank: int, world: int, local: int):
    """The batched ensemble: `args.ensemble` seeded impacts split over the
    ranks by particle totals; each rank steps its share as one Ensemble
    (theta gravity + mixed precision per instance, tuned when --autotune).
    value = all instances' particle-steps / max over ranks of the device time;
    per-instance total-energy change over the timed steps (FP64 diagnostics)
    is gathered to rank 0."""
    import torch
    pkg = importlib.import_module("real-time-planetary-impacts-mps_b200")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    specs = pkg.ensemble.make_specs(args.ensemble, seed=args.ensemble_seed)
    sizes = [s["n"] for s in specs]
    mine = pkg.ensemble.shard(sizes, world)[rank]
    t0 = time.perf_counter()
    ics = [pkg.ensemble.make_ic(specs[i]) for i in mine]
    form = {"gravity": "theta", "theta": args.theta, "precision": "mixed"}
    ens = pkg.Ensemble(ics, [form] * len(ics), autotune=args.autotune, max_children_in_leaf=LEAF,
                       max_tree_depth=DEPTH)
    log(f"rank {rank}: {len(mine)} instances, {sum(ens.sizes)} particles, created and tuned in "
        f"{time.perf_counter() - t0:.1f} s")
    stream = torch.cuda.Stream()
    e0 = [c.diagnostics(stream)["total"] for c in ens.instances]
    with torch.cuda.stream(stream):
        ens.step(args.warmup, stream)
    ens.synchronize(stream)
    K = args.steps
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        if uuid and not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    ens.step(K, stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    # end to end: the same steps timed on the host clock through the public
    # API, with each instance's global time read back after every step
    t_h = time.perf_counter()
    d2h = 0
    for _ in range(K):
        ens.step(1, stream)
        for c in ens.instances:
            c.download("global_time")
            d2h += 4
    ens.synchronize(stream)
    e2e_s = time.perf_counter() - t_h
    e1 = [c.diagnostics(stream)["total"] for c in ens.instances]
    tun = ens.tuning()
    records = {i: {"n": sizes[i], "rank": rank, "rel_energy_change": abs(b - a) / abs(a) if a else None,
                   "tuning": tun[j]} for j, (i, a, b) in enumerate(zip(mine, e0, e1))}
    ens.close()
    t = torch.tensor([ms, e2e_s], device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_s = float(t[0]), float(t[1])
    merged = pkg.ensemble.gather(records)
    if rank == 0:
        total = sum(sizes)
        value = total * K / (ms / 1e3)
        drifts = [r["rel_energy_change"] for r in merged.values() if r["rel_energy_change"] is not None]
        leaves = [r["tuning"]["max_children_in_leaf"] for r in merged.values()]
        tiles = [r["tuning"]["tile_block_max"] for r in merged.values()]
        line = {
            "metric": ENSEMBLE_METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32 (FP64 positions, time and reductions)",
            "data": "synthetic (seeded impacts, per-instance generator seeds)",
            "config": {"workload": f"ensemble of {len(specs)} impacts, N log-uniform in [2e4, 5e5] "
                                   f"(total {total}), angles 30-60 deg, speeds 1.0-1.4 v_esc, mass ratios 0.08-0.15",
                       "form": f"theta {args.theta} gravity + mixed precision", "autotune": bool(args.autotune),
                       "parallelism": f"instances split over {world} GPU(s) by particle totals",
                       "l2": "state larger than L2 (no flush)", "timing": "cuda-graph, one launch per step"},
            "per_instance_rel_energy_change": {"median": float(np.median(drifts)), "max": float(np.max(drifts)),
                                               "steps": K + args.warmup + K},
            "tuning": {"leaf_capacity_counts": {str(v): leaves.count(v) for v in sorted(set(leaves))},
                       "tile_block_max_counts": {str(v): tiles.count(v) for v in sorted(set(tiles))}},
            "e2e": {"value": total * K / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(d2h // max(K, 1)) * world,
                    "path": "sph_ensemble_step(1) + every instance's global time read back, per step"},
            "gpu_launches": launches_per_step(DEPTH, True, seed=False) * len(specs) * K,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="particle count relative to 1e6 (diagnostics)")
    ap.add_argument("--no-coarse-tiles", action="store_true",
                    help="hand particles whose neighbour boxes reach past 3 cells to the per-particle walk")
    ap.add_argument("--theta", type=float, default=0.6, help="opening angle of the chosen form's gravity")
    ap.add_argument("--train-iters", type=int, default=600, help="Adam steps after each warm-up step")
    ap.add_argument("--online-iters", type=int, default=4,
                    help="Adam steps of the seed's online refresh per step (0: seed trained in warm-up only)")
    ap.add_argument("--drift-steps", type=int, default=100,
                    help="steps of the energy-drift comparison (the 1000-step comparison runs at config 0 in the tests)")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="time the batched ensemble of this many impacts instead of the N=1e6 impact")
    ap.add_argument("--ensemble-seed", type=int, default=0)
    ap.add_argument("--autotune", action="store_true", help="ensemble: tune tiles and leaf capacity per instance")
    ap.add_argument("--single-thread-baseline", action="store_true",
                    help="also time the CPU reference on one thread (about two minutes at N=1e6)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.ensemble > 0:
        run_ensemble(args, rank, world, local)
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
    n = int(ic["n"])
    log(f"ic ready: {n} particles")
    stream = torch.cuda.Stream()
    lib = pkg._lib.load()
    peak32 = fp32_peak(lib, stream)
    log(f"fp32 fma peak {peak32:.1f} TFLOP/s")
    K = args.steps

    # ---- plain form -------------------------------------------------------
    cp = pkg.Compute(ic, max_children_in_leaf=LEAF, max_tree_depth=DEPTH)
    if args.no_coarse_tiles:
        cp.set_tiling(coarse=False)
    cp.hseed_capture(True)  # allocates the density-pass counters; records nothing once off
    cp.hseed_capture(False)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            cp.step(stream)
    stream.synchronize()
    cp.synchronize()
    # ---- chosen form: theta gravity, mixed precision, learned h seed --------
    cc = pkg.Compute(ic, max_children_in_leaf=LEAF, max_tree_depth=DEPTH)
    if args.no_coarse_tiles:
        cc.set_tiling(coarse=False)
    cc.set_form(gravity="theta", theta=args.theta, precision="mixed")
    cc.hseed_capture(True)
    train_ms = []
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            cc.step(stream)
            stream.synchronize()
            t0 = time.perf_counter()
            torch.cuda.nvtx.range_push("seed_training")
            cc.hseed_train(args.train_iters, 16384, 1e-3, stream)
            torch.cuda.nvtx.range_pop()
            train_ms.append((time.perf_counter() - t0) * 1e3)
    cc.hseed_capture(False)
    cc.set_form(gravity="theta", theta=args.theta, precision="mixed", h_seed="learned")
    if args.online_iters > 0:
        cc.hseed_online(args.online_iters, 16384, 1e-3)
    with torch.cuda.stream(stream):
        cc.step(stream)
    stream.synchronize()
    cc.synchronize()
    log(f"warm-up done; seed training {np.mean(train_ms):.1f} ms per call of {args.train_iters} Adam steps")

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        if uuid and not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = None
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    plain_ms, mode = graph_time(cp, stream, K)
    chosen_ms, mode_c = graph_time(cc, stream, K)
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    if dist is not None:
        t = torch.tensor([plain_ms, chosen_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        plain_ms, chosen_ms = float(t[0]), float(t[1])
    value = world * n * K / (chosen_ms / 1e3)
    plain_value = world * n * K / (plain_ms / 1e3)
    log(f"timed: plain {plain_ms / K:.3f} ms/step, chosen {chosen_ms / K:.3f} ms/step")

    pp = pass_times(cp, stream, K, "plain_passes")
    sp = cp.hseed_stats()
    pc = pass_times(cc, stream, K, "chosen_passes")
    st = cc.hseed_stats()
    log("plain  per-pass ms: " + ", ".join(f"{p} {v:.3f}" for p, v in pp.items()))
    log("chosen per-pass ms: " + ", ".join(f"{p} {v:.3f}" for p, v in pc.items()))

    # ---- end to end through the public API, chosen form ---------------------
    fields = {"pos64": np.float64, "vel": np.float32, "u": np.float32, "h": np.float32, "rho": np.float32}
    host = {}
    for f, dtp in fields.items():
        a = cc.download(f)
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        host[f] = (t, t.numpy())
    h2d = sum(a.nbytes for _, a in host.values())
    d2h = h2d
    state = {f: a for f, (_, a) in host.items()}
    cc.step_host(state, state, stream)  # first call: eager step + graph capture, outside the timed region
    stream.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        # inputs copied in, one step, outputs copied back: every step through host memory
        cc.step_host(state, state, stream)
        stream.synchronize()
    e2e_s = time.perf_counter() - t0
    cc.synchronize()
    log(f"e2e: {e2e_s / args.e2e_steps * 1e3:.2f} ms/step")
    e2e_times = torch.tensor([e2e_s], device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_times, op=dist.ReduceOp.MAX)
    e2e_value = world * n * args.e2e_steps / float(e2e_times.item())

    extra = {}
    if rank == 0:
        rng = np.random.default_rng(12)
        targets = rng.choice(n, 16384, replace=False).astype(np.int32)
        extra["gravity_error"] = {"chosen": gravity_error(cc, targets), "plain": gravity_error(cp, targets)}
        log(f"gravity error: {extra['gravity_error']}")
        if args.drift_steps > 0:
            extra["energy_drift"] = {"plain": energy_drift(cp, args.drift_steps),
                                     "chosen": energy_drift(cc, args.drift_steps)}
            dp = extra["energy_drift"]["plain"]["max_rel_change_total_energy"]
            dc = extra["energy_drift"]["chosen"]["max_rel_change_total_energy"]
            extra["energy_drift"]["chosen_over_plain"] = dc / dp if dp > 0 else None
            log(f"energy drift over {args.drift_steps} steps: plain {dp:.3e}, chosen {dc:.3e}")

    if rank == 0:
        peaks = load_peaks()
        traffic = load_traffic()
        dom = max(pc, key=pc.get)
        achieved = ALGO_BYTES[dom] * n / (pc[dom] / 1e3) / 1e9
        sweeps = st["sweeps"] / max(st["particles"], 1)
        # density flops per particle: 20 per neighbour per sweep + 45 per neighbour in the gradient sweep
        dens_flops = (20.0 * sweeps + 45.0) * 63.0
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": chosen_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 positions, time and reductions in the chosen form)",
            "data": "synthetic (seeded two-body impact generator)",
            "config": {"workload": f"two-body impact N={n} ({int(N_TARGET * args.scale)}+"
                                   f"{int(N_IMPACTOR * args.scale)}), leaf {LEAF}, depth {DEPTH}",
                       "form": f"chosen: theta {args.theta} gravity + mixed precision + learned h seed"
                               + (f" (refreshed online, {args.online_iters} Adam steps per step)"
                                  if args.online_iters > 0 else ""),
                       "n_particles": n, "leaf_capacity": LEAF, "max_tree_depth": DEPTH,
                       "parallelism": f"replicas x{world}", "l2": "state larger than L2 (no flush)",
                       "timing": mode_c},
            "chosen_over_plain": plain_ms / chosen_ms,
            "plain": {"value": plain_value, "ms_per_step": plain_ms / K, "timing": mode},
            "pass_ms": {"chosen": {p: round(v, 4) for p, v in pc.items()},
                        "plain": {p: round(v, 4) for p, v in pp.items()}},
            "h_seed": {"sweeps_per_particle": sweeps, "max_sweeps": st["max_sweeps"],
                       "fallback_rate": st["fallbacks"] / max(st["particles"], 1),
                       "plain_sweeps_per_particle": sp["sweeps"] / max(sp["particles"], 1),
                       "density_tiles": st["tiles"], "density_deferred_particles": st["deferred"],
                       "acceleration_deferred_particles": st["accel_deferred"],
                       "density_coarse_tiles": st["coarse_tiles"],
                       "acceleration_coarse_tiles": st["accel_coarse_tiles"],
                       "training_ms_per_call": float(np.mean(train_ms)), "adam_steps_per_call": args.train_iters,
                       "online_adam_steps_per_step": args.online_iters},
            "roofline": {"bound": "hbm", "kernel": f"{dom} pass ({PASS_KERNELS[dom]}), chosen form",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "algo_bytes_per_particle": ALGO_BYTES[dom],
                         "traffic": traffic.get(dom, {}).get("bytes_per_launch"),
                         "traffic_source": traffic.get(dom, {}).get("source"),
                         "fp32": {"peak_tflops_measured": peak32,
                                  "density_achieved_tflops": dens_flops * n / (pc["density"] / 1e3) / 1e12,
                                  "density_flops_per_particle": dens_flops}},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "form": "chosen",
                    "path": "sph_step_host (pos64, vel, u, h, rho in and out, pinned), one sync per step"},
            "gpu_launches": launches_per_step(DEPTH, True, args.online_iters) * K,
            "clocks": clocks,
        }
        line.update(extra)
        if not args.no_cpu_baseline and world == 1:
            log("cpu baseline ...")
            hc = host_cores()
            cb = cpu_reference(ic, steps=10, warmup=1, budget_s=20.0, threads=hc["logical"])
            log(f"cpu baseline: {cb['value']:.3e} particle-steps/s on {cb['cores']} threads")
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "physical_cores")}
            if args.single_thread_baseline:
                one = cpu_reference(ic, steps=1, warmup=1, threads=1)
                log(f"cpu baseline, one thread: {one['value']:.3e} particle-steps/s")
                line["cpu_baseline"]["single_thread"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}
                set_omp_threads(hc["logical"])
        print(json.dumps(line), flush=True)
    cp.close()
    cc.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
