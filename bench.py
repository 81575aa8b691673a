"""Benchmark of the B200 force-layout step (libgvizcuda).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ba1m|grid32|er65k_exact]

Default workload (the headline configuration): Barabasi-Albert graph,
n = 1,048,576, m = 4 (4,194,294 edges, seeded), LinLog with gravity 1.0 and
degree-sized prevent-overlap (r = 1.0 * (1 + 0.5 sqrt(deg))), Barnes-Hut
theta = 0.8, start uniform in [-1000, 1000]^2 (rand_r, seed 7), FP32 walk.

A step is one full gvizForceEmbedderStep equivalent: quadtree rebuild,
attraction, Barnes-Hut repulsion, gravity, FA2 speed and position update.
``value`` is iterations/s over all ranks, timed with CUDA events on the
library's stream around K replays of the captured step; ``e2e`` times the
same step through gvizCudaForceStepHost with the positions copied from and
back to pinned host memory every step. N > 1 runs independent replicas (the
layout of one graph does not shard across GPUs here), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "ba1m": dict(kind="ba", V=1 << 20, m=4, model=1, theta=0.8, gravity=1.0,
                 radius_base=1.0, radius_per_degree=0.5, overlap=True, box=1000.0, bh=True),
    "grid32": dict(kind="grid", V=1024, model=0, theta=0.5, gravity=0.0, radius_base=0.0,
                   radius_per_degree=0.0, overlap=False, box=1.0, bh=True),
    "er65k_exact": dict(kind="er", V=65536, E=262144, model=0, theta=1.0, gravity=0.0,
                        radius_base=0.0, radius_per_degree=0.0, overlap=False, box=1.0,
                        bh=False),
}
SEED = 7
FLOP_PER_INTERACTION = 20  # pair or pseudo-body term (GPU Gems 3 ch. 31 convention)


def describe(w):
    d = dict(w)
    d["workload"] = {"ba": f"barabasi_albert n={w['V']} m={w.get('m')}",
                     "grid": "grid 32x32", "er": f"erdos_renyi n={w['V']} m={w.get('E')}"}[w["kind"]]
    d["model"] = "linlog" if w["model"] == 1 else "fr"
    return d


def make_edges(w):
    from grapher_b200 import graphs
    if w["kind"] == "ba":
        return graphs.barabasi_albert(w["V"], w["m"], SEED)
    if w["kind"] == "grid":
        return graphs.grid(32, 32)
    return graphs.erdos_renyi(w["V"], w["E"], SEED)


def configure(lay, w):
    lay.set_params(theta=w["theta"], gravityK=w["gravity"], radiusBase=w["radius_base"],
                   radiusPerDegree=w["radius_per_degree"], preventOverlap=int(w["overlap"]),
                   barnesHutEnabled=int(w["bh"]), precision=0)
    lay.box_extent = w["box"]


def initial_positions(w):
    from grapher_b200 import graphs
    if w["kind"] == "er":
        return graphs.unit_disk_positions(w["V"], SEED)
    return graphs.randomize_positions(w["V"], w["box"], SEED)


class ClockSampler:
    """nvidia-smi samples during the timed region (clock and throttle reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# ---------------------------------------------------------------- reference CPU
def reference_layout(w, a, b):
    from oracle.bindings import Reference, make_params
    ref = Reference()
    lay = ref.create_edges(w["V"], a, b, w["model"])
    p = make_params(model=w["model"], theta=w["theta"], bh=w["bh"], gravity=w["gravity"],
                    radius_base=w["radius_base"], radius_per_degree=w["radius_per_degree"],
                    prevent_overlap=w["overlap"])
    lay.configure(p, w["box"])
    lay.begin(SEED)
    if w["kind"] == "er":
        lay.set_positions(initial_positions(w))
    return ref, lay


def cpu_baseline(w, a, b, budget_s=20.0, max_steps=5):
    """The reference's own multithreaded step on this host, a bounded sample."""
    from oracle.bindings import Reference
    if Reference.available():
        ref, lay = reference_layout(w, a, b)
        times = []
        t_start = time.perf_counter()
        while len(times) < max_steps and time.perf_counter() - t_start < budget_s:
            times.append(float(lay.time_steps(1)[0]))
        lay.close()
        v = len(times) / sum(times)
        return {"value": v, "unit": "iters/s", "cores": ref.pool_threads(), "kind": "reference",
                "sample": f"{len(times)} full reference steps (gvizForceEmbedderStep, "
                          f"gvizThreadPool over {ref.pool_threads()} threads) of the same workload"}
    from oracle.bindings import Oracle, make_params
    from grapher_b200 import graphs
    o = Oracle()
    row, col = graphs.to_csr(w["V"], a, b)
    deg = np.diff(row).astype(np.uint64)
    mass = np.ones(w["V"]) if w["model"] == 0 else 1.0 + deg
    p = make_params(model=w["model"], theta=w["theta"], bh=w["bh"], gravity=w["gravity"],
                    radius_base=w["radius_base"], radius_per_degree=w["radius_per_degree"],
                    prevent_overlap=w["overlap"])
    pos = initial_positions(w)
    sf = np.zeros(2 * w["V"])
    ss = np.array([1.0, 1.0])
    t0 = time.perf_counter()
    o.step((row, col), mass, deg, p, pos, sf, ss)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "iters/s", "cores": 1, "kind": "port",
            "sample": "1 step of the single-threaded oracle restatement (reference library absent)"}


def run_reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    a, b = make_edges(w)
    from oracle.bindings import Reference
    if not Reference.available():
        base = cpu_baseline(w, a, b)
        line = {"impl": "reference", "metric": metric_name(w), "value": base["value"],
                "unit": "iters/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                "higher_is_better": True, "config": config_of(w, args), "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "iters/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    ref, lay = reference_layout(w, a, b)
    if args.warmup:
        lay.time_steps(args.warmup)
    t = lay.time_steps(args.steps)
    lay.close()
    v = args.steps / float(t.sum())
    base = {"value": v, "unit": "iters/s", "cores": ref.pool_threads(), "kind": "reference",
            "sample": f"{args.steps} full reference steps after {args.warmup} warm-up steps"}
    line = {"impl": "reference", "metric": metric_name(w), "value": v, "unit": "iters/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(t.mean()), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_of(w, args),
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def metric_name(w):
    return "layout iters/sec"


def config_of(w, args):
    d = describe(w)
    return {"workload": d["workload"], "model": d["model"], "theta": w["theta"],
            "barnes_hut": w["bh"], "gravity": w["gravity"],
            "overlap_radius": (f"{w['radius_base']}*(1+{w['radius_per_degree']}*sqrt(deg))"
                               if w["overlap"] else None),
            "vertices": w["V"], "box_extent": w["box"], "seed": SEED, "precision": "fp32-walk",
            "parallelism": f"replicas{args.gpus}",
            "l2": "per-step working set > L2 (tree rebuilt every step, ~300 MB touched)"}


# ---------------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ba1m", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, w)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from grapher_b200 import ForceLayout, graphs
    a, b = make_edges(w)
    row, col = graphs.to_csr(w["V"], a, b)
    lay = ForceLayout(row, col, model=w["model"], device=local)
    configure(lay, w)
    x0 = initial_positions(w)
    lay.begin(0, positions=x0)
    for _ in range(args.warmup):
        lay.step()

    def barrier():
        if dist:
            dist.barrier()

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    ms = lay.time_steps(args.steps)
    barrier()
    clocks = sampler.stop()
    if dist:
        import torch
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.steps / (ms / 1e3)

    # e2e: host buffers through gvizCudaForceStepHost
    import torch
    V = w["V"]
    pinned = torch.empty(2 * V, dtype=torch.float64, pin_memory=True)
    pinned.numpy()[:] = lay.positions()
    xy = pinned.numpy()
    e2e_steps = max(3, min(args.steps, 50))
    lay.step_host(xy)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        lay.step_host(xy)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * e2e_steps / e2e_s, "unit": "iters/s",
           "h2d_bytes_per_step": 16 * V, "d2h_bytes_per_step": 16 * V + 40,
           "steps": e2e_steps, "timer": "host wall clock around synchronous calls"}

    # per-kernel breakdown and roofline of the dominant kernel
    prof = lay.profile_step()
    kernels = lay.L.gvizCudaForceStepKernelCount(lay.h)
    inter, visits = lay.count_interactions()
    peaks, peak_src = load_peaks()
    walk_ms = dict(prof).get("bh_walk_f32") or dict(prof).get("exact_f32")
    step_ms = sum(t for _, t in prof)
    flops = FLOP_PER_INTERACTION * inter
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    roofline = {"kernel": "bh_walk_f32" if w["bh"] else "exact_f32", "bound": "fp32",
                "achieved": flops / (walk_ms * 1e-3) / 1e12, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": flops / (walk_ms * 1e-3) / 1e12 / fp32_peak,
                "traffic": None,
                "peak_source": "nominal FP32 (148 SM x 128 lanes x 2) at MEASURED_PEAKS sm_max_mhz",
                "algorithmic": f"{FLOP_PER_INTERACTION} FLOP x {inter} interactions per launch",
                "share_of_step": walk_ms / step_ms, "warp_node_visits": visits}

    line = {
        "metric": metric_name(w), "value": value, "unit": "iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_of(w, args), "clocks": clocks, "e2e": e2e,
        "gpu_launches": kernels * args.steps, "kernels_per_step": kernels,
        "vertex_updates_per_s": value * V, "roofline": roofline,
        "kernel_ms": {k: round(v, 4) for k, v in prof}, "peaks": peak_src,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, a, b)
    if rank == 0:
        print(json.dumps(line))
    lay.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
