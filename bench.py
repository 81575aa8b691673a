"""Benchmark of the B200 force-layout step (libgvizcuda).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ba1m_learned|rmat4m_learned|ba1m|batch4096|grid32|er65k_exact
                                |grip_ba200k]

Default workload (the headline metric: learned vs plain Barnes-Hut at equal
force error): Barabasi-Albert graph, n = 1,048,576, m = 4 (4,194,294 edges,
seeded), LinLog with gravity 1.0, start uniform in [-1000, 1000]^2 (rand_r,
seed 7). Setup (untimed, in the FP64 path so that the judged state does not
depend on FP32 rounding): 20 plain steps at theta = 0.5, then four snapshots
of this layout (iterations 20, 25, 30, 30) from which pairs are harvested for
32,768 sampled vertices each at theta = 0.7, 0.95, 1.2 and 1.05; the
far-field MLP is trained on them on the GPU (320 epochs with a step-decayed
learning rate, reported as train_s), and the state of iteration 30 is judged
and timed. Force error is the
normalised RMS of the repulsion against exact FP64 all-pairs repulsion on
every vertex (on 65,536 sampled vertices for layouts above 2^20 vertices),
all configurations judged on the same positions; the error tables also carry
the RMS of the per-vertex relative errors and the largest per-vertex error
over the RMS force.
The plain walk runs at theta = 0.5; the learned walk (the cell-group walk:
one warp per group of <= 32 targets cut from the tree, one network row per
accepted cell) at the largest theta of 1.3, 1.275, ..., 0.6 whose error is
not above the plain walk's. It is judged alone and with hub targets (the
V / 1024 or V / 256 heaviest vertices take the plain monopole walk at
theta = 0.35, since LinLog's force on a vertex scales with its mass); each
at its own largest qualifying theta, the fastest of those that reach
theta = 1.2 (the opening angle the network is meant to stand in for theta =
0.5 at), or the fastest of all when none does (10 timed steps each, from one
saved state), is the learned configuration (--hub-targets fixes the count
instead). ``value`` is the learned path's iterations/s;
the plain path's are in ``plain``. Both are timed from the same saved
layout state.
rmat4m_learned: the same comparison on an R-MAT graph, scale 22 (4,194,304
vertices), 33,554,432 edge draws with (a,b,c,d) = (.57,.19,.19,.05),
deduplicated, no self-loops, start uniform in [-1000, 1000]^2; adds the
error of both paths every 20 iterations over 100 untimed iterations.
ba1m: the same graph with degree-sized prevent-overlap
(r = 1.0 * (1 + 0.5 sqrt(deg))), plain theta = 0.8, FP32 walk.
batch4096: 4096 independent graphs, sizes log-uniform in [32, 8192], each an
Erdos-Renyi graph (mean degree U[3,6]), a random tree or a square grid,
FR theta = 0.7, laid out together in one handle (one step = every graph steps).
grip_ba200k: GRIP refinement rounds at layer 0 (see grip_bench).

A step is one full gvizForceEmbedderStep equivalent: quadtree rebuild,
attraction, Barnes-Hut repulsion, gravity, FA2 speed and position update.
``value`` is iterations/s over all ranks, timed with CUDA events on the
library's stream around K replays of the captured step; ``e2e`` times the
same steps through gvizCudaForceRunHost with the positions copied from and
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

SEED = 7
FLOP_PER_INTERACTION = 20  # pair or pseudo-body term (GPU Gems 3 ch. 31 convention)
MLP_FLOP_PER_ROW = 2 * (10 * 64 + 64 * 64 + 64 * 2)  # one 10-64-64-2 evaluation

SPECS = {
    "ba1m_learned": dict(model=1, theta=0.5, gravity=1.0, radius_base=0.0,
                         radius_per_degree=0.0, overlap=False, bh=True),
    "rmat4m_learned": dict(model=1, theta=0.5, gravity=1.0, radius_base=0.0,
                           radius_per_degree=0.0, overlap=False, bh=True),
    "ba1m": dict(model=1, theta=0.8, gravity=1.0, radius_base=1.0, radius_per_degree=0.5,
                 overlap=True, bh=True),
    "batch4096": dict(model=0, theta=0.7, gravity=0.0, radius_base=0.0,
                      radius_per_degree=0.0, overlap=False, bh=True),
    "grid32": dict(model=0, theta=0.5, gravity=0.0, radius_base=0.0, radius_per_degree=0.0,
                   overlap=False, bh=True),
    "er65k_exact": dict(model=0, theta=1.0, gravity=0.0, radius_base=0.0,
                        radius_per_degree=0.0, overlap=False, bh=False),
}


class Workload:
    """Graphs (edge lists in gvizGraphAddEdge order), their combined CSR and
    the initial positions; one entry per graph of a batch."""

    def __init__(self, name):
        from grapher_b200 import graphs
        self.name = name
        self.spec = SPECS[name]
        self.graphs = []  # (V, a, b, box, seed)
        if name == "rmat4m_learned":
            V = 1 << 22
            a, b = graphs.rmat(22, 1 << 25, 0.57, 0.19, 0.19, SEED)
            self.graphs.append((V, a, b, 1000.0, SEED))
            self.desc = (f"rmat scale=22 draws=33554432 (a,b,c,d)=(.57,.19,.19,.05) "
                         f"deduplicated, edges={len(a)}")
        elif name in ("ba1m", "ba1m_learned"):
            V = 1 << 20
            a, b = graphs.barabasi_albert(V, 4, SEED)
            self.graphs.append((V, a, b, 1000.0, SEED))
            self.desc = f"barabasi_albert n={V} m=4 edges={len(a)}"
        elif name == "grid32":
            a, b = graphs.grid(32, 32)
            self.graphs.append((1024, a, b, 1.0, SEED))
            self.desc = "grid 32x32"
        elif name == "er65k_exact":
            a, b = graphs.erdos_renyi(65536, 262144, SEED)
            self.graphs.append((65536, a, b, None, SEED))
            self.desc = "erdos_renyi n=65536 m=262144, unit disk"
        else:
            rng = np.random.default_rng(SEED)
            for g in range(4096):
                V = int(round(math.exp(rng.uniform(math.log(32), math.log(8192)))))
                kind = int(rng.integers(3))
                if kind == 0:
                    m = int(round(V * rng.uniform(3.0, 6.0) / 2))
                    a, b = graphs.erdos_renyi(V, m, 1000 + g)
                elif kind == 1:
                    a, b = graphs.random_connected(V, 0.0, 1000 + g)
                else:
                    s = max(1, int(round(math.sqrt(V))))
                    V = s * s
                    a, b = graphs.grid(s, s)
                # the embedder's default box (src/embedders/gvizForceEmbedder.c:12-17)
                self.graphs.append((V, a, b, 0.5 * math.sqrt(V) * 10.0, 1000 + g))
            self.desc = "4096 graphs, V log-uniform [32, 8192], ER/random tree/grid"
        self.G = len(self.graphs)
        self.V = int(sum(g[0] for g in self.graphs))
        self._csr = None
        self._x0 = None

    # The combined CSR and the initial positions come from libgvizcuda
    # (gvizCudaEdgesToCsr, gvizCudaRandomizePositions): built on first use,
    # so the reference arm, which never asks for them, does not load it.
    def _build_csr(self):
        from grapher_b200 import graphs
        if self._csr is None:
            if self.G == 1:
                V, a, b, _, _ = self.graphs[0]
                row, col = graphs.to_csr(V, a, b)
                self._csr = (row, col, None)
            else:
                self._csr = graphs.batch([(V, a, b) for V, a, b, _, _ in self.graphs])
        return self._csr

    @property
    def row(self):
        return self._build_csr()[0]

    @property
    def col(self):
        return self._build_csr()[1]

    @property
    def goff(self):
        return self._build_csr()[2]

    @property
    def x0(self):
        from grapher_b200 import graphs
        if self._x0 is None:
            self._x0 = np.concatenate(
                [graphs.unit_disk_positions(V, seed) if box is None
                 else graphs.randomize_positions(V, box, seed)
                 for V, a, b, box, seed in self.graphs])
        return self._x0

    def unit_disk_start(self, g):
        """Initial positions of graph g when it starts in the unit disk
        (numpy only), else None (the reference's own Begin places it)."""
        from grapher_b200 import graphs
        V, _, _, box, seed = self.graphs[g]
        return graphs.unit_disk_positions(V, seed) if box is None else None

    def metric(self):
        """The metric string, the same in both arms."""
        if self.name == "ba1m_learned":
            return "layout iters/sec, 1M-vertex BA graph: learned vs plain BH at equal force error"
        if self.name == "rmat4m_learned":
            return ("layout iters/sec, R-MAT scale-22 graph: learned vs plain BH at equal "
                    "force error")
        return f"layout iters/sec, {self.name}"

    def configure(self, lay):
        s = self.spec
        lay.set_params(theta=s["theta"], gravityK=s["gravity"], radiusBase=s["radius_base"],
                       radiusPerDegree=s["radius_per_degree"], preventOverlap=int(s["overlap"]),
                       barnesHutEnabled=int(s["bh"]), precision=0)

    def oracle_params(self):
        from oracle.bindings import make_params
        s = self.spec
        return make_params(model=s["model"], theta=s["theta"], bh=s["bh"], gravity=s["gravity"],
                           radius_base=s["radius_base"], radius_per_degree=s["radius_per_degree"],
                           prevent_overlap=s["overlap"])

    def config(self, args):
        s = self.spec
        return {"workload": f"{self.name}: {self.desc}", "model": "linlog" if s["model"] else "fr",
                "theta": s["theta"], "barnes_hut": s["bh"], "gravity": s["gravity"],
                "overlap_radius": (f"{s['radius_base']}*(1+{s['radius_per_degree']}*sqrt(deg))"
                                   if s["overlap"] else None),
                "graphs": self.G, "vertices": self.V, "seed": SEED, "precision": "fp32-walk",
                "parallelism": f"replicas{args.gpus}",
                "l2": "per-step working set > L2 (tree rebuilt every step)"}


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
            threading.Thread(target=self._read, daemon=True).start()
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


# DRAM bytes per launch of the dominant kernels (ncu dram__bytes_read.sum +
# dram__bytes_write.sum, one capture each), reported as roofline.traffic on the
# workload the capture ran: kernel -> (workload, bytes, capture)
NCU_TRAFFIC = {
    "bh_walk_f32_learned": ("ba1m_learned", 685.8e6 + 187.2e6,
                            "profiles/learned_walk_ba1m.md (theta 1.225, 1024 hub targets)"),
    "bh_walk_f32": ("ba1m_learned", 613.3e6 + 169.9e6,
                    "profiles/plain_walk_ba1m.md (theta 0.5)"),
    "exact_f32": ("er65k_exact", 1.356e6 + 0.0, "profiles/exact_er65k.md"),
    "k_grip_pass1": ("grip_ba200k", 121.1e6 + 8.4e6, "profiles/grip_round_ba200k.md"),
}


def ncu_traffic(kernel, workload):
    """(bytes per launch, capture) from NCU_TRAFFIC when the capture ran this
    workload, else (None, None)."""
    t = NCU_TRAFFIC.get(kernel)
    if t is None or t[0] != workload:
        return None, None
    return t[1], t[2]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# ---------------------------------------------------------------- reference CPU
def reference_graph(w, g):
    """The reference embedder for graph g of the workload, begun."""
    from oracle.bindings import Reference
    ref = Reference()
    V, a, b, box, seed = w.graphs[g]
    lay = ref.create_edges(V, a, b, w.spec["model"])
    lay.configure(w.oracle_params(), box if box else 0.0)
    lay.begin(seed)
    start = w.unit_disk_start(g)
    if start is not None:
        lay.set_positions(start)
    return ref, lay


def reference_iteration_time(w, budget_s=20.0, max_steps=5):
    """Seconds per iteration of the whole workload for the reference's own
    multithreaded step (one embedder per graph, as gviz runs them), from a
    bounded sample: up to max_steps steps, or for a batch the first graphs
    until the budget is spent, scaled by vertex count to the whole batch."""
    from oracle.bindings import Reference
    t_start = time.perf_counter()
    if w.G == 1:
        ref, lay = reference_graph(w, 0)
        times = []
        while len(times) < max_steps and time.perf_counter() - t_start < budget_s:
            times.append(float(lay.time_steps(1)[0]))
        lay.close()
        return float(np.mean(times)), ref.pool_threads(), (
            f"{len(times)} full reference steps (gvizForceEmbedderStep, gvizThreadPool over "
            f"{ref.pool_threads()} threads) of the same workload")
    total, sampled_v, n = 0.0, 0, 0
    threads = Reference().pool_threads()
    while n < w.G and time.perf_counter() - t_start < budget_s:
        _, lay = reference_graph(w, n)
        total += float(np.mean(lay.time_steps(3)))
        sampled_v += w.graphs[n][0]
        lay.close()
        n += 1
    return total * w.V / sampled_v, threads, (
        f"first {n} of {w.G} graphs, 3 reference steps each (one embedder per graph, "
        f"gvizThreadPool over {threads} threads), scaled by vertex count to the batch")


def cpu_baseline(w):
    from oracle.bindings import Reference
    if Reference.available():
        t, cores, sample = reference_iteration_time(w)
        return {"value": 1.0 / t, "unit": "iters/s", "cores": cores, "kind": "reference",
                "cpu_model": cpu_model(), "sample": sample}
    from oracle.bindings import Oracle
    o = Oracle()
    V, a, b, box, seed = w.graphs[0]
    row, col = csr_numpy(V, a, b)
    deg = np.diff(row).astype(np.uint64)
    mass = np.ones(V) if w.spec["model"] == 0 else 1.0 + deg
    start = w.unit_disk_start(0)
    pos = start.copy() if start is not None else rand_r_positions(V, box, seed)
    sf, ss = np.zeros(2 * V), np.array([1.0, 1.0])
    t0 = time.perf_counter()
    o.step((row, col), mass, deg, w.oracle_params(), pos, sf, ss)
    t = (time.perf_counter() - t0) * w.V / V
    return {"value": 1.0 / t, "unit": "iters/s", "cores": 1, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": "1 step of the single-thread oracle on the first graph, scaled by vertex "
                      "count (reference library absent)"}


def csr_numpy(V, a, b):
    """Adjacency as gvizGraphAddEdge builds it (edge (a,b) appends b to a's
    list and a to b's, in edge order), with numpy alone."""
    src = np.empty(2 * len(a), np.int64)
    dst = np.empty(2 * len(a), np.uint32)
    src[0::2], src[1::2] = a, b
    dst[0::2], dst[1::2] = b, a
    order = np.argsort(src, kind="stable")
    row = np.zeros(V + 1, np.uint64)
    np.cumsum(np.bincount(src, minlength=V), out=row[1:])
    return row, np.ascontiguousarray(dst[order])


def rand_r_positions(V, box, seed):
    """The reference's Begin placement (libc rand_r, x then y per vertex),
    through the C library directly."""
    import ctypes
    libc = ctypes.CDLL(None)
    st = ctypes.c_uint(seed)
    r = np.array([libc.rand_r(ctypes.byref(st)) for _ in range(2 * V)], np.float64)
    return box * (2.0 * (r / (2147483647.0 + 1.0)) - 1.0)


def cpu_model():
    """The host CPU's model name and the logical CPUs online."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return f"{name}, {os.cpu_count()} logical CPUs"


def run_reference_arm(args, w):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from oracle.bindings import Reference
    line = {"impl": "reference", "metric": w.metric(), "unit": "iters/s",
            "n_gpus": args.gpus, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": w.config(args)}
    if Reference.available() and w.G == 1:
        ref, lay = reference_graph(w, 0)
        if args.warmup:
            lay.time_steps(args.warmup)
        t = lay.time_steps(args.steps)
        lay.close()
        v = args.steps / float(t.sum())
        line.update(steps=args.steps, warmup=args.warmup, ms_per_step=1e3 * float(t.mean()))
        base = {"value": v, "unit": "iters/s", "cores": ref.pool_threads(), "kind": "reference",
                "cpu_model": cpu_model(),
                "sample": f"{args.steps} full reference steps after {args.warmup} warm-up steps"}
    else:
        base = cpu_baseline(w)
        v = base["value"]
        line.update(steps=1, warmup=0)
    line.update(value=v, cpu_baseline=base,
                e2e={"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": 0})
    print(json.dumps(line))
    return 0


class nvtx_range:
    """NVTX range around a timed region, so that a profiler can be limited
    to it (ncu --nvtx --nvtx-include <name>/)."""

    def __init__(self, name):
        self.name = name

    def __enter__(self):
        import torch
        torch.cuda.nvtx.range_push(self.name)

    def __exit__(self, *exc):
        import torch
        torch.cuda.nvtx.range_pop()


def reduce_max(x, dist=None, device="cpu"):
    """The maximum of x over all ranks (x itself without a process group)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ms_max, steps, world):
    """Whole-job iterations/s of `world` replicas that each ran `steps`
    steps, the slowest in ms_max milliseconds."""
    return world * steps / (ms_max / 1e3)


# ------------------------------------------------------------ learned setup
LEARNED_THETAS = tuple(round(1.3 - 0.025 * i, 3) for i in range(29))  # 1.3, 1.275 ... 0.6
LEARNED_SPREAD = 1.0
LEARNED_CELL_GROUPS = 1  # the cell-group walk: one warp per tree-cut group of <= 32 targets
HUB_SHARES = (1024, 256)  # hub-target candidates: the V / share heaviest vertices
HUB_THETA = 0.35         # their plain walk's opening threshold
TARGET_THETA = 1.2       # candidates reaching it are preferred (see pick_candidate)
HARVEST_TARGETS = 32768  # sampled target vertices per training snapshot
# Adam passes over the harvested pairs as (epochs, learning rate): a step
# decay; the optimiser's moments carry over from one stage to the next
TRAIN_SCHEDULE = ((192, 2e-3), (80, 6e-4), (48, 2e-4))
# The learned comparison starts from a fixed point of the layout, whatever
# --warmup asks for: LEARNED_PRE_STEPS plain steps from the initial
# positions, then the harvest snapshots of HARVEST_SCHEDULE, all in the FP64
# path; the judged and timed state is the one of the last snapshot. --warmup
# steps run before each timed region, from that saved state.
LEARNED_PRE_STEPS = 20
# (steps before the snapshot, opening threshold of its pairs): earlier
# states at smaller thresholds, and the state the learned walk then runs
# from at the large ones it is meant for (the network fits the layout it is
# trained on; the judge checks it on every vertex of that state)
HARVEST_SCHEDULE = ((0, 0.7), (5, 0.95), (5, 1.2), (0, 1.05))
JUDGE_VERTICES = 65536
JUDGE_ALL_MAX = 1 << 20  # layouts up to this size are judged on every vertex
JUDGE_CHUNK = 262144     # targets per exact FP64 repulsion call
CHOICE_STEPS = 10        # timed steps per candidate when choosing the learned config


def force_error(lay, targets, exact):
    """Error of the current repulsion on the judged targets: the normalised
    RMS (the metric's error), the RMS of the per-vertex relative errors and
    the largest per-vertex error relative to the RMS force."""
    rep = lay.repulsion()[targets]
    d = np.linalg.norm(rep - exact, axis=1)
    n = np.linalg.norm(exact, axis=1)
    rms_force = float(np.sqrt(np.mean(n * n)))
    return (float(np.sqrt(np.sum(d * d) / np.sum(n * n))),
            float(np.sqrt(np.mean((d / np.maximum(n, 1e-300)) ** 2))),
            float(np.max(d) / max(rms_force, 1e-300)))


def error_entry(e):
    return {"rms_err": e[0], "rms_rel_err_per_vertex": e[1], "max_err_over_rms_force": e[2]}


def learned_params(linfo):
    """set_params arguments of the chosen learned configuration."""
    return dict(theta=linfo["learned_theta"], farField=1, farGroupSpread=LEARNED_SPREAD,
                farCellGroups=LEARNED_CELL_GROUPS, farHubTargets=linfo["hub_targets"],
                farHubTheta=HUB_THETA)


def setup_steps(lay, n):
    """n untimed steps of the learned setup in the FP64 path (the reference's
    arithmetic), so that the state the comparison judges and times does not
    move with the FP32 kernels' rounding; the FP32 path is restored after."""
    if n <= 0:
        return
    lay.set_params(precision=1)
    for _ in range(n):
        lay.step()
    lay.set_params(precision=0)


def pick_candidate(cands):
    """Hub-target count of the learned configuration: among the candidates
    (each at its own largest qualifying theta) the fastest of those that
    reach TARGET_THETA, or the fastest of all when none does."""
    at_target = [c for c in cands if c["theta"] >= TARGET_THETA - 1e-9]
    return min(at_target or cands, key=lambda c: c["ms_per_step"])["hub_targets"]


def learned_setup(lay, w, reduce=lambda x: x, hub_targets="auto"):
    """Trains the far-field MLP on this layout's own harvested pairs, judges
    plain theta = 0.5 and the learned walk, without and with hub targets,
    against exact FP64 repulsion on the same positions, and picks the
    learned configuration (see the module text). `reduce` takes the maximum
    of a time over ranks, so that every rank picks the same one;
    `hub_targets` other than "auto" fixes the hub count instead."""
    from grapher_b200.farfield import FarFieldModel, harvest_training_set
    rng = np.random.default_rng(SEED)
    t0 = time.perf_counter()
    Xs, Ts, Ws = [], [], []
    for snap, (gap, th) in enumerate(HARVEST_SCHEDULE):  # cells of every angular size
        setup_steps(lay, gap)
        t = np.sort(rng.choice(w.V, HARVEST_TARGETS, replace=False)).astype(np.uint32)
        X, T, Wt = harvest_training_set(lay, th, t)
        Xs.append(X), Ts.append(T), Ws.append(Wt)
    model = FarFieldModel(seed=SEED)
    X, T, Wt = np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ws)
    losses = np.concatenate([model.train(X, T, Wt, epochs=ep, batch=4096, lr=lr, seed=SEED + i)
                             for i, (ep, lr) in enumerate(TRAIN_SCHEDULE)])
    train_s = time.perf_counter() - t0
    if w.V <= JUDGE_ALL_MAX:
        targets = np.arange(w.V, dtype=np.uint32)
    else:
        targets = np.sort(rng.choice(w.V, JUDGE_VERTICES, replace=False)).astype(np.uint32)
    exact = np.concatenate([lay.exact_repulsion(targets[i:i + JUDGE_CHUNK])
                            for i in range(0, len(targets), JUDGE_CHUNK)])
    lay.set_params(theta=w.spec["theta"], farField=0)
    e_plain, e_plain_pv, e_plain_max = force_error(lay, targets, exact)
    model.attach(lay)
    fixed = hub_targets != "auto"
    counts = sorted({0, min(int(hub_targets), w.V)} if fixed else
                    {0} | {w.V // share for share in HUB_SHARES})
    tables, picks = {}, {}
    for k in counts:
        table, pick = {}, None
        for th in LEARNED_THETAS:
            lay.set_params(theta=th, farField=1, farGroupSpread=LEARNED_SPREAD,
                           farCellGroups=LEARNED_CELL_GROUPS, farHubTargets=k,
                           farHubTheta=HUB_THETA)
            err = force_error(lay, targets, exact)
            table[str(th)] = error_entry(err)
            if pick is None and err[0] <= e_plain:
                pick = th
        tables[k], picks[k] = table, (pick if pick is not None else LEARNED_THETAS[-1])
    # the faster of the two qualifying configurations, from the same state
    x_s, fa2_s = lay.positions(), lay.fa2_state()
    times = {}
    for k in counts:
        lay.set_params(theta=picks[k], farField=1, farGroupSpread=LEARNED_SPREAD,
                       farCellGroups=LEARNED_CELL_GROUPS, farHubTargets=k, farHubTheta=HUB_THETA)
        lay.time_steps(3)
        times[k] = reduce(lay.time_steps(CHOICE_STEPS)) / CHOICE_STEPS
        lay.set_positions(x_s)
        lay.set_fa2_state(*fa2_s)
    k_best = counts[-1] if fixed else pick_candidate(
        [{"hub_targets": k, "theta": picks[k], "ms_per_step": times[k]} for k in counts])
    chosen, table = picks[k_best], tables[k_best]
    lay.set_params(theta=w.spec["theta"], farField=0, farCellGroups=0, farHubTargets=0)
    plain_table = {}
    for th in (0.3, 0.4, 0.5, 0.6, 0.8, 1.0, 1.2):
        lay.set_params(theta=th)
        plain_table[str(th)] = error_entry(force_error(lay, targets, exact))
    lay.set_params(theta=w.spec["theta"])
    info = {"train_s": train_s, "train_pairs": int(sum(len(x) for x in Xs)),
            "train_loss_first_last": [float(losses[0]), float(losses[-1])],
            "judge_vertices": int(len(targets)), "plain_rms_err": e_plain,
            "plain_rms_rel_err_per_vertex": e_plain_pv,
            "plain_max_err_over_rms_force": e_plain_max, "learned_theta": chosen,
            "hub_targets": k_best, "hub_theta": HUB_THETA,
            "learned_errors": table, "plain_errors": plain_table,
            "hub_choice": "fixed" if fixed else "auto",
            "candidates": [{"hub_targets": k, "theta": picks[k], "ms_per_step": times[k],
                            "rms_err": tables[k][str(picks[k])]["rms_err"]} for k in counts],
            "learned_errors_by_hub_targets": {str(k): tables[k] for k in counts},
            "group_spread": LEARNED_SPREAD,
            "walk": "cell groups" if LEARNED_CELL_GROUPS else "per target"}
    return model, info


def error_trajectory(lay, w, linfo, chunks=5, every=20):
    """Normalised RMS force error of the learned and the plain walk every
    `every` iterations along `chunks` x `every` iterations from one state."""
    rng = np.random.default_rng(SEED + 1)
    targets = np.sort(rng.choice(w.V, min(JUDGE_VERTICES, w.V), replace=False)).astype(np.uint32)
    x_s, (sf_s, sp_s, ef_s) = lay.positions(), lay.fa2_state()
    out = {}
    for name, th, ff in (("learned", linfo["learned_theta"], 1), ("plain", w.spec["theta"], 0)):
        lay.set_positions(x_s)
        lay.set_fa2_state(sf_s, sp_s, ef_s)
        lay.set_params(**(learned_params(linfo) if ff else
                          dict(theta=th, farField=0, farCellGroups=0, farHubTargets=0)))
        errs = []
        for c in range(chunks):
            lay.time_steps(every)
            exact = lay.exact_repulsion(targets)
            errs.append(force_error(lay, targets, exact)[0])
        out[name] = {"theta": th, "iterations": [every * (c + 1) for c in range(chunks)],
                     "rms_err": errs}
    lay.set_params(**learned_params(linfo))
    return out


# ----------------------------------------------------------- precision reports
STRESS_SOURCES = 16
JUDGE_SAMPLE = 65536


def layout_stress(row, col, xy, sources=STRESS_SOURCES, seed=SEED):
    """Normalised stress of a layout at its best scale, over the pairs
    (source, vertex) of `sources` seeded breadth-first sources:
    min_s mean((s |x_i - x_j| - d_ij)^2 / d_ij^2) = 1 - A1^2 / (n A2) with
    A1 = sum e/d, A2 = sum (e/d)^2 over the n reachable pairs."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import shortest_path
    V = len(row) - 1
    A = sp.csr_matrix((np.ones(len(col), np.float32), np.asarray(col, np.int64),
                       np.asarray(row, np.int64)), shape=(V, V))
    rng = np.random.default_rng(seed)
    src = rng.choice(V, min(sources, V), replace=False)
    D = shortest_path(A, method="D", unweighted=True, indices=src)
    p = np.asarray(xy).reshape(-1, 2)
    a1 = a2 = 0.0
    n = 0
    for i, s0 in enumerate(src):
        d = D[i]
        m = np.isfinite(d) & (d > 0)
        r = np.linalg.norm(p[m] - p[s0], axis=1) / d[m]
        a1 += float(r.sum())
        a2 += float((r * r).sum())
        n += int(m.sum())
    return float(1.0 - a1 * a1 / (n * a2)) if n and a2 > 0 else None


def vector_error(a, b):
    """Error of per-vertex vectors a against b: normalised RMS over all
    vertices, RMS and maximum of the per-vertex relative errors."""
    a = np.asarray(a).reshape(-1, 2)
    b = np.asarray(b).reshape(-1, 2)
    d = np.linalg.norm(a - b, axis=1)
    n = np.linalg.norm(b, axis=1)
    rel = d / np.maximum(n, 1e-300)
    return {"rms_err": float(np.sqrt(np.sum(d * d) / max(np.sum(n * n), 1e-300))),
            "rms_rel_err_per_vertex": float(np.sqrt(np.mean(rel * rel))),
            "max_rel_err_per_vertex": float(rel.max())}


def run_from(lay, x0, steps, precision, strict=0):
    """Positions after `steps` steps from x0 (FA2 state reset, as Begin),
    and the device time of the steps."""
    lay.set_params(precision=precision, strictReductions=strict)
    lay.set_positions(x0)
    lay.set_fa2_state(np.zeros(2 * lay.V), 1.0, 1.0)
    ms = lay.time_steps(steps) if steps else 0.0
    return lay.positions(), ms


def precision_report(lay, w, args):
    """FP32 GPU against FP64 GPU (and the reference's CPU step where the CPU
    baseline leg runs) on this workload: per-vertex force errors, free-run
    drift and final-layout stress. Untimed; the layout is left at its state."""
    x_s, (sf_s, sp_s, ef_s) = lay.positions(), lay.fa2_state()
    rng = np.random.default_rng(SEED + 2)
    out = {}
    if w.name == "ba1m":
        t = np.sort(rng.choice(w.V, min(JUDGE_SAMPLE, w.V), replace=False)).astype(np.uint32)
        exact = lay.exact_repulsion(t)
        lay.set_params(precision=0)
        r32 = lay.repulsion()[t]
        lay.set_params(precision=1)
        r64 = lay.repulsion()[t]
        out["forces"] = {"sample": f"{len(t)} seeded vertices, at the timed state",
                         "fp32_bh_vs_fp64_bh": vector_error(r32, r64),
                         "fp32_bh_vs_exact_fp64": vector_error(r32, exact),
                         "fp64_bh_vs_exact_fp64": vector_error(r64, exact)}
        iters = 200
    elif w.name == "er65k_exact":
        lay.set_params(precision=0)
        r32 = lay.repulsion()
        lay.set_params(precision=1)
        r64 = lay.repulsion()
        out["forces"] = {"sample": f"all {w.V} vertices, at the timed state",
                         "fp32_kahan_exact_vs_fp64_exact": vector_error(r32, r64)}
        iters = 100
    else:  # grid32
        iters = 500
    x0 = w.x0
    xy32, ms32 = run_from(lay, x0, iters, 0)
    xy64, ms64 = run_from(lay, x0, iters, 1, strict=1 if w.name == "grid32" else 0)
    ext = float(np.abs(xy64).max())
    dr = np.linalg.norm((xy32 - xy64).reshape(-1, 2), axis=1) / max(ext, 1e-300)
    out["free_run"] = {
        "iterations": iters, "from": "the initial positions",
        "fp32_vs_fp64_drift_over_extent": {"median": float(np.median(dr)),
                                           "max": float(dr.max())},
        "fp64_ms_per_step": ms64 / iters, "fp32_ms_per_step": ms32 / iters,
        "stress": {"initial": layout_stress(w.row, w.col, x0),
                   "fp32": layout_stress(w.row, w.col, xy32),
                   "fp64": layout_stress(w.row, w.col, xy64),
                   "sources": STRESS_SOURCES}}
    if not args.no_cpu_baseline:
        out["reference"] = reference_comparison(lay, w, iters)
    lay.set_params(precision=0, strictReductions=0)
    lay.set_positions(x_s)
    lay.set_fa2_state(sf_s, sp_s, ef_s)
    return out


def reference_comparison(lay, w, iters):
    """The reference's own CPU step (oracle/_ref, the CPU baseline's
    library) against the GPU paths, free-running from the same Begin: every
    iteration of the 32x32 grid; for larger layouts the first steps only
    (the CPU step takes seconds there)."""
    from oracle.bindings import Reference
    if not Reference.available():
        return None
    ref, rl = reference_graph(w, 0)
    x0 = rl.positions()
    n = iters if w.V <= 4096 else 2
    marks = sorted({1, 2, 10, 50, 100, 200, 500} & set(range(1, n + 1)))
    res = {"steps": n, "threads": ref.pool_threads(), "at": marks}
    refpos = {}
    for s in range(1, n + 1):
        rl.step()
        if s in marks:
            refpos[s] = rl.positions()
    rl.close()
    for name, prec, strict in (("fp64", 1, 1), ("fp32", 0, 0)):
        lay.set_params(precision=prec, strictReductions=strict)
        lay.set_positions(x0)
        lay.set_fa2_state(np.zeros(2 * lay.V), 1.0, 1.0)
        drift = []
        for s in range(1, n + 1):
            lay.step()
            if s in marks:
                p, q = lay.positions(), refpos[s]
                ext = max(float(np.abs(q).max()), 1e-300)
                d = np.linalg.norm((p - q).reshape(-1, 2), axis=1) / ext
                drift.append({"iteration": s, "median": float(np.median(d)),
                              "max": float(d.max())})
        res[name] = drift
        if n == iters:
            res[name + "_stress"] = layout_stress(w.row, w.col, lay.positions())
    if n == iters:
        res["reference_stress"] = layout_stress(w.row, w.col, refpos[n])
    return res


# ---------------------------------------------------------------------- GRIP
GRIP_V, GRIP_M, GRIP_K = 200_000, 3, 128


def grip_graph():
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(GRIP_V, GRIP_M, SEED)
    row, col = graphs.to_csr(GRIP_V, a, b)
    return a, b, row, col


def grip_reference_rounds(a, b, max_rounds, budget_s=20.0):
    """Seconds per round of the reference's own GRIP (pooled, as it runs by
    default) at layer 0 of its pipeline on the same graph, and its threads."""
    from oracle.bindings import Reference
    ref = Reference()
    rg = ref.create_grip(GRIP_V, a, b, serial=False)
    rg.begin()
    while rg.layer > 0:
        rg.next_stage()
    rg.refine()  # warm-up
    times = []
    t_start = time.perf_counter()
    while len(times) < max_rounds and time.perf_counter() - t_start < budget_s:
        t0 = time.perf_counter()
        rg.refine()
        times.append(time.perf_counter() - t0)
    rg.close()
    return float(np.mean(times)), ref.pool_threads(), len(times)


def grip_bench(args):
    """GRIP refinement rounds at layer 0 (every vertex active): BA
    n = 200,000, m = 3, k = 128 nearest by graph distance, positions uniform
    in [-1000, 1000]^2. value = rounds/s on the device; e2e = rounds with the
    positions copied from and back to host memory every round."""
    a, b, row, col = grip_graph()
    metric = "GRIP refinement rounds/sec, layer 0"
    config = {"workload": f"grip_ba200k: barabasi_albert n={GRIP_V} m={GRIP_M} "
                          f"edges={len(a)}, layer 0, k={GRIP_K}",
              "precision": "fp64", "parallelism": "replicas1",
              "l2": "positions fit in L2; k-nearest lists (200 MB) do not"}
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        t, cores, n = grip_reference_rounds(a, b, max(args.steps, 1))
        base = {"value": 1.0 / t, "unit": "rounds/s", "cores": cores, "kind": "reference",
                "sample": f"{n} rounds of the reference's GRIP (gvizGRIPEmbedderRefineRound, "
                          f"gvizThreadPool over {cores} threads) at layer 0 of its own pipeline"}
        print(json.dumps({"impl": "reference", "metric": metric, "value": base["value"],
                          "unit": "rounds/s", "n_gpus": args.gpus, "steps": n, "warmup": 1,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic", "config": config,
                          "cpu_baseline": base,
                          "e2e": {"value": base["value"], "unit": "rounds/s",
                                  "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0
    from grapher_b200 import graphs
    from grapher_b200.grip import GripRefiner, k_nearest
    local = int(os.environ.get("LOCAL_RANK", "0"))
    act = np.arange(GRIP_V, dtype=np.uint32)
    off, kv, kd = k_nearest(row, col, act, GRIP_K)
    x0 = graphs.randomize_positions(GRIP_V, 1000.0, SEED)
    g = GripRefiner(row, col, device=local)
    g.set_positions(x0)
    g.set_layer(0, act, off, kv, kd)
    g.time_rounds(args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    ms, fms = g.time_rounds(args.steps)
    clocks = sampler.stop()
    value = args.steps / (ms / 1e3)
    # e2e through the C ABI with host positions every round
    import torch
    pinned = torch.empty(2 * GRIP_V, dtype=torch.float64, pin_memory=True)
    pinned.numpy()[:] = g.positions()
    xy = pinned.numpy()
    n_e2e = max(3, min(args.steps, 50))
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        g.set_positions(xy)
        g.refine_round()
        xy[:] = g.positions()
    e2e_s = time.perf_counter() - t0
    # force kernel: algorithmic bytes per launch
    E2, K = int(row[-1]), int(off[-1])
    per_vertex = 8 + 16 + 4 + 16 + 16 + 16 + 16 + 16 + 8 + 2  # offsets, row, id, state
    bytes_launch = GRIP_V * per_vertex + K * (4 + 4 + 16) + E2 * (4 + 16)
    fwd_ms = fms / args.steps
    peaks, src = load_peaks()
    achieved = bytes_launch / (fwd_ms * 1e-3) / 1e9
    line = {
        "metric": metric, "value": value, "unit": "rounds/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config, "clocks": clocks,
        "e2e": {"value": n_e2e / e2e_s, "unit": "rounds/s", "h2d_bytes_per_step": 16 * GRIP_V,
                "d2h_bytes_per_step": 16 * GRIP_V + 32, "steps": n_e2e,
                "timer": "host wall clock around synchronous calls"},
        "gpu_launches": 5 * args.steps, "kernels_per_step": 5,
        "roofline": {"kernel": "k_grip_pass1", "bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "traffic": ncu_traffic("k_grip_pass1", "grip_ba200k")[0],
                     "traffic_source": ncu_traffic("k_grip_pass1", "grip_ba200k")[1],
                     "peak_source": f"hbm_gbs ({src})",
                     "algorithmic": (f"{bytes_launch} B per launch: {GRIP_V} vertices x "
                                     f"{per_vertex} B + {K} nearest x 24 B + {E2} edge "
                                     "entries x 20 B (the gathered positions mostly hit L2)"),
                     "share_of_step": fms / ms},
        "knn_entries": K, "peaks": src,
    }
    if not args.no_cpu_baseline:
        t, cores, n = grip_reference_rounds(a, b, 10)
        line["cpu_baseline"] = {"value": 1.0 / t, "unit": "rounds/s", "cores": cores,
                                "kind": "reference",
                                "sample": f"{n} rounds of the reference's GRIP at layer 0 of its "
                                          f"own pipeline on the same graph, gvizThreadPool over "
                                          f"{cores} threads"}
    g.close()
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ba1m_learned", choices=sorted(SPECS) + ["grip_ba200k"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--hub-targets", default="auto",
                    help="learned workloads: hub targets of the learned walk; 'auto' (default) "
                         "times 0, V/1024 and V/256 at their own largest qualifying theta and "
                         "keeps the fastest, a number fixes the count")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload == "grip_ba200k":
        return grip_bench(args)
    w = Workload(args.workload)
    learned = args.workload in ("ba1m_learned", "rmat4m_learned")
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

    from grapher_b200 import ForceLayout
    lay = ForceLayout(w.row, w.col, model=w.spec["model"], graph_offsets=w.goff, device=local)
    w.configure(lay)
    lay.begin(0, positions=w.x0)
    if learned:
        setup_steps(lay, LEARNED_PRE_STEPS)
    else:
        for _ in range(args.warmup):
            lay.step()
    # the walk's launch shape for this layout (block size, static or
    # persistent schedule), timed on the warmed-up positions
    shape = lay.autotune() if w.spec["bh"] else None

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, dist, f"cuda:{local}")

    model, linfo, plain_line = None, None, None
    if learned:
        model, linfo = learned_setup(lay, w, max_over_ranks, args.hub_targets)
        x_s, (sf_s, sp_s, ef_s) = lay.positions(), lay.fa2_state()
        # plain theta = 0.5 from the saved state
        lay.set_params(theta=w.spec["theta"], farField=0)
        lay.time_steps(args.warmup)
        lay.set_positions(x_s)
        lay.set_fa2_state(sf_s, sp_s, ef_s)
        barrier()
        with nvtx_range("plain_steps"):
            pms = max_over_ranks(lay.time_steps(args.steps))
        pprof = lay.profile_step()
        p_inter, p_visits = lay.count_interactions()
        p_walk = dict(pprof).get("bh_walk_f32")
        fp32_peak = 148 * 128 * 2 * load_peaks()[0].get("sm_max_mhz", 1965.0) * 1e6 / 1e12
        plain_line = {"theta": w.spec["theta"], "value": world * args.steps / (pms / 1e3),
                      "ms_per_step": pms / args.steps, "rms_err": linfo["plain_rms_err"],
                      "kernel_ms": {k: round(v, 4) for k, v in pprof},
                      "interactions": p_inter, "warp_node_visits": p_visits,
                      "walk_fp32_frac": (FLOP_PER_INTERACTION * p_inter / (p_walk * 1e-3) / 1e12
                                         / fp32_peak) if p_walk else None,
                      "walk_traffic": ncu_traffic("bh_walk_f32", args.workload)[0]}
        # then the learned walk from the same state
        lay.set_positions(x_s)
        lay.set_fa2_state(sf_s, sp_s, ef_s)
        lay.set_params(**learned_params(linfo))
        lay.time_steps(args.warmup)
        lay.set_positions(x_s)
        lay.set_fa2_state(sf_s, sp_s, ef_s)

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    with nvtx_range("learned_steps" if learned else "timed_steps"):
        ms = lay.time_steps(args.steps)
    barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(ms)
    value = replica_value(ms, args.steps, world)

    # e2e: host buffers through gvizCudaForceRunHost (every step uploads the
    # positions from page-locked host memory and reads the new ones back)
    import torch
    V = w.V
    pinned = torch.empty(2 * V, dtype=torch.float64, pin_memory=True)
    pinned.numpy()[:] = lay.positions()
    xy = pinned.numpy()
    e2e_steps = max(3, min(args.steps, 50))
    lay.run_host(xy, 1)
    barrier()
    t0 = time.perf_counter()
    lay.run_host(xy, e2e_steps)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * e2e_steps / e2e_s, "unit": "iters/s",
           "h2d_bytes_per_step": 16 * V, "d2h_bytes_per_step": 16 * V,
           "steps": e2e_steps,
           "timer": "host wall clock around one gvizCudaForceRunHost call of `steps` steps: "
                    "positions to the device before and back after every step, the copies "
                    "of consecutive steps pipelined; step stats read once at the end"}

    # per-kernel breakdown and roofline of the dominant kernel
    prof = lay.profile_step()
    kernels = lay.L.gvizCudaForceStepKernelCount(lay.h)
    inter, visits = lay.count_interactions()
    peaks, peak_src = load_peaks()
    pd = dict(prof)
    kname = ("bh_walk_f32_learned" if learned else "bh_walk_f32") if w.spec["bh"] else "exact_f32"
    walk_ms = pd.get(kname)
    step_ms = sum(t for _, t in prof)
    flops = FLOP_PER_INTERACTION * inter
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved = flops / (walk_ms * 1e-3) / 1e12
    traffic, traffic_src = ncu_traffic(kname, args.workload)
    roofline = {"kernel": kname, "bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
                "traffic_source": traffic_src,
                "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 FLOP) at the "
                               "MEASURED_PEAKS.json max SM clock (no measured FP32 figure)",
                "algorithmic": f"{FLOP_PER_INTERACTION} FLOP x {inter} interactions per launch",
                "share_of_step": walk_ms / step_ms, "warp_node_visits": visits}
    if learned:
        g_rows, l_rows = lay.count_far_rows()
        rows = g_rows + l_rows
        mlp_flop = MLP_FLOP_PER_ROW * rows
        tc = mlp_flop / (walk_ms * 1e-3) / 1e12
        roofline = {"kernel": kname, "bound": "tensor", "achieved": tc,
                    "peak": peaks.get("bf16_tflops", 1590.0), "unit": "TFLOP/s",
                    "frac": tc / peaks.get("bf16_tflops", 1590.0), "traffic": traffic,
                    "traffic_source": traffic_src,
                    "peak_source": f"bf16_tflops ({peak_src})",
                    "algorithmic": (f"{MLP_FLOP_PER_ROW} FLOP (10-64-64-2 MLP) x {rows} rows "
                                    f"({g_rows} shared, {l_rows} per target) per launch"),
                    "share_of_step": walk_ms / step_ms, "warp_node_visits": visits,
                    "fp32_view": {"achieved": achieved, "peak": fp32_peak,
                                  "frac": achieved / fp32_peak,
                                  "algorithmic": f"{FLOP_PER_INTERACTION} FLOP x {inter} "
                                                 "monopole/pair interactions per launch"}}

    line = {
        "metric": w.metric(), "value": value, "unit": "iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": w.config(args), "clocks": clocks, "e2e": e2e,
        "gpu_launches": kernels * args.steps, "kernels_per_step": kernels,
        "vertex_updates_per_s": value * V, "roofline": roofline,
        "kernel_ms": {k: round(v, 4) for k, v in prof}, "peaks": peak_src,
    }
    if shape:
        line["walk_shape"] = {"threads": shape[0], "persistent": shape[1],
                              "stack_entries": lay.walk_shape()[2],
                              "autotune_walk_ms": round(shape[2], 4)}
    if learned and args.workload == "rmat4m_learned":
        # the error along the run, every 20 iterations, for both paths from
        # the state after the timed steps (untimed)
        line["error_every_20"] = error_trajectory(lay, w, linfo)
    if learned:
        line["learned"] = dict(linfo, value=value, theta=linfo["learned_theta"],
                               rms_err=linfo["learned_errors"][str(linfo["learned_theta"])]["rms_err"])
        line["plain"] = plain_line
        line["config"]["theta"] = {"plain": w.spec["theta"], "learned": linfo["learned_theta"]}
        line["config"]["hub_targets"] = linfo["hub_targets"]
    if rank == 0 and world == 1 and w.name in ("ba1m", "er65k_exact", "grid32"):
        line["precision"] = precision_report(lay, w, args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w)
    if rank == 0:
        print(json.dumps(line))
    lay.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
