"""ForceLayout: Python mirror of the gvizForceEmbedder API over libgvizcuda.

Method names and argument meaning follow include/embedders/gvizForceEmbedder.h
(Configure* with "0 keeps the current value" where the reference does that,
Begin(seed) placing vertices with the reference's rand_r stream, Step
returning maxDisp, Run returning the round count or -1 before Begin). All the
work happens in the CUDA library; this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N


def default_box_extent(vertex_count: int, edge_length: float) -> float:
    """src/embedders/gvizForceEmbedder.c:12-17"""
    if vertex_count == 0:
        return edge_length
    return 0.5 * math.sqrt(float(vertex_count)) * edge_length


class ForceLayout:
    """One layout (or a batch of independent layouts) on one GPU.

    ``row_offsets``/``neighbors`` is the CSR of the (sub)graph in compact
    vertex order; ``graph_offsets`` (optional) splits the vertices into
    independent graphs laid out together.
    """

    def __init__(self, row_offsets, neighbors, model=N.MODEL_FR, degree=None,
                 graph_offsets=None, device=0):
        self.L = N.lib()
        self.row = np.ascontiguousarray(row_offsets, dtype=np.uint64)
        self.col = np.ascontiguousarray(neighbors, dtype=np.uint32)
        self.V = int(self.row.shape[0] - 1)
        self.model = model
        self.degree = (np.ascontiguousarray(degree, dtype=np.uint64) if degree is not None
                       else np.diff(self.row).astype(np.uint64))
        if graph_offsets is None:
            self.goff = np.array([0, self.V], dtype=np.uint64)
        else:
            self.goff = np.ascontiguousarray(graph_offsets, dtype=np.uint64)
        self.G = int(self.goff.shape[0] - 1)
        desc = N.GraphDesc()
        desc.vertexCount = self.V
        desc.rowOffsets = N.ptr(self.row, C.c_uint64)
        desc.neighbors = N.ptr(self.col, C.c_uint32) if self.col.size else None
        desc.degree = N.ptr(self.degree, C.c_uint64)
        desc.graphCount = self.G
        desc.graphOffsets = N.ptr(self.goff, C.c_uint64) if self.G > 1 else None
        desc.model = model
        desc.device = device
        h = C.c_void_p()
        N.check(self.L.gvizCudaForceCreate(C.byref(h), C.byref(desc)), "gvizCudaForceCreate")
        self.h = h
        self.params = N.ForceParams()
        self.L.gvizCudaForceDefaultParams(C.byref(self.params))
        self.box_extent = default_box_extent(self.V, self.params.edgeLength)
        self.begun = False
        self._push()

    # ---------------------------------------------------------------- config
    def _push(self):
        N.check(self.L.gvizCudaForceSetParams(self.h, C.byref(self.params)),
                "gvizCudaForceSetParams")

    def configure(self, edge_length=0.0, box_extent=0.0):
        """gvizForceEmbedderConfigure (src/embedders/gvizForceEmbedder.c:357-363)"""
        if edge_length > 0.0:
            self.params.edgeLength = edge_length
        if box_extent > 0.0:
            self.box_extent = box_extent
        self._push()

    def configure_speed(self, tolerance):
        """gvizForceEmbedderConfigureSpeed (:365-369)"""
        if tolerance > 0.0:
            self.params.jitterTolerance = tolerance
        self._push()

    def configure_barnes_hut(self, theta, nodes_per_cell):
        """gvizForceEmbedderConfigureBarnesHut (:371-377)"""
        if theta > 0.0:
            self.params.theta = theta
        if nodes_per_cell > 0:
            self.params.nodesPerCell = nodes_per_cell
        self._push()

    def set_barnes_hut_enabled(self, enabled):
        self.params.barnesHutEnabled = 1 if enabled else 0
        self._push()

    def configure_gravity(self, k):
        """assigned unconditionally (:384-387)"""
        self.params.gravityK = k
        self._push()

    def configure_radius(self, base, per_degree):
        """assigned unconditionally (:395-399)"""
        self.params.radiusBase = base
        self.params.radiusPerDegree = per_degree
        self._push()

    def configure_overlap_prevention(self, constant):
        if constant > 0.0:
            self.params.overlapConstant = constant
        self._push()

    def set_prevent_overlap_enabled(self, enabled):
        self.params.preventOverlap = 1 if enabled else 0
        self._push()

    def toggle_overlap_prevention(self):
        """the "forceEmbedder.toggleOverlapPrevention" action (:210-217)"""
        self.set_prevent_overlap_enabled(not self.params.preventOverlap)

    def set_precision(self, precision):
        self.params.precision = N.FP64 if precision in (N.FP64, "fp64") else N.FP32
        self._push()

    def set_strict_reductions(self, on):
        self.params.strictReductions = 1 if on else 0
        self._push()

    def set_params(self, **kw):
        for k, v in kw.items():
            setattr(self.params, k, v)
        self._push()

    def vertex_radius(self, index):
        """gvizForceEmbedderVertexRadius (:389-393)"""
        return self.params.radiusBase * (
            1.0 + self.params.radiusPerDegree * math.sqrt(float(self.degree[index])))

    # -------------------------------------------------------------- lifecycle
    def begin(self, seed, positions=None):
        """gvizForceEmbedderBegin (:412-443): rand_r placement in
        [-boxExtent, boxExtent]^2 (or the given positions), FA2 reset."""
        if positions is None:
            positions = np.zeros(2 * self.V)
            self.L.gvizCudaRandomizePositions(N.ptr(positions, C.c_double), self.V,
                                              self.box_extent, seed)
        self.set_positions(positions)
        N.check(self.L.gvizCudaForceBegin(self.h), "gvizCudaForceBegin")
        self.begun = True
        return 0

    def set_positions(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        assert xy.shape[0] == 2 * self.V
        N.check(self.L.gvizCudaForceSetPositions(self.h, N.ptr(xy, C.c_double)),
                "gvizCudaForceSetPositions")

    def positions(self):
        xy = np.zeros(2 * self.V)
        N.check(self.L.gvizCudaForceGetPositions(self.h, N.ptr(xy, C.c_double)),
                "gvizCudaForceGetPositions")
        return xy

    def set_fa2_state(self, struct_force=None, speed=None, efficiency=None):
        sf = None if struct_force is None else np.ascontiguousarray(struct_force, np.float64)
        sp = None if speed is None else np.ascontiguousarray(np.broadcast_to(speed, (self.G,)), np.float64)
        ef = None if efficiency is None else np.ascontiguousarray(np.broadcast_to(efficiency, (self.G,)), np.float64)
        N.check(self.L.gvizCudaForceSetFa2State(self.h, N.ptr(sf, C.c_double),
                                                N.ptr(sp, C.c_double), N.ptr(ef, C.c_double)),
                "gvizCudaForceSetFa2State")

    def fa2_state(self):
        sf = np.zeros(2 * self.V)
        sp = np.zeros(self.G)
        ef = np.zeros(self.G)
        N.check(self.L.gvizCudaForceGetFa2State(self.h, N.ptr(sf, C.c_double),
                                                N.ptr(sp, C.c_double), N.ptr(ef, C.c_double)),
                "gvizCudaForceGetFa2State")
        return sf, sp, ef

    # --------------------------------------------------------------- stepping
    def step(self):
        """gvizForceEmbedderStep: returns graph 0's maxDisp."""
        st = (N.StepStats * self.G)()
        md = self.L.gvizCudaForceStep(self.h, st)
        if md < 0:
            N.check(int(md), "gvizCudaForceStep")
        self.last_stats = st
        return md

    def step_host(self, xy):
        """End-to-end step over a host position buffer (updated in place)."""
        st = (N.StepStats * self.G)()
        md = self.L.gvizCudaForceStepHost(self.h, N.ptr(xy, C.c_double), st)
        if md < 0:
            N.check(int(md), "gvizCudaForceStepHost")
        self.last_stats = st
        return md

    def run_host(self, xy, steps):
        """`steps` end-to-end steps over a host position buffer (updated in
        place after every step; copies pipelined across steps)."""
        st = (N.StepStats * self.G)()
        md = self.L.gvizCudaForceRunHost(self.h, N.ptr(xy, C.c_double), steps, st)
        if md < 0:
            N.check(int(md), "gvizCudaForceRunHost")
        self.last_stats = st
        return md

    def enqueue_steps(self, n):
        N.check(self.L.gvizCudaForceEnqueueSteps(self.h, n), "gvizCudaForceEnqueueSteps")

    def synchronize(self):
        N.check(self.L.gvizCudaForceSynchronize(self.h), "gvizCudaForceSynchronize")

    def time_steps(self, n):
        ms = C.c_float()
        N.check(self.L.gvizCudaForceTimeSteps(self.h, n, C.byref(ms)), "gvizCudaForceTimeSteps")
        return ms.value

    def run(self, max_iters, epsilon):
        """gvizForceEmbedderRun (:497-510): rounds run (graph 0), -1 before Begin."""
        if not self.begun:
            return -1
        rounds = np.zeros(self.G, np.uint64)
        N.check(self.L.gvizCudaForceRun(self.h, max_iters, epsilon, N.ptr(rounds, C.c_uint64)),
                "gvizCudaForceRun")
        self.rounds = rounds
        return int(rounds[0])

    def stat_history(self, graph=0):
        """rows of {maxDisp, speed, meanAtt, meanRep, meanGrav} since Begin"""
        n = self.L.gvizCudaForceStatHistory(self.h, graph, None, 0)
        N.check(int(n), "gvizCudaForceStatHistory")
        out = np.zeros((max(int(n), 1), 5))
        self.L.gvizCudaForceStatHistory(self.h, graph, N.ptr(out, C.c_double), int(n))
        return out[: int(n)]

    def forces(self):
        V = self.V
        out = {k: np.zeros(2 * V) for k in ("disp", "structForce", "applied")}
        out.update({k: np.zeros(V) for k in ("attMag", "repMag", "swing", "traction")})
        N.check(self.L.gvizCudaForceGetForces(
            self.h, N.ptr(out["disp"], C.c_double), N.ptr(out["structForce"], C.c_double),
            N.ptr(out["attMag"], C.c_double), N.ptr(out["repMag"], C.c_double),
            N.ptr(out["swing"], C.c_double), N.ptr(out["traction"], C.c_double),
            N.ptr(out["applied"], C.c_double)), "gvizCudaForceGetForces")
        return out

    # ------------------------------------------------------------- inspection
    def tree_leaves(self):
        V = self.V
        depth = np.zeros(V, np.int32)
        hi = np.zeros(V, np.uint64)
        lo = np.zeros(V, np.uint64)
        cnt = C.c_uint64()
        N.check(self.L.gvizCudaForceTreeLeaves(self.h, N.ptr(depth, C.c_int32),
                                               N.ptr(hi, C.c_uint64), N.ptr(lo, C.c_uint64),
                                               C.byref(cnt)), "gvizCudaForceTreeLeaves")
        return depth, hi, lo, cnt.value

    def tree_nodes(self):
        cap = 3 * self.V + 64
        depth = np.zeros(cap, np.int32)
        hi = np.zeros(cap, np.uint64)
        lo = np.zeros(cap, np.uint64)
        mass = np.zeros(cap)
        cx = np.zeros(cap)
        cy = np.zeros(cap)
        cnt = np.zeros(cap, np.uint64)
        n = self.L.gvizCudaForceTreeNodes(self.h, cap, N.ptr(depth, C.c_int32),
                                          N.ptr(hi, C.c_uint64), N.ptr(lo, C.c_uint64),
                                          N.ptr(mass, C.c_double), N.ptr(cx, C.c_double),
                                          N.ptr(cy, C.c_double), N.ptr(cnt, C.c_uint64))
        N.check(int(n), "gvizCudaForceTreeNodes")
        n = int(n)
        return dict(depth=depth[:n], hi=hi[:n], lo=lo[:n], mass=mass[:n], comX=cx[:n],
                    comY=cy[:n], count=cnt[:n])

    def exact_repulsion(self, targets):
        t = np.ascontiguousarray(targets, dtype=np.uint32)
        out = np.zeros(2 * t.shape[0])
        N.check(self.L.gvizCudaForceExactRepulsion(self.h, N.ptr(t, C.c_uint32), t.shape[0],
                                                   N.ptr(out, C.c_double)),
                "gvizCudaForceExactRepulsion")
        return out.reshape(-1, 2)

    def repulsion(self):
        out = np.zeros(2 * self.V)
        N.check(self.L.gvizCudaForceRepulsion(self.h, N.ptr(out, C.c_double)),
                "gvizCudaForceRepulsion")
        return out.reshape(-1, 2)

    def count_interactions(self):
        a, b = C.c_uint64(), C.c_uint64()
        N.check(self.L.gvizCudaForceCountInteractions(self.h, C.byref(a), C.byref(b)),
                "gvizCudaForceCountInteractions")
        return a.value, b.value

    def autotune(self):
        """Times the FP32 walk's launch shapes on the current positions and
        keeps the fastest: returns (threads per block, persistent, walk ms)."""
        t, p, ms = C.c_uint32(), C.c_int32(), C.c_float()
        N.check(self.L.gvizCudaForceAutotune(self.h, C.byref(t), C.byref(p), C.byref(ms)),
                "gvizCudaForceAutotune")
        return int(t.value), bool(p.value), float(ms.value)

    def set_far_judge(self, every=0, samples=4096, plain_theta=0.5, slack=1.0, seed=1):
        """The learned walk's judge (gvizCudaForceSetFarJudge): checks every
        `every` steps (0: on request) against the plain walk at plain_theta
        on `samples` vertices; a learned error above slack times the plain
        one turns the learned walk off."""
        N.check(self.L.gvizCudaForceSetFarJudge(self.h, every, samples, float(plain_theta),
                                                 float(slack), seed),
                "gvizCudaForceSetFarJudge")

    def judge_far_field(self):
        """One check now: (learned error, plain error, fell back)."""
        le, pe, fb = C.c_double(), C.c_double(), C.c_int32()
        N.check(self.L.gvizCudaForceJudgeFarField(self.h, C.byref(le), C.byref(pe),
                                                   C.byref(fb)),
                "gvizCudaForceJudgeFarField")
        return le.value, pe.value, bool(fb.value)

    def far_judge_status(self):
        """(checks run, last learned error, last plain error, fell back)."""
        n, le, pe, fb = C.c_uint64(), C.c_double(), C.c_double(), C.c_int32()
        N.check(self.L.gvizCudaForceFarJudgeStatus(self.h, C.byref(n), C.byref(le),
                                                    C.byref(pe), C.byref(fb)),
                "gvizCudaForceFarJudgeStatus")
        return n.value, le.value, pe.value, bool(fb.value)

    def set_walk_stack_cap(self, entries):
        """Stack entries per warp of the FP32 walks, plain and learned
        (32..512; 0 restores the default: the autotuner's pick for the plain
        walk, else 512): forces agree up to the order of the per-target sums."""
        N.check(self.L.gvizCudaForceSetWalkStackCap(self.h, entries),
                "gvizCudaForceSetWalkStackCap")

    def set_walk_shape(self, threads, persistent):
        N.check(self.L.gvizCudaForceSetWalkShape(self.h, threads, int(persistent)),
                "gvizCudaForceSetWalkShape")

    def walk_shape(self):
        """The plain FP32 walk's shape in use: (threads per block, persistent,
        stack entries per warp)."""
        t, p, c = C.c_uint32(), C.c_int32(), C.c_uint32()
        N.check(self.L.gvizCudaForceGetWalkShape(self.h, C.byref(t), C.byref(p), C.byref(c)),
                "gvizCudaForceGetWalkShape")
        return int(t.value), bool(p.value), int(c.value)

    # ------------------------------------------------------------ checkpoints
    def save_checkpoint(self, filename, name=""):
        """Lossless checkpoint (positions, FA2 history, counters, stats)."""
        N.check(self.L.gvizCudaForceSaveCheckpoint(self.h, name.encode(), str(filename).encode()),
                "gvizCudaForceSaveCheckpoint")

    def load_checkpoint(self, filename, restore_params=False):
        """Restores a checkpoint of this graph; returns the saved name."""
        buf = C.create_string_buffer(256)
        N.check(self.L.gvizCudaForceLoadCheckpoint(self.h, str(filename).encode(),
                                                   int(restore_params), buf, 256),
                "gvizCudaForceLoadCheckpoint")
        if restore_params:
            self.L.gvizCudaForceGetParams(self.h, C.byref(self.params))
        self.begun = True
        return buf.value.decode()

    def save_embedding_text(self, filename, name=""):
        """Positions in gviz's text format, every bit kept (17 digits)."""
        N.check(self.L.gvizCudaForceSaveEmbeddingText(self.h, name.encode(),
                                                      str(filename).encode()),
                "gvizCudaForceSaveEmbeddingText")

    def count_far_rows(self, causes=False):
        """(shared rows, per-target rows) of MLP evaluations in one force
        evaluation with the learned correction on; with causes=True also the
        per-target rows by cause (too few targets, spread, centroid test)."""
        a, b = C.c_uint64(), C.c_uint64()
        why = np.zeros(3, np.uint64)
        N.check(self.L.gvizCudaForceCountFarRows(self.h, C.byref(a), C.byref(b),
                                                 N.ptr(why, C.c_uint64)),
                "gvizCudaForceCountFarRows")
        if causes:
            return a.value, b.value, [int(x) for x in why]
        return a.value, b.value

    def far_groups(self):
        """The target groups of the learned cell-group walk on the current
        positions: (per-vertex group index, number of groups)."""
        out = np.zeros(self.V, np.uint32)
        n = C.c_uint64()
        N.check(self.L.gvizCudaForceFarGroups(self.h, N.ptr(out, C.c_uint32), C.byref(n)),
                "gvizCudaForceFarGroups")
        return out, n.value

    def profile_step(self):
        names = (C.c_char_p * 64)()
        ms = np.zeros(64)
        n = self.L.gvizCudaForceProfileStep(self.h, 64, names, N.ptr(ms, C.c_double))
        N.check(int(n), "gvizCudaForceProfileStep")
        return [(names[i].decode(), float(ms[i])) for i in range(n)]

    def last_error(self):
        return int(self.L.gvizCudaForceLastError(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.gvizCudaForceDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
