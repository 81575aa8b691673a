"""ctypes bindings for the test/baseline infrastructure under oracle/.

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py; never by the grapher_b200 package.

- ``Oracle``: the CPU restatement (oracle/liboracle.so, from gviz_oracle.c).
- ``Reference``: the unmodified gviz reference compiled from source with the
  flat driver ref_driver.c (oracle/_ref/libgviz_ref.so), when it was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgviz_ref.so")

MODEL_FR = 0
MODEL_LINLOG = 1


class Params(C.Structure):
    """Same fields as orcParams / refParams; mirrors the reference embedder's
    configuration (include/embedders/gvizForceEmbedder.h:52-125)."""

    _fields_ = [
        ("model", C.c_int32),
        ("barnesHutEnabled", C.c_int32),
        ("preventOverlap", C.c_int32),
        ("_pad", C.c_int32),
        ("nodesPerCell", C.c_uint64),
        ("edgeLength", C.c_double),
        ("theta", C.c_double),
        ("gravityK", C.c_double),
        ("radiusBase", C.c_double),
        ("radiusPerDegree", C.c_double),
        ("overlapConstant", C.c_double),
        ("jitterTolerance", C.c_double),
    ]


def make_params(model=MODEL_FR, theta=1.0, nodes_per_cell=1, bh=True,
                edge_length=10.0, gravity=0.0, radius_base=0.0,
                radius_per_degree=0.0, overlap_constant=100.0,
                prevent_overlap=False, jitter_tolerance=1.0) -> Params:
    p = Params()
    p.model = model
    p.barnesHutEnabled = 1 if bh else 0
    p.preventOverlap = 1 if prevent_overlap else 0
    p.nodesPerCell = nodes_per_cell
    p.edgeLength = edge_length
    p.theta = theta
    p.gravityK = gravity
    p.radiusBase = radius_base
    p.radiusPerDegree = radius_per_degree
    p.overlapConstant = overlap_constant
    p.jitterTolerance = jitter_tolerance
    return p


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


D = C.c_double
U64 = C.c_uint64
U32 = C.c_uint32
I32 = C.c_int32


def build(quiet=True) -> None:
    """Compiles liboracle.so (and _ref when the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_step.restype = D
        L.orc_forces.restype = C.c_int
        L.orc_quadtree_leaves.restype = C.c_int
        L.orc_quadtree_nodes.restype = C.c_size_t

    # ---- pair formulas (include/core/gvizVec.h) ----
    def pair(self, name, *args):
        fn = getattr(self.lib, "orc_pair_" + name)
        acc = np.zeros(2)
        conv = []
        for a in args:
            if isinstance(a, (list, tuple, np.ndarray)):
                arr = np.ascontiguousarray(a, dtype=np.float64)
                conv.append(arr)
            else:
                conv.append(float(a))
        cargs = [(_ptr(a, D) if isinstance(a, np.ndarray) else D(a)) for a in conv]
        fn(*cargs, _ptr(acc, D))
        return acc

    def dir_table(self):
        out = np.zeros(512)
        self.lib.orc_dir_table(_ptr(out, D))
        return out.reshape(256, 2)

    def coincident_dir(self, i, j):
        ux, uy = D(), D()
        self.lib.orc_coincident_dir(U64(i), U64(j), C.byref(ux), C.byref(uy))
        return ux.value, uy.value

    # ---- quadtree ----
    def quadtree_leaves(self, pts, mass, k=1):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        n = mass.shape[0]
        depth = np.zeros(n, np.int32)
        hi = np.zeros(n, np.uint64)
        lo = np.zeros(n, np.uint64)
        cnt = C.c_size_t()
        rc = self.lib.orc_quadtree_leaves(_ptr(pts, D), _ptr(mass, D), C.c_size_t(n),
                                          C.c_size_t(k), _ptr(depth, I32), _ptr(hi, U64),
                                          _ptr(lo, U64), C.byref(cnt))
        assert rc == 0
        return depth, hi, lo, cnt.value

    def quadtree_nodes(self, pts, mass, k=1, cap=None):
        return _nodes_call(self.lib.orc_quadtree_nodes, pts, mass, k, cap)

    # ---- forces / step ----
    def forces(self, csr, mass, degree, params, pos):
        row, col = csr
        V = mass.shape[0]
        disp = np.zeros(2 * V)
        sf = np.zeros(2 * V)
        att = np.zeros(V)
        rep = np.zeros(V)
        inter = np.zeros(V, np.uint64)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        rc = self.lib.orc_forces(C.c_size_t(V), _ptr(row, U64), _ptr(col, U32), _ptr(mass, D),
                                 _ptr(degree, U64), C.byref(params), _ptr(pos, D),
                                 _ptr(disp, D), _ptr(sf, D), _ptr(att, D), _ptr(rep, D),
                                 _ptr(inter, U64))
        assert rc == 0
        return dict(disp=disp, structForce=sf, attMag=att, repMag=rep, interactions=inter)

    def step(self, csr, mass, degree, params, pos, struct_force, speed_state):
        """One step; pos, struct_force (2V float64) and speed_state (2,) are
        updated in place. Returns a dict of per-vertex outputs and stats."""
        row, col = csr
        V = mass.shape[0]
        stats = np.zeros(5)
        out = {k: np.zeros(2 * V) for k in ("disp", "applied")}
        out.update({k: np.zeros(V) for k in ("attMag", "repMag", "swing", "traction")})
        md = self.lib.orc_step(C.c_size_t(V), _ptr(row, U64), _ptr(col, U32), _ptr(mass, D),
                               _ptr(degree, U64), C.byref(params), _ptr(pos, D),
                               _ptr(struct_force, D), _ptr(speed_state, D), _ptr(stats, D),
                               _ptr(out["disp"], D), _ptr(out["attMag"], D),
                               _ptr(out["repMag"], D), _ptr(out["swing"], D),
                               _ptr(out["traction"], D), _ptr(out["applied"], D))
        out["stats"] = stats
        out["maxDisp"] = md
        return out

    def exact_repulsion(self, mass, degree, params, pos, targets):
        V = mass.shape[0]
        targets = np.ascontiguousarray(targets, dtype=np.uint64)
        out = np.zeros(2 * targets.shape[0])
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        self.lib.orc_exact_repulsion(C.c_size_t(V), _ptr(mass, D), _ptr(degree, U64),
                                     C.byref(params), _ptr(pos, D), _ptr(targets, U64),
                                     C.c_size_t(targets.shape[0]), _ptr(out, D))
        return out.reshape(-1, 2)


def _nodes_call(fn, pts, mass, k, cap):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    cap = cap or max(16, 8 * n + 64)
    depth = np.zeros(cap, np.int32)
    hi = np.zeros(cap, np.uint64)
    lo = np.zeros(cap, np.uint64)
    m = np.zeros(cap)
    cx = np.zeros(cap)
    cy = np.zeros(cap)
    leaf = np.zeros(cap, np.int32)
    cnt = np.zeros(cap, np.uint64)
    fn.restype = C.c_size_t
    w = fn(_ptr(pts, D), _ptr(mass, D), C.c_size_t(n), C.c_size_t(k), C.c_size_t(cap),
           _ptr(depth, I32), _ptr(hi, U64), _ptr(lo, U64), _ptr(m, D), _ptr(cx, D),
           _ptr(cy, D), _ptr(leaf, I32), _ptr(cnt, U64))
    return dict(depth=depth[:w], hi=hi[:w], lo=lo[:w], mass=m[:w], comX=cx[:w],
                comY=cy[:w], isLeaf=leaf[:w], count=cnt[:w])


class Reference:
    """The real gviz embedder (compiled from the reference's sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        # global symbols: glue libraries loaded later resolve gviz's API here
        self.lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
        L = self.lib
        for name in ("ref_create_edges", "ref_create_builtin"):
            getattr(L, name).restype = C.c_void_p
        L.ref_step.restype = D
        L.ref_vertex_count.restype = C.c_size_t
        L.ref_box_extent.restype = D
        L.ref_get_stats.restype = C.c_size_t
        L.ref_pool_threads.restype = C.c_long
        L.ref_quadtree_nodes.restype = C.c_size_t
        L.ref_state.restype = C.c_void_p
        for name in ("ref_step", "ref_vertex_count", "ref_box_extent", "ref_begin",
                     "ref_init_result", "ref_run", "ref_release", "ref_configure",
                     "ref_get_csr", "ref_get_degree_mass", "ref_get_positions",
                     "ref_set_positions", "ref_set_fa2_state", "ref_get_state",
                     "ref_get_stats", "ref_time_steps", "ref_set_prevent_overlap",
                     "ref_invoke_step_action"):
            getattr(L, name).argtypes = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def pool_threads(self) -> int:
        return int(self.lib.ref_pool_threads())

    # ---- embedder lifecycle ----
    def create_edges(self, V, ea, eb, model):
        ea = np.ascontiguousarray(ea, dtype=np.uint32)
        eb = np.ascontiguousarray(eb, dtype=np.uint32)
        h = self.lib.ref_create_edges(C.c_size_t(V), _ptr(ea, U32), _ptr(eb, U32),
                                      C.c_size_t(ea.shape[0]), C.c_int(model))
        return RefLayout(self, h)

    # ---- the reference's graph loaders, exported as CSR ----
    def _load_csr(self, fn, *args):
        fn.restype = C.c_longlong
        n = C.c_size_t()
        V = fn(*args, None, None, C.byref(n))
        if V < 0:
            return None
        row = np.zeros(V + 1, np.uint64)
        col = np.zeros(max(1, n.value), np.uint32)
        fn(*args, _ptr(row, C.c_uint64), _ptr(col, U32), C.byref(n))
        return row, col[:n.value]

    def load_edges_csr(self, path, directed=False, skip_header=False):
        """gvizGraphLoadFromEdgesFile, then the graph's adjacency as CSR;
        None when the loader fails."""
        return self._load_csr(self.lib.ref_load_edges_csr, str(path).encode(),
                              C.c_int(int(directed)), C.c_int(int(skip_header)))

    def load_obj_csr(self, path):
        """gvizGraphLoadFromObjFile, then the adjacency as CSR (or None)."""
        return self._load_csr(self.lib.ref_load_obj_csr, str(path).encode())

    def load_gexf_csr(self, path):
        """gvizGraphLoadFromGexfFile, then the adjacency as CSR (or None)."""
        return self._load_csr(self.lib.ref_load_gexf_csr, str(path).encode())

    def create_builtin(self, kind, a, b=0, density=0.0, seed=0, model=MODEL_FR):
        h = self.lib.ref_create_builtin(C.c_int(kind), C.c_size_t(a), C.c_size_t(b),
                                        D(density), C.c_uint(seed), C.c_int(model))
        return RefLayout(self, h)

    def quadtree_leaves(self, pts, mass, k=1):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        n = mass.shape[0]
        depth = np.zeros(n, np.int32)
        hi = np.zeros(n, np.uint64)
        lo = np.zeros(n, np.uint64)
        cnt = C.c_size_t()
        rc = self.lib.ref_quadtree_leaves(_ptr(pts, D), _ptr(mass, D), C.c_size_t(n),
                                          C.c_size_t(k), _ptr(depth, I32), _ptr(hi, U64),
                                          _ptr(lo, U64), C.byref(cnt))
        assert rc == 0
        return depth, hi, lo, cnt.value

    def quadtree_nodes(self, pts, mass, k=1, cap=None):
        return _nodes_call(self.lib.ref_quadtree_nodes, pts, mass, k, cap)

    def create_grip(self, V, ea, eb, serial=True):
        """The reference's GRIP embedder (2-D) on an ordered edge list;
        serial=True runs its parallel phases on the calling thread (see
        ref_grip_create: pooled rounds race on the dispCalculated marks)."""
        return RefGrip(self, V, ea, eb, serial)


class RefGrip:
    """gvizGRIPEmbedder driven through ref_driver.c: Begin / NextStage /
    RefineRound, and the layer's filtration order, k-nearest lists,
    positions and decorators read back."""

    def __init__(self, ref: Reference, V, ea, eb, serial=True):
        L = ref.lib
        L.ref_grip_create.restype = C.c_void_p
        for name in ("ref_grip_layer", "ref_grip_layer_count", "ref_grip_active", "ref_grip_knn"):
            getattr(L, name).restype = C.c_size_t
        self.L = L
        self.V = int(V)
        self._ea = np.ascontiguousarray(ea, dtype=np.uint32)
        self._eb = np.ascontiguousarray(eb, dtype=np.uint32)
        self.h = C.c_void_p(L.ref_grip_create(C.c_size_t(V), _ptr(self._ea, U32),
                                              _ptr(self._eb, U32),
                                              C.c_size_t(self._ea.shape[0]),
                                              C.c_int(int(bool(serial)))))
        assert L.ref_grip_init_result(self.h) == 0

    def begin(self):
        self.L.ref_grip_begin(self.h)

    def next_stage(self):
        self.L.ref_grip_next_stage(self.h)

    @property
    def layer(self):
        return int(self.L.ref_grip_layer(self.h))

    @property
    def layer_count(self):
        return int(self.L.ref_grip_layer_count(self.h))

    def active(self):
        out = np.zeros(self.V, np.uint32)
        n = int(self.L.ref_grip_active(self.h, _ptr(out, U32), C.c_size_t(self.V)))
        return out[:n]

    def knn(self):
        """(offsets over the active order, vertices, graph distances)"""
        n = len(self.active())
        total = int(self.L.ref_grip_knn(self.h, None, None, None, C.c_size_t(0)))
        off = np.zeros(n + 1, np.uint64)
        v = np.zeros(max(total, 1), np.uint32)
        d = np.zeros(max(total, 1), np.uint32)
        self.L.ref_grip_knn(self.h, _ptr(off, U64), _ptr(v, U32), _ptr(d, U32), C.c_size_t(total))
        return off, v[:total], d[:total]

    def refine(self):
        """one round; (maxDisplacement, meanDisplacement, meanForce)"""
        st = np.zeros(3)
        self.L.ref_grip_refine(self.h, _ptr(st, D))
        return st

    def positions(self):
        xy = np.zeros(2 * self.V)
        self.L.ref_grip_get_positions(self.h, _ptr(xy, D))
        return xy

    def set_positions(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        self.L.ref_grip_set_positions(self.h, _ptr(xy, D))

    def decorators(self):
        heat = np.zeros(self.V)
        disp = np.zeros(2 * self.V)
        oc = np.zeros(self.V)
        self.L.ref_grip_get_decorators(self.h, _ptr(heat, D), _ptr(disp, D), _ptr(oc, D))
        return heat, disp, oc

    def state_ptr(self):
        self.L.ref_grip_state.restype = C.c_void_p
        return self.L.ref_grip_state(self.h)

    def invoke_refine(self):
        """the "grip.refineRound" action by name (whatever handler holds it)"""
        return int(self.L.ref_grip_invoke_refine(self.h))

    def last_stats(self):
        """(lastRoundStats as an array, currRound)"""
        self.L.ref_grip_last_stats.restype = C.c_size_t
        st = np.zeros(3)
        r = int(self.L.ref_grip_last_stats(self.h, _ptr(st, D)))
        return st, r

    def close(self):
        if self.h:
            self.L.ref_grip_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefLayout:
    def __init__(self, ref: Reference, handle):
        self.ref = ref
        self.h = C.c_void_p(handle)
        self.L = ref.lib
        assert self.L.ref_init_result(self.h) == 0
        self.V = int(self.L.ref_vertex_count(self.h))

    def configure(self, params: Params, box_extent=0.0):
        self.L.ref_configure(self.h, C.byref(params), D(box_extent))

    def set_prevent_overlap(self, on):
        self.L.ref_set_prevent_overlap(self.h, C.c_int(1 if on else 0))

    def set_barnes_hut(self, on):
        """gvizForceEmbedderSetBarnesHutEnabled (a live toggle)."""
        self.L.ref_set_barnes_hut(self.h, C.c_int(1 if on else 0))

    def begin(self, seed):
        return self.L.ref_begin(self.h, C.c_uint(seed))

    def box_extent(self):
        return self.L.ref_box_extent(self.h)

    def csr(self):
        row = np.zeros(self.V + 1, np.uint64)
        self.L.ref_get_csr(self.h, _ptr(row, U64), None)
        col = np.zeros(int(row[-1]) if self.V else 0, np.uint32)
        self.L.ref_get_csr(self.h, _ptr(row, U64), _ptr(col, U32) if col.size else None)
        return row, col

    def degree_mass(self):
        deg = np.zeros(self.V, np.uint64)
        mass = np.zeros(self.V)
        self.L.ref_get_degree_mass(self.h, _ptr(deg, U64), _ptr(mass, D))
        return deg, mass

    def positions(self):
        xy = np.zeros(2 * self.V)
        self.L.ref_get_positions(self.h, _ptr(xy, D))
        return xy

    def set_positions(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        self.L.ref_set_positions(self.h, _ptr(xy, D))

    def set_fa2_state(self, struct_force, speed, efficiency):
        sf = None if struct_force is None else np.ascontiguousarray(struct_force, np.float64)
        self.L.ref_set_fa2_state(self.h, _ptr(sf, D), D(speed), D(efficiency))

    def step(self):
        return self.L.ref_step(self.h)

    def invoke_step_action(self):
        return self.L.ref_invoke_step_action(self.h)

    def invoke_toggle_overlap(self):
        return self.L.ref_invoke_toggle_overlap(self.h)

    def state_ptr(self):
        return C.c_void_p(self.L.ref_state(self.h))

    def load_embedding(self, path):
        """gvizEmbeddedGraphLoadEmbedding; 0 or -1."""
        return int(self.L.ref_load_embedding(self.h, str(path).encode()))

    def save_embedding(self, path, name="ref"):
        """gvizEmbeddedGraphSaveEmbedding (six decimals); 0 or -1."""
        return int(self.L.ref_save_embedding(self.h, name.encode(), str(path).encode()))

    def run(self, max_iters, eps):
        return self.L.ref_run(self.h, C.c_size_t(max_iters), D(eps))

    def state(self):
        V = self.V
        out = {k: np.zeros(2 * V) for k in ("disp", "structForce", "applied")}
        out.update({k: np.zeros(V) for k in ("attMag", "repMag", "swing", "traction")})
        sc = np.zeros(5)
        self.L.ref_get_state(self.h, _ptr(out["disp"], D), _ptr(out["structForce"], D),
                             _ptr(out["attMag"], D), _ptr(out["repMag"], D),
                             _ptr(out["swing"], D), _ptr(out["traction"], D),
                             _ptr(out["applied"], D), _ptr(sc, D))
        out["speed"], out["efficiency"], out["iteration"] = sc[0], sc[1], int(sc[2])
        out["lastMaxDisp"], out["meanDegreePlusOne"] = sc[3], sc[4]
        return out

    def stats(self):
        res = []
        for w in range(5):
            n = int(self.L.ref_get_stats(self.h, C.c_int(w), None, C.c_size_t(0)))
            buf = np.zeros(max(n, 1))
            self.L.ref_get_stats(self.h, C.c_int(w), _ptr(buf, D), C.c_size_t(n))
            res.append(buf[:n])
        return np.stack(res, axis=1) if res and len(res[0]) else np.zeros((0, 5))

    def time_steps(self, steps):
        out = np.zeros(steps)
        self.L.ref_time_steps(self.h, C.c_int(steps), _ptr(out, D))
        return out

    def close(self):
        if self.h:
            self.L.ref_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
