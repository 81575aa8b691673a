"""The force phase of gviz's GRIP embedder on the GPU (libgvizcuda's
gvizCudaGrip*): one refinement round (gvizGRIPEmbedderRefineRound,
src/embedders/gvizGRIPEmbedder.c:1289-1334) over a layer whose filtration
order and k-nearest lists the caller hands over, as gviz builds them.

    g = GripRefiner(row, col)
    g.set_positions(xy)                       # the embedding's positions
    g.set_layer(layer, active, off, knn_v, knn_d)
    stats = g.refine_round()                  # maxDisplacement, ...
    xy = g.positions()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def k_nearest(row_offsets, neighbors, sources, k, visible=None):
    """GRIP's k-nearest lists (gvizCudaGripKNearest): (offsets over the
    sources, vertices, graph distances)."""
    L = N.lib()
    row = np.ascontiguousarray(row_offsets, dtype=np.uint64)
    col = np.ascontiguousarray(neighbors, dtype=np.uint32)
    src = np.ascontiguousarray(sources, dtype=np.uint32)
    vis = None if visible is None else np.ascontiguousarray(visible, dtype=np.uint8)
    n = src.shape[0]
    off = np.zeros(n + 1, np.uint64)
    kv = np.zeros(max(1, n * int(k)), np.uint32)
    kd = np.zeros(max(1, n * int(k)), np.uint32)
    tot = L.gvizCudaGripKNearest(row.shape[0] - 1, N.ptr(row, C.c_uint64), N.ptr(col, C.c_uint32),
                                 N.ptr(src, C.c_uint32), n, N.ptr(vis, C.c_uint8), int(k),
                                 N.ptr(off, C.c_uint64), N.ptr(kv, C.c_uint32),
                                 N.ptr(kd, C.c_uint32))
    N.check(int(tot) if tot < 0 else 0, "gvizCudaGripKNearest")
    return off, kv[:tot].copy(), kd[:tot].copy()


class GripRefiner:
    def __init__(self, row_offsets, neighbors, device=0):
        self.L = N.lib()
        row = np.ascontiguousarray(row_offsets, dtype=np.uint64)
        col = np.ascontiguousarray(neighbors, dtype=np.uint32)
        self.V = int(row.shape[0] - 1)
        h = C.c_void_p()
        N.check(self.L.gvizCudaGripCreate(C.byref(h), self.V, N.ptr(row, C.c_uint64),
                                           N.ptr(col, C.c_uint32), device),
                "gvizCudaGripCreate")
        self.h = h

    def set_strict_reductions(self, on=True):
        N.check(self.L.gvizCudaGripSetStrictReductions(self.h, int(bool(on))),
                "gvizCudaGripSetStrictReductions")

    def set_positions(self, xy):
        xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        assert xy.shape[0] == 2 * self.V
        N.check(self.L.gvizCudaGripSetPositions(self.h, N.ptr(xy, C.c_double)),
                "gvizCudaGripSetPositions")

    def positions(self):
        out = np.zeros(2 * self.V)
        N.check(self.L.gvizCudaGripGetPositions(self.h, N.ptr(out, C.c_double)),
                "gvizCudaGripGetPositions")
        return out

    def set_layer(self, layer, active, knn_offsets, knn_vertices, knn_distances):
        """The layer's active vertices in filtration order and their
        k-nearest lists (CSR over that order); clears the decorators."""
        act = np.ascontiguousarray(active, dtype=np.uint32)
        off = np.ascontiguousarray(knn_offsets, dtype=np.uint64)
        kv = np.ascontiguousarray(knn_vertices, dtype=np.uint32)
        kd = np.ascontiguousarray(knn_distances, dtype=np.uint32)
        N.check(self.L.gvizCudaGripSetLayer(self.h, int(layer), N.ptr(act, C.c_uint32),
                                             act.shape[0], N.ptr(off, C.c_uint64),
                                             N.ptr(kv, C.c_uint32), N.ptr(kd, C.c_uint32)),
                "gvizCudaGripSetLayer")

    def refine_round(self):
        """One round; (maxDisplacement, meanDisplacement, meanForce, meanHeat)."""
        st = N.GripRoundStats()
        N.check(self.L.gvizCudaGripRefineRound(self.h, C.byref(st)), "gvizCudaGripRefineRound")
        return np.array([st.maxDisplacement, st.meanDisplacement, st.meanForce, st.meanHeat])

    def time_rounds(self, rounds):
        """(total ms, force-kernel ms) of `rounds` device-resident rounds,
        CUDA events on the handle's stream."""
        tot, frc = C.c_float(), C.c_float()
        N.check(self.L.gvizCudaGripTimeRounds(self.h, int(rounds), C.byref(tot), C.byref(frc)),
                "gvizCudaGripTimeRounds")
        return tot.value, frc.value

    def decorators(self):
        """Per vertex: heat, last displacement (2), previous cosine."""
        heat = np.zeros(self.V)
        disp = np.zeros(2 * self.V)
        oc = np.zeros(self.V)
        N.check(self.L.gvizCudaGripGetDecorators(self.h, N.ptr(heat, C.c_double),
                                                  N.ptr(disp, C.c_double),
                                                  N.ptr(oc, C.c_double)),
                "gvizCudaGripGetDecorators")
        return heat, disp, oc

    def close(self):
        if getattr(self, "h", None):
            self.L.gvizCudaGripDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
