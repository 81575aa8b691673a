"""Workload graphs as numpy arrays.

The generators come from libgvizworkloads (host only; importing them does
not load libgvizcuda). Edge lists are ordered (a[i], b[i]) pairs;
``to_csr`` (libgvizcuda) builds adjacency the way gvizGraphAddEdge does
(src/ds/gvizGraph.c:163-172).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def _gen(fn, *args):
    L = N.workloads_lib()
    f = getattr(L, fn)
    E = int(f(*args, None, None))
    a = np.zeros(E, np.uint32)
    b = np.zeros(E, np.uint32)
    f(*args, N.ptr(a, C.c_uint32), N.ptr(b, C.c_uint32))
    return a, b


def grid(rows, cols):
    """build_rect_mesh (src/utils/graphs.c:285-316)"""
    return _gen("gvizGenGrid", rows, cols)


def random_connected(n, density, seed):
    """build_random_connected_graph (src/utils/graphs.c:598-639)"""
    return _gen("gvizGenRandomConnected", n, float(density), seed)


def barabasi_albert(n, m, seed):
    return _gen("gvizGenBarabasiAlbert", n, m, seed)


def erdos_renyi(n, m, seed):
    return _gen("gvizGenErdosRenyi", n, m, seed)


def rmat(scale, draws, a=0.57, b=0.19, c=0.19, seed=1):
    return _gen("gvizGenRmat", scale, draws, a, b, c, seed)


def to_csr(V, a, b):
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    row = np.zeros(V + 1, np.uint64)
    col = np.zeros(2 * a.shape[0], np.uint32)
    N.check(N.lib().gvizCudaEdgesToCsr(V, N.ptr(a, C.c_uint32), N.ptr(b, C.c_uint32),
                                       a.shape[0], N.ptr(row, C.c_uint64),
                                       N.ptr(col, C.c_uint32)), "gvizCudaEdgesToCsr")
    return row, col


def randomize_positions(V, box_extent, seed):
    """gvizEmbeddedGraphRandomizePositions (src/embedders/gvizEmbeddedGraph.c:406-426)"""
    xy = np.zeros(2 * V)
    N.lib().gvizCudaRandomizePositions(N.ptr(xy, C.c_double), V, float(box_extent), seed)
    return xy


def unit_disk_positions(V, seed):
    """Seeded uniform positions in the unit disk (the exact-mode workload)."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.random(V))
    t = 2.0 * np.pi * rng.random(V)
    return np.stack([r * np.cos(t), r * np.sin(t)], axis=1).reshape(-1)


def batch(graphs):
    """Concatenates [(V, a, b), ...] into one CSR plus graph offsets."""
    offs = [0]
    aa, bb = [], []
    for V, a, b in graphs:
        aa.append(np.asarray(a, np.uint32) + np.uint32(offs[-1]))
        bb.append(np.asarray(b, np.uint32) + np.uint32(offs[-1]))
        offs.append(offs[-1] + V)
    a = np.concatenate(aa) if aa else np.zeros(0, np.uint32)
    b = np.concatenate(bb) if bb else np.zeros(0, np.uint32)
    row, col = to_csr(offs[-1], a, b)
    return row, col, np.asarray(offs, np.uint64)


def _take_csr(rc, csr, what):
    """Copies a library-owned gvizCudaCsr into numpy arrays and frees it."""
    L = N.lib()
    if rc != 0:
        raise OSError(f"{what}: gviz loader rules rejected the file or it could not be read")
    try:
        V, nnz = int(csr.vertexCount), int(csr.entryCount)
        row = np.ctypeslib.as_array(csr.rowOffsets, shape=(V + 1,)).copy()
        col = (np.ctypeslib.as_array(csr.neighbors, shape=(nnz,)).copy() if nnz
               else np.zeros(0, np.uint32))
        ext = (np.ctypeslib.as_array(csr.externalIds, shape=(V,)).copy()
               if bool(csr.externalIds) else None)
    finally:
        L.gvizCudaCsrFree(C.byref(csr))
    return row, col, ext


def load_edges_file(path, directed=False, skip_header=False):
    """gvizGraphLoadFromEdgesFile straight to CSR: (row_offsets, neighbors,
    external_ids) with gviz's vertex numbering and neighbour order."""
    csr = N.Csr()
    rc = N.lib().gvizCudaLoadEdgesFile(str(path).encode(), int(directed), int(skip_header),
                                        C.byref(csr))
    return _take_csr(rc, csr, f"load_edges_file({path})")


def load_obj_file(path):
    """gvizGraphLoadFromObjFile straight to CSR: (row_offsets, neighbors)."""
    csr = N.Csr()
    rc = N.lib().gvizCudaLoadObjFile(str(path).encode(), C.byref(csr))
    row, col, _ = _take_csr(rc, csr, f"load_obj_file({path})")
    return row, col


def load_gexf_file(path):
    """gvizGraphLoadFromGexfFile straight to CSR: (row_offsets, neighbors),
    vertices in <node> order, undirected edges in <edge> order."""
    csr = N.Csr()
    rc = N.lib().gvizCudaLoadGexfFile(str(path).encode(), C.byref(csr))
    row, col, _ = _take_csr(rc, csr, f"load_gexf_file({path})")
    return row, col
