"""Shared test helpers: one configuration dict drives both the oracle and the
CUDA path, golden fixtures are loaded from tests/golden/."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

DEFAULTS = dict(model=0, theta=1.0, k=1, bh=True, edge_length=10.0, gravity=0.0,
                radius_base=0.0, radius_per_degree=0.0, overlap_constant=100.0,
                prevent_overlap=False, jitter=1.0, precision="fp32", strict=False)


def cfg(**kw):
    c = dict(DEFAULTS)
    c.update(kw)
    return c


def oracle_params(c):
    from oracle.bindings import make_params
    return make_params(model=c["model"], theta=c["theta"], nodes_per_cell=c["k"],
                       bh=c["bh"], edge_length=c["edge_length"], gravity=c["gravity"],
                       radius_base=c["radius_base"],
                       radius_per_degree=c["radius_per_degree"],
                       overlap_constant=c["overlap_constant"],
                       prevent_overlap=c["prevent_overlap"], jitter_tolerance=c["jitter"])


def make_layout(row, col, c, graph_offsets=None):
    from grapher_b200 import ForceLayout
    lay = ForceLayout(row, col, model=c["model"], graph_offsets=graph_offsets)
    lay.set_params(theta=c["theta"], nodesPerCell=c["k"], barnesHutEnabled=int(c["bh"]),
                   edgeLength=c["edge_length"], gravityK=c["gravity"],
                   radiusBase=c["radius_base"], radiusPerDegree=c["radius_per_degree"],
                   overlapConstant=c["overlap_constant"],
                   preventOverlap=int(c["prevent_overlap"]), jitterTolerance=c["jitter"],
                   precision=1 if c["precision"] == "fp64" else 0,
                   strictReductions=int(c["strict"]))
    return lay


def golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_cfg(g):
    p = g["params"]
    return cfg(model=int(g["model"]), bh=bool(p[0]), prevent_overlap=bool(p[1]), k=int(p[2]),
               edge_length=float(p[3]), theta=float(p[4]), gravity=float(p[5]),
               radius_base=float(p[6]), radius_per_degree=float(p[7]),
               overlap_constant=float(p[8]), jitter=float(p[9]))


def csr_of(V, a, b):
    from grapher_b200 import graphs
    return graphs.to_csr(V, a, b)


def degree_mass(row, model):
    deg = np.diff(row).astype(np.uint64)
    mass = np.ones(len(deg)) if model == 0 else 1.0 + deg.astype(np.float64)
    return deg, mass


def rel_err(a, b, floor=0.0):
    """per-row relative error |a-b| / max(|b|, floor) for (n,2) vectors"""
    a = np.asarray(a).reshape(-1, 2)
    b = np.asarray(b).reshape(-1, 2)
    num = np.linalg.norm(a - b, axis=1)
    den = np.maximum(np.linalg.norm(b, axis=1), floor)
    return num / np.where(den > 0, den, 1.0)
