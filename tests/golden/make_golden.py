"""Generates tests/golden/*.npz from the gviz reference compiled from source
(oracle/_ref/libgviz_ref.so, built by `make -C oracle`).

    python tests/golden/make_golden.py

Every fixture stores its inputs (edges or points) next to the reference's
outputs, so tests need neither the reference sources nor the generator.
Trajectory fixtures: positions / structForce / speed state after each of a few
reference steps (gvizForceEmbedderStep, src/embedders/gvizForceEmbedder.c:445-495)
plus the five stat series. Quadtree fixtures: per point the depth and
quadrant path of its leaf, per non-empty node depth / path / mass / centre of
mass / point count (gvizQuadtreeInit, src/ds/gvizQuadtree.c:200-225).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import MODEL_FR, MODEL_LINLOG, Reference, make_params  # noqa: E402
from grapher_b200 import graphs  # noqa: E402

STEPS = 4


def trajectory(name, V, a, b, model, params, box, seed, ref):
    r = ref.create_edges(V, a, b, model)
    r.configure(params, box)
    r.begin(seed)
    x0 = r.positions().copy()
    pos, sf, sc, md = [], [], [], []
    for _ in range(STEPS):
        md.append(r.step())
        st = r.state()
        pos.append(r.positions().copy())
        sf.append(st["structForce"].copy())
        sc.append([st["speed"], st["efficiency"]])
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), V=V, ea=a, eb=b, model=model,
        params=np.array([params.barnesHutEnabled, params.preventOverlap, params.nodesPerCell,
                         params.edgeLength, params.theta, params.gravityK, params.radiusBase,
                         params.radiusPerDegree, params.overlapConstant,
                         params.jitterTolerance]),
        box=box, seed=seed, x0=x0, pos=np.array(pos), structForce=np.array(sf),
        speedState=np.array(sc), maxDisp=np.array(md), stats=r.stats())
    r.close()


def quadtree(name, pts, mass, ks, ref):
    out = dict(pts=pts, mass=mass, ks=np.array(ks))
    for k in ks:
        d, hi, lo, nc = ref.quadtree_leaves(pts, mass, k)
        out[f"k{k}_leafDepth"] = d
        out[f"k{k}_pathHi"] = hi
        out[f"k{k}_pathLo"] = lo
        nd = ref.quadtree_nodes(pts, mass, k)
        for key, val in nd.items():
            out[f"k{k}_node_{key}"] = val
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def main():
    ref = Reference()
    a, b = graphs.grid(32, 32)
    trajectory("traj_grid32_fr_theta05", 1024, a, b, MODEL_FR,
               make_params(MODEL_FR, theta=0.5), 1.0, 7, ref)
    a, b = graphs.random_connected(300, 0.02, 5)
    trajectory("traj_rc300_linlog_theta08_grav_overlap", 300, a, b, MODEL_LINLOG,
               make_params(MODEL_LINLOG, theta=0.8, gravity=1.0, radius_base=1.0,
                           radius_per_degree=0.5, prevent_overlap=True), 100.0, 11, ref)
    a, b = graphs.random_connected(200, 0.05, 9)
    trajectory("traj_rc200_fr_exact", 200, a, b, MODEL_FR,
               make_params(MODEL_FR, bh=False), 0.0, 3, ref)
    a, b = graphs.random_connected(500, 0.0, 3)
    trajectory("traj_rc500_linlog_theta12_k3", 500, a, b, MODEL_LINLOG,
               make_params(MODEL_LINLOG, theta=1.2, nodes_per_cell=3), 0.0, 5, ref)

    rng = np.random.default_rng(2024)
    pts = rng.uniform(-1000.0, 1000.0, size=(3000, 2))
    mass = rng.integers(1, 6, size=3000).astype(np.float64)
    quadtree("qt_uniform3000", pts, mass, [1, 3], ref)

    # duplicates, near-duplicates below 1e-9 (overflow leaves), deep clusters
    base = rng.uniform(-5.0, 5.0, size=(40, 2))
    parts = [base, base[:10], base[:5] + 1e-12, base[5:9] + 3e-7,
             rng.normal(0.0, 1e-6, size=(30, 2)) + 2.0]
    pts2 = np.concatenate(parts)
    mass2 = np.ones(pts2.shape[0])
    quadtree("qt_duplicates", pts2, mass2, [1, 2], ref)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
