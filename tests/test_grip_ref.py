"""The reference GRIP embedder as the GPU GRIP tests use it (oracle/_ref,
src/embedders/gvizGRIPEmbedder.c compiled from its sources): layers nest,
the finest layer holds every vertex, every k-nearest list names active
vertices of the layer at graph distances >= 1, and rounds move the layout
without NaNs (the reference's own invariant, :1322-1323)."""
import numpy as np


def test_reference_grip_layers_and_knn(ref):
    from grapher_b200 import graphs
    a, b = graphs.grid(10, 10)
    rg = ref.create_grip(100, a, b)
    rg.begin()
    assert rg.layer == rg.layer_count - 1 >= 2
    prev = set()
    while True:
        act = rg.active()
        assert len(set(act.tolist())) == len(act)
        assert prev <= set(act.tolist())
        prev = set(act.tolist())
        off, kv, kd = rg.knn()
        assert off[0] == 0 and np.all(np.diff(off.astype(np.int64)) >= 0)
        assert set(kv.tolist()) <= prev and np.all(kd >= 1)
        x0 = rg.positions()
        st = rg.refine()
        assert np.all(np.isfinite(st)) and np.all(np.isfinite(rg.positions()))
        moved = np.abs(rg.positions() - x0).reshape(-1, 2).max(1)
        assert moved[act].max() > 0
        if rg.layer == 0:
            break
        rg.next_stage()
    assert len(prev) == 100
    rg.close()
