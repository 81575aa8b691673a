"""The reference GRIP embedder as the GPU GRIP tests use it (oracle/_ref,
src/embedders/gvizGRIPEmbedder.c compiled from its sources): layers nest,
the finest layer holds every vertex, every k-nearest list names active
vertices of the layer at graph distances >= 1, and rounds move the layout
without NaNs (the reference's own invariant, :1322-1323). The library's own
k-nearest search (gvizCudaGripKNearest) reproduces the reference's lists."""
import numpy as np
import pytest


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


def _grip_graph(kind):
    from grapher_b200 import graphs
    if kind == "grid":
        a, b = graphs.grid(12, 12)
        return 144, a, b
    if kind == "ba":
        a, b = graphs.barabasi_albert(1500, 3, 5)
        return 1500, a, b
    a, b = graphs.random_connected(400, 0.02, 3)
    return 400, np.asarray(a), np.asarray(b)


@pytest.mark.parametrize("kind", ["grid", "ba", "random"])
def test_k_nearest_matches_reference_on_every_layer(ref, kind):
    """gvizCudaGripKNearest (host, all threads) gives the reference's
    refinement lists (k = 128, the layer's vertices visible) entry for
    entry on every layer."""
    from grapher_b200 import graphs
    from grapher_b200.grip import k_nearest
    V, a, b = _grip_graph(kind)
    row, col = graphs.to_csr(V, a, b)
    rg = ref.create_grip(V, a, b)
    rg.begin()
    while True:
        act = rg.active()
        vis = np.zeros(V, np.uint8)
        vis[act] = 1
        off, kv, kd = rg.knn()
        o2, v2, d2 = k_nearest(row, col, act, 128, vis)
        assert np.array_equal(off, o2) and np.array_equal(kv, v2) and np.array_equal(kd, d2)
        if rg.layer == 0:
            break
        rg.next_stage()
    rg.close()


def test_identical_states_stay_identical_after_heap_reuse(ref):
    """Two GRIP states built from the same graph take the same filtration,
    k-nearest lists and rounds on every layer, also after a released state
    has left its BFS stamps on the heap: the driver clears the stamp array
    the reference allocates without clearing
    (src/embedders/gvizGRIPEmbedder.c:253) before Begin reads it."""
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(600, 3, 5)
    for _ in range(3):    # states whose freed stamps hold small epochs
        old = ref.create_grip(600, a, b)
        old.begin()
        old.close()
    s1, s2 = ref.create_grip(600, a, b), ref.create_grip(600, a, b)
    s1.begin()
    s2.begin()
    layers = 0
    while True:
        assert np.array_equal(s1.active(), s2.active())
        for x, y in zip(s1.knn(), s2.knn()):
            assert np.array_equal(x, y)
        for _ in range(2):
            assert np.array_equal(s1.refine(), s2.refine())
            assert np.array_equal(s1.positions(), s2.positions())
        layers += 1
        if s1.layer == 0:
            break
        s1.next_stage()
        s2.next_stage()
    assert layers >= 3
    s1.close()
    s2.close()
