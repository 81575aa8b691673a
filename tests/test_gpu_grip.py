"""The GRIP force phase on the GPU (gvizCudaGrip*) against the reference's own
GRIP embedder (src/embedders/gvizGRIPEmbedder.c, compiled from its sources
into oracle/_ref): both start every layer from the reference's positions,
filtration order and k-nearest lists, then run refinement rounds side by
side. With strict reductions every round is bit-identical (positions, round
statistics, heat); with the default chunked sums positions agree to 1e-9 of
the layout's extent."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(kind):
    from grapher_b200 import graphs
    if kind == "grid":
        a, b = graphs.grid(12, 12)
        return 144, a, b
    if kind == "ba":
        a, b = graphs.barabasi_albert(1500, 3, 5)
        return 1500, a, b
    a, b = graphs.random_connected(400, 0.02, 3)
    return 400, np.asarray(a), np.asarray(b)


def _lockstep(ref, kind, strict, rounds=5, check=None):
    from grapher_b200 import graphs
    from grapher_b200.grip import GripRefiner
    V, a, b = _graph(kind)
    rg = ref.create_grip(V, a, b)
    rg.begin()
    row, col = graphs.to_csr(V, a, b)
    g = GripRefiner(row, col)
    g.set_strict_reductions(strict)
    layers = 0
    try:
        while True:
            act = rg.active()
            off, kv, kd = rg.knn()
            g.set_positions(rg.positions())
            g.set_layer(rg.layer, act, off, kv, kd)
            for _ in range(rounds):
                s_ref = rg.refine()
                s_gpu = g.refine_round()
                check(rg, g, act, s_ref, s_gpu)
            layers += 1
            if rg.layer == 0:
                break
            rg.next_stage()
    finally:
        g.close()
        rg.close()
    return layers


@pytest.mark.parametrize("kind", ["grid", "ba", "random"])
def test_rounds_bit_identical_with_strict_reductions(ref, kind):
    def check(rg, g, act, s_ref, s_gpu):
        assert np.array_equal(rg.positions(), g.positions())
        assert np.array_equal(s_ref, s_gpu[:3])
        h_ref, d_ref, c_ref = rg.decorators()
        h_gpu, d_gpu, c_gpu = g.decorators()
        assert np.array_equal(h_ref[act], h_gpu[act])
        assert np.array_equal(c_ref[act], c_gpu[act])
        sel = np.stack([2 * act, 2 * act + 1], 1).reshape(-1)
        assert np.array_equal(d_ref[sel], d_gpu[sel])
    assert _lockstep(ref, kind, True, check=check) >= 2


@pytest.mark.parametrize("kind", ["grid", "ba"])
def test_rounds_close_with_chunked_reductions(ref, kind):
    def check(rg, g, act, s_ref, s_gpu):
        x_ref, x_gpu = rg.positions(), g.positions()
        ext = np.abs(x_ref).max()
        assert np.abs(x_ref - x_gpu).max() <= 1e-9 * ext
        assert np.allclose(s_ref, s_gpu[:3], rtol=1e-9, atol=0)
    _lockstep(ref, kind, False, rounds=8, check=check)


def test_chunked_rounds_are_deterministic(ref):
    from grapher_b200 import graphs
    from grapher_b200.grip import GripRefiner
    V, a, b = _graph("ba")
    rg = ref.create_grip(V, a, b)
    rg.begin()
    while rg.layer > 0:
        rg.next_stage()
    act, (off, kv, kd), x0 = rg.active(), rg.knn(), rg.positions()
    row, col = graphs.to_csr(V, a, b)
    outs = []
    for _ in range(2):
        g = GripRefiner(row, col)
        g.set_positions(x0)
        g.set_layer(0, act, off, kv, kd)
        for _ in range(10):
            g.refine_round()
        outs.append(g.positions())
        g.close()
    rg.close()
    assert np.array_equal(outs[0], outs[1])


def test_grip_argument_checks():
    from grapher_b200 import graphs
    from grapher_b200._native import GvizCudaError
    from grapher_b200.grip import GripRefiner
    a, b = graphs.grid(4, 4)
    row, col = graphs.to_csr(16, a, b)
    g = GripRefiner(row, col)
    with pytest.raises(GvizCudaError):      # no layer yet
        g.refine_round()
    off = np.array([0, 1], np.uint64)
    with pytest.raises(GvizCudaError):      # active vertex out of range
        g.set_layer(0, np.array([16], np.uint32), off, np.array([1], np.uint32),
                    np.array([1], np.uint32))
    with pytest.raises(GvizCudaError):      # k-nearest vertex out of range
        g.set_layer(0, np.array([0], np.uint32), off, np.array([99], np.uint32),
                    np.array([1], np.uint32))
    g.set_layer(0, np.array([0, 1, 2], np.uint32), np.array([0, 0, 0, 0], np.uint64),
                np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert np.all(np.isfinite(g.refine_round()))
    g.close()
