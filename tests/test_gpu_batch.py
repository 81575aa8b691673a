"""Batched layout (one handle, many independent graphs: a forest of per-graph
quadtrees, per-graph speed and stats) against each graph laid out alone.
Every graph's tree, traversal order, chunking and reductions are the same in
both, so the results must be identical bit for bit, in FP32 and FP64."""
import numpy as np
import pytest

from helpers import cfg, make_layout

pytestmark = pytest.mark.gpu


def small_graphs(seed=1):
    from grapher_b200 import graphs
    rng = np.random.default_rng(seed)
    out = []
    for i, V in enumerate([1, 2, 33, 300, 64, 1000, 7, 529]):
        kind = i % 3
        if kind == 0 and V >= 2:
            a, b = graphs.erdos_renyi(V, max(1, int(V * rng.uniform(1.5, 3.0))), 100 + i)
        elif kind == 1:
            a, b = graphs.random_connected(V, 0.0, 200 + i)
        else:
            s = max(1, int(round(np.sqrt(V))))
            a, b = graphs.grid(s, s)
            V = s * s
        out.append((V, a, b))
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_batch_equals_individual_layouts(prec):
    from grapher_b200 import graphs
    gs = small_graphs()
    c = cfg(model=0, theta=0.7, precision=prec)
    row, col, offs = graphs.batch(gs)
    x0 = [graphs.randomize_positions(V, 10.0, 7 + i) for i, (V, _, _) in enumerate(gs)]
    batch = make_layout(row, col, c, graph_offsets=offs)
    batch.begin(0, positions=np.concatenate(x0))
    singles = []
    for (V, a, b), x in zip(gs, x0):
        r, cc = graphs.to_csr(V, a, b)
        lay = make_layout(r, cc, c)
        lay.begin(0, positions=x)
        singles.append(lay)
    for _ in range(6):
        batch.step()
        for lay in singles:
            lay.step()
    pb = batch.positions()
    for g, lay in enumerate(singles):
        s = slice(2 * int(offs[g]), 2 * int(offs[g + 1]))
        assert np.array_equal(pb[s], lay.positions()), f"graph {g}"
        assert np.array_equal(batch.stat_history(g), lay.stat_history(0)), f"graph {g}"


def test_batch_run_stops_each_graph_on_its_own():
    from grapher_b200 import graphs
    gs = small_graphs(2)
    c = cfg(model=0, theta=0.7)
    row, col, offs = graphs.batch(gs)
    x0 = [graphs.randomize_positions(V, 10.0, 3 + i) for i, (V, _, _) in enumerate(gs)]
    batch = make_layout(row, col, c, graph_offsets=offs)
    batch.begin(0, positions=np.concatenate(x0))
    batch.run(200, 1e-3)
    rounds = batch.rounds.copy()
    for g, ((V, a, b), x) in enumerate(zip(gs, x0)):
        r, cc = graphs.to_csr(V, a, b)
        lay = make_layout(r, cc, c)
        lay.begin(0, positions=x)
        assert lay.run(200, 1e-3) == int(rounds[g]), f"graph {g}"
        s = slice(2 * int(offs[g]), 2 * int(offs[g + 1]))
        assert np.array_equal(batch.positions()[s], lay.positions())
    assert rounds.min() < rounds.max() or rounds.min() == 200


def test_walk_shapes_and_autotune_give_identical_forces():
    """The walk's launch shape (block size, static or persistent work-queue
    schedule) changes which warp runs a task, never what it computes: every
    shape gives the same forces and steps bit for bit, single and batched."""
    from grapher_b200 import graphs
    from grapher_b200._native import GvizCudaError
    gs = small_graphs(3)
    row, col, offs = graphs.batch(gs)
    x0 = np.concatenate([graphs.randomize_positions(V, 10.0, 3 + i) for i, (V, _, _) in enumerate(gs)])
    c = cfg(model=1, theta=0.8, gravity=1.0)
    ref = make_layout(row, col, c, graph_offsets=offs)
    ref.begin(0, positions=x0)
    want = ref.repulsion()
    for _ in range(3):
        ref.step()
    for threads in (64, 128, 256, 512):
        for persistent in (False, True):
            lay = make_layout(row, col, c, graph_offsets=offs)
            lay.begin(0, positions=x0)
            lay.set_walk_shape(threads, persistent)
            assert np.array_equal(lay.repulsion(), want)
            for _ in range(3):
                lay.step()
            assert np.array_equal(lay.positions(), ref.positions())
    lay = make_layout(row, col, c, graph_offsets=offs)
    lay.begin(0, positions=x0)
    threads, persistent, ms = lay.autotune()
    assert threads in (64, 128, 256, 512) and ms > 0
    t2, p2, cap = lay.walk_shape()
    assert (t2, p2) == (threads, persistent) and cap in (128, 256, 512)
    # the tuned stack: the same forces as the default shape with that stack
    chk = make_layout(row, col, c, graph_offsets=offs)
    chk.begin(0, positions=x0)
    chk.set_walk_stack_cap(cap)
    assert np.array_equal(lay.repulsion(), chk.repulsion())
    chk.close()
    with pytest.raises(GvizCudaError):
        lay.set_walk_shape(100, False)
