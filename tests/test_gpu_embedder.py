"""The reference's behavioural tests (tests/embedders/gvizForceEmbedderTests.c)
re-run on the CUDA path through the ForceLayout mirror of its API."""
import math

import numpy as np
import pytest

from helpers import csr_of

pytestmark = pytest.mark.gpu


def layout(V, edges, model=0, **cfg):
    from grapher_b200 import ForceLayout
    a = np.array([e[0] for e in edges], np.uint32)
    b = np.array([e[1] for e in edges], np.uint32)
    row, col = csr_of(V, a, b)
    lay = ForceLayout(row, col, model=model)
    for k, v in cfg.items():
        getattr(lay, k)(*v) if isinstance(v, tuple) else getattr(lay, k)(v)
    return lay


def dist(p, i, j):
    return math.hypot(p[2 * i] - p[2 * j], p[2 * i + 1] - p[2 * j + 1])


def place(lay, pts):
    xy = lay.positions()
    for i, (x, y) in pts.items():
        xy[2 * i], xy[2 * i + 1] = x, y
    lay.set_positions(xy)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_begin_positions_within_box(prec):
    # gvizForceEmbedderTests.c:126-149
    lay = layout(20, [(i, i + 1) for i in range(19)], set_precision=prec)
    lay.begin(42)
    p = lay.positions()
    assert np.all(np.abs(p) <= lay.box_extent)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_edge_attracts(prec):
    # :152-179
    lay = layout(2, [(0, 1)], set_precision=prec)
    lay.begin(1)
    place(lay, {0: (-50, 0), 1: (50, 0)})
    before = dist(lay.positions(), 0, 1)
    lay.step()
    assert dist(lay.positions(), 0, 1) < before


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_non_edge_repels(prec):
    # :182-208
    lay = layout(2, [], set_precision=prec)
    lay.begin(1)
    place(lay, {0: (-1, 0), 1: (1, 0)})
    lay.step()
    assert dist(lay.positions(), 0, 1) > 2.0


def test_edge_repels_when_very_close():
    # :214-241
    lay = layout(2, [(0, 1)])
    lay.begin(1)
    place(lay, {0: (-0.5, 0), 1: (0.5, 0)})
    lay.step()
    assert dist(lay.positions(), 0, 1) > 1.0


def test_radius_increases_short_range_repulsion():
    # :457-499
    plain = layout(2, [], set_barnes_hut_enabled=False)
    radial = layout(2, [], set_barnes_hut_enabled=False, configure_radius=(2.0, 0.0),
                    set_prevent_overlap_enabled=True)
    for lay in (plain, radial):
        lay.begin(1)
        place(lay, {0: (-0.5, 0), 1: (0.5, 0)})
        lay.step()
    assert dist(radial.positions(), 0, 1) > dist(plain.positions(), 0, 1)


def test_radius_formula():
    # :504-524, :532-564
    lay = layout(3, [(0, 1), (0, 2)])
    assert lay.vertex_radius(0) == 0.0
    lay.configure_radius(1.0, 2.0)
    for i in range(3):
        assert lay.vertex_radius(i) == 1.0 * (1.0 + 2.0 * math.sqrt(float(lay.degree[i])))
    lay.configure_radius(1.0, 0.5)
    r1 = lay.vertex_radius(0) / lay.vertex_radius(1)
    lay.configure_radius(20.0, 0.5)
    assert abs(lay.vertex_radius(0) / lay.vertex_radius(1) - r1) < 1e-9 and r1 > 1.0


@pytest.mark.parametrize("model", [0, 1])
def test_radius_many_steps_stay_bounded(model):
    # :576-605
    from grapher_b200 import graphs
    a, b = graphs.random_connected(60, 0.05, 7)
    lay = layout(60, list(zip(a, b)), model=model, configure_radius=(0.5, 0.3),
                 set_prevent_overlap_enabled=True)
    lay.begin(7)
    bound = 50.0 * lay.box_extent
    for _ in range(100):
        md = lay.step()
        p = lay.positions()
        assert math.isfinite(md) and np.all(np.isfinite(p)) and np.all(np.abs(p) < bound)


def test_radius_without_prevent_overlap_is_noop():
    # :610-641
    from grapher_b200 import graphs
    a, b = graphs.random_connected(30, 0.1, 5)
    e = list(zip(a, b))
    plain = layout(30, e, model=1)
    conf = layout(30, e, model=1, configure_radius=(5.0, 3.0))
    for lay in (plain, conf):
        lay.begin(11)
        for _ in range(20):
            lay.step()
    np.testing.assert_allclose(plain.positions(), conf.positions(), atol=1e-9, rtol=0)


def test_run_converges_or_stops():
    # :243-266
    from grapher_b200 import graphs
    a, b = graphs.random_connected(40, 0.05, 123)
    lay = layout(40, list(zip(a, b)))
    assert lay.run(300, 1e-6) == -1  # before Begin the reference returns -1
    lay.begin(7)
    rounds = lay.run(300, 1e-6)
    assert 0 < rounds <= 300
    assert np.all(np.isfinite(lay.positions()))
    hist = lay.stat_history()
    assert len(hist) == rounds
    if rounds < 300:
        assert hist[-1, 0] < 1e-6 and np.all(hist[:-1, 0] >= 1e-6)


def test_restart_rebuilds():
    # :268-305
    lay = layout(12, [(i, i + 1) for i in range(11)])
    lay.begin(1)
    first = lay.positions()
    lay.begin(2)
    assert np.any(np.abs(lay.positions() - first) > 1e-9)
    assert math.isfinite(lay.step())


def test_barnes_hut_tiny_theta_matches_exact_direction():
    # :316-375
    edges = [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0), (0, 3)]
    exact = layout(6, edges, set_barnes_hut_enabled=False)
    bh = layout(6, edges, configure_barnes_hut=(0.05, 1))
    exact.begin(99)
    bh.begin(99)
    before = exact.positions()
    assert np.array_equal(before, bh.positions())
    exact.step()
    bh.step()
    de = (exact.positions() - before).reshape(-1, 2)
    db = (bh.positions() - before).reshape(-1, 2)
    ne, nb = np.linalg.norm(de, axis=1), np.linalg.norm(db, axis=1)
    assert np.all(ne > 1e-9) and np.all(nb > 1e-9)
    assert np.all(np.abs(de / ne[:, None] - db / nb[:, None]) <= 0.1)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_coincident_positions_stay_finite(prec):
    # :379-408
    lay = layout(6, [(0, 1), (2, 3), (4, 5)], set_precision=prec)
    lay.begin(3)
    lay.set_positions(np.zeros(12))
    md = lay.step()
    p = lay.positions()
    assert math.isfinite(md) and np.all(np.isfinite(p))
    # the deterministic antisymmetric direction separates every pair
    q = p.reshape(-1, 2)
    assert len({(round(x, 9), round(y, 9)) for x, y in q}) == 6


def test_linlog_non_edge_repels_with_nonzero_degree():
    # :416-448
    lay = layout(3, [(0, 2), (1, 2)], model=1, configure_barnes_hut=(0.05, 1))
    lay.begin(1)
    place(lay, {0: (-1, 0), 1: (1, 0), 2: (0, 1000)})
    lay.step()
    assert dist(lay.positions(), 0, 1) > 2.0


def test_barnes_hut_disabled_still_attracts():
    # :646-679
    lay = layout(2, [(0, 1)], set_barnes_hut_enabled=False)
    lay.begin(1)
    place(lay, {0: (-50, 0), 1: (50, 0)})
    md = lay.step()
    assert math.isfinite(md) and dist(lay.positions(), 0, 1) < 100.0


def test_gravity_pulls_toward_origin():
    # :687-714
    lay = layout(2, [], configure_gravity=100.0)
    lay.begin(1)
    place(lay, {0: (100, 0), 1: (-100, 0)})
    lay.step()
    p = lay.positions()
    assert math.hypot(p[0], p[1]) < 100.0


def test_step_before_begin_and_nan_are_errors():
    from grapher_b200 import ForceLayout, GvizCudaError
    import ctypes as C
    from grapher_b200 import _native as N
    lay = layout(3, [(0, 1)])
    md = N.lib().gvizCudaForceStep(lay.h, None)
    assert md == -5  # Begin has not been called
    lay.begin(1)
    xy = lay.positions()
    xy[1] = float("nan")
    lay.set_positions(xy)
    with pytest.raises(GvizCudaError) as e:
        lay.step()
    assert e.value.code == -6
    assert lay.last_error() == -6
    del ForceLayout, C
