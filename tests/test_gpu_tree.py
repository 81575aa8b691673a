"""Device quadtree vs the reference quadtree: every point must sit in a leaf
with the same depth and quadrant path (bit-exact membership), and every
compressed cell must carry the reference node's mass and point count exactly
and its centre of mass to FP64 rounding."""
import numpy as np
import pytest

from helpers import golden

pytestmark = pytest.mark.gpu

COM_RTOL = 1e-12  # running mean (reference) vs bottom-up sum (device), FP64


def point_layout(pts, mass, k=1, graph_offsets=None):
    """LinLog layout with no edges whose degree array gives mass = 1 + deg."""
    from grapher_b200 import ForceLayout
    V = len(mass)
    row = np.zeros(V + 1, np.uint64)
    col = np.zeros(0, np.uint32)
    deg = (np.asarray(mass) - 1.0).astype(np.uint64)
    lay = ForceLayout(row, col, model=1, degree=deg, graph_offsets=graph_offsets)
    lay.set_params(nodesPerCell=k)
    lay.set_positions(np.asarray(pts, np.float64).reshape(-1))
    return lay


def check_cells(nd, ref_nodes, pts_scale):
    keys = {(int(d), int(h), int(l)): i for i, (d, h, l) in
            enumerate(zip(ref_nodes["depth"], ref_nodes["hi"], ref_nodes["lo"]))}
    for i in range(len(nd["depth"])):
        key = (int(nd["depth"][i]), int(nd["hi"][i]), int(nd["lo"][i]))
        assert key in keys, f"cell {key} has no reference node"
        j = keys[key]
        assert nd["mass"][i] == ref_nodes["mass"][j]
        assert nd["count"][i] == ref_nodes["count"][j]
        tol = COM_RTOL * max(pts_scale, 1.0)
        assert abs(nd["comX"][i] - ref_nodes["comX"][j]) <= tol
        assert abs(nd["comY"][i] - ref_nodes["comY"][j]) <= tol


@pytest.mark.parametrize("name", ["qt_uniform3000", "qt_duplicates"])
def test_membership_matches_reference_golden(name):
    g = golden(name)
    for k in g["ks"]:
        k = int(k)
        lay = point_layout(g["pts"], g["mass"], k)
        d, hi, lo, _ = lay.tree_leaves()
        assert np.array_equal(d, g[f"k{k}_leafDepth"]), f"k={k}"
        assert np.array_equal(hi, g[f"k{k}_pathHi"]) and np.array_equal(lo, g[f"k{k}_pathLo"])
        ref_nodes = {key: g[f"k{k}_node_{key}"] for key in
                     ("depth", "hi", "lo", "mass", "comX", "comY", "count")}
        check_cells(lay.tree_nodes(), ref_nodes, float(np.abs(g["pts"]).max()))
        lay.close()


def _cases():
    rng = np.random.default_rng(7)
    yield "uniform", rng.uniform(-1000, 1000, (5000, 2))
    blobs = [rng.normal(c, s, (400, 2)) for c, s in
             [((0, 0), 1e-3), ((50, -20), 1.0), ((-300, 400), 1e-6), ((1e3, 1e3), 30.0)]]
    yield "clusters", np.concatenate(blobs)
    yield "offset", rng.uniform(-1, 1, (2000, 2)) * 5.0 + 1e6
    yield "tiny_span", rng.uniform(-1e-10, 1e-10, (50, 2))
    yield "line", np.stack([np.linspace(-1, 1, 1000), np.zeros(1000)], 1)
    base = rng.uniform(-10, 10, (300, 2))
    yield "deep_runs", np.concatenate([base, base[:100] + 1e-8, base[:50] + 2e-8, base[:20]])
    yield "one_point", np.array([[3.0, 4.0]])
    yield "two_equal", np.array([[2.0, 2.0], [2.0, 2.0]])
    yield "all_origin", np.zeros((64, 2))


@pytest.mark.parametrize("k", [1, 2, 4])
@pytest.mark.parametrize("case", [c[0] for c in _cases()])
def test_membership_matches_oracle(oracle, case, k):
    pts = dict(_cases())[case]
    mass = 1.0 + (np.arange(len(pts)) % 5).astype(np.float64)
    od, ohi, olo, _ = oracle.quadtree_leaves(pts, mass, k)
    lay = point_layout(pts, mass, k)
    d, hi, lo, _ = lay.tree_leaves()
    assert np.array_equal(d, od)
    assert np.array_equal(hi, ohi) and np.array_equal(lo, olo)
    check_cells(lay.tree_nodes(), oracle.quadtree_nodes(pts, mass, k), float(np.abs(pts).max()))
    lay.close()


def test_forest_membership_matches_each_graph(oracle):
    rng = np.random.default_rng(3)
    sizes = [1, 2, 37, 500, 3, 1200, 64]
    pts = [rng.normal(0, 10 ** rng.uniform(-3, 3), (n, 2)) for n in sizes]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    allp = np.concatenate(pts)
    mass = np.ones(len(allp))
    lay = point_layout(allp, mass, 1, graph_offsets=offs)
    d, hi, lo, _ = lay.tree_leaves()
    for g, p in enumerate(pts):
        od, ohi, olo, _ = oracle.quadtree_leaves(p, np.ones(len(p)), 1)
        s = slice(int(offs[g]), int(offs[g + 1]))
        assert np.array_equal(d[s], od) and np.array_equal(hi[s], ohi) and np.array_equal(lo[s], olo)
    lay.close()


@pytest.mark.parametrize("k", [1, 4])
def test_membership_with_many_sort_and_scan_tiles(oracle, k):
    """300,000 points: the radix sort's passes run over 74 tiles of 4,096 keys
    and the scans over 147 tiles of 2,048, so every tile's offsets come from
    the look-back over the tiles before it."""
    rng = np.random.default_rng(11)
    pts = np.concatenate([rng.uniform(-1000, 1000, (250000, 2)),
                          rng.normal(0, 1e-2, (50000, 2))])
    mass = 1.0 + (np.arange(len(pts)) % 7).astype(np.float64)
    od, ohi, olo, _ = oracle.quadtree_leaves(pts, mass, k)
    lay = point_layout(pts, mass, k)
    d, hi, lo, _ = lay.tree_leaves()
    assert np.array_equal(d, od)
    assert np.array_equal(hi, ohi) and np.array_equal(lo, olo)
    check_cells(lay.tree_nodes(), oracle.quadtree_nodes(pts, mass, k), 1000.0)
    lay.close()


def test_forest_of_many_graphs(oracle):
    """9,000 graphs of 1 to 39 points: the scan over the graphs' node counts
    runs over several tiles (more than one block's worth of entries)."""
    rng = np.random.default_rng(5)
    sizes = rng.integers(1, 40, 9000)
    pts = [rng.uniform(-10, 10, (int(n), 2)) * 10 ** rng.uniform(-2, 2) for n in sizes]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    allp = np.concatenate(pts)
    lay = point_layout(allp, np.ones(len(allp)), 1, graph_offsets=offs)
    d, hi, lo, _ = lay.tree_leaves()
    for g, p in enumerate(pts):
        od, ohi, olo, _ = oracle.quadtree_leaves(p, np.ones(len(p)), 1)
        s = slice(int(offs[g]), int(offs[g + 1]))
        assert np.array_equal(d[s], od) and np.array_equal(hi[s], ohi) and np.array_equal(lo[s], olo)
    lay.close()
