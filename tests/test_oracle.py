"""Pins the oracle (oracle/gviz_oracle.c) before it is trusted as the checker:
against the reference's own known-answer tests, against golden fixtures made
by the reference compiled from source, and (when that build is present in
this container) against the live reference, bit for bit."""
import numpy as np
import pytest

from helpers import cfg, csr_of, degree_mass, golden, golden_cfg, oracle_params


# --- known answers from tests/core/gvizVecTests.c:66-117 -------------------

def test_pair_fr_att_known_answer(oracle):
    # gvizVecTests.c:71-76: (0,0)->(3,4), k=5 gives (3,4)
    np.testing.assert_allclose(oracle.pair("fr_att", [0.0, 0.0], [3.0, 4.0], 5.0), [3.0, 4.0], atol=1e-12)


def test_pair_fr_rep_known_answer(oracle):
    # gvizVecTests.c:79-84: u=(2,0), k=1, no radius -> (-0.5, 0)
    np.testing.assert_allclose(oracle.pair("fr_rep", [0.0, 0.0], [2.0, 0.0], 1.0, 0.0, 100.0), [-0.5, 0.0], atol=1e-12)


def test_pair_fr_rep_radius_sum(oracle):
    # gvizVecTests.c:89-95: radiusSum 1 -> gap 1 -> (-1, 0)
    np.testing.assert_allclose(oracle.pair("fr_rep", [0.0, 0.0], [2.0, 0.0], 1.0, 1.0, 100.0), [-1.0, 0.0], atol=1e-12)


def test_pair_fr_rep_overlap_saturates(oracle):
    # gvizVecTests.c:100-106: gap -1 -> k^2*C = 10 along -(1,0)
    np.testing.assert_allclose(oracle.pair("fr_rep", [0.0, 0.0], [1.0, 0.0], 1.0, 2.0, 10.0), [-10.0, 0.0], atol=1e-12)


def test_pair_fr_rep_coincident_finite_and_bounded(oracle):
    # gvizVecTests.c:111-117: coincident -> finite, |f| = k^2 * C
    acc = oracle.pair("fr_rep", [0.0, 0.0], [0.0, 0.0], 2.0, 1.0, 10.0)
    assert np.all(np.isfinite(acc))
    assert abs(np.linalg.norm(acc) - 40.0) < 1e-9


def test_coincident_direction_antisymmetric(oracle):
    for i, j in [(0, 1), (5, 9), (1000, 3)]:
        a = np.array(oracle.coincident_dir(i, j))
        b = np.array(oracle.coincident_dir(j, i))
        assert np.allclose(a, -b, atol=0) and abs(np.linalg.norm(a) - 1.0) < 1e-15


def test_pair_linlog(oracle):
    acc = oracle.pair("linlog_att", [0.0, 0.0], [3.0, 4.0])
    np.testing.assert_allclose(acc, np.log(6.0) / 5.0 * np.array([3.0, 4.0]), rtol=1e-15)
    acc = oracle.pair("linlog_rep", [0.0, 0.0], [2.0, 0.0], 3.0, 4.0, 0.0, 100.0)
    np.testing.assert_allclose(acc, [-6.0, 0.0], rtol=1e-15)


# --- quadtree known answers, tests/ds/gvizQuadtreeTests.c ----------------

def _leaves(oracle, pts, mass, k=1):
    return oracle.quadtree_leaves(np.array(pts, float), np.array(mass, float), k)


def test_quadtree_quadrant_order(oracle):
    # gvizQuadtreeTests.c:53-104: NW, NE, SW, SE children hold points 0..3
    d, hi, lo, _ = _leaves(oracle, [[-5, 5], [5, 5], [-5, -5], [5, -5]], [1, 1, 1, 1])
    assert list(d) == [1, 1, 1, 1]
    assert [int(h >> 62) for h in hi] == [0, 1, 2, 3]


def test_quadtree_nodes_per_cell(oracle):
    # gvizQuadtreeTests.c:106-123: k=3 keeps 3 points in the root leaf
    d, _, _, n = _leaves(oracle, [[1, 1], [2, 2], [3, 3]], [1, 1, 1], k=3)
    assert list(d) == [0, 0, 0] and n == 1


def test_quadtree_com_known_answer(oracle):
    # gvizQuadtreeTests.c:154-178: COM 24/5, mass 5
    nd = oracle.quadtree_nodes(np.array([[0, 0], [10, 0], [0, 10], [10, 10], [4, 4]], float), np.ones(5))
    root = np.where(nd["depth"] == 0)[0][0]
    assert nd["comX"][root] == 24.0 / 5.0 and nd["comY"][root] == 24.0 / 5.0 and nd["mass"][root] == 5


def test_quadtree_weighted_and_zero_mass(oracle):
    # gvizQuadtreeTests.c:272-343
    nd = oracle.quadtree_nodes(np.array([[0, 0], [10, 0]], float), np.array([1.0, 3.0]))
    r = np.where(nd["depth"] == 0)[0][0]
    assert nd["mass"][r] == 4.0 and nd["comX"][r] == 7.5 and nd["comY"][r] == 0.0
    nd = oracle.quadtree_nodes(np.array([[0, 0], [5, 5], [10, 10]], float), np.array([0.0, 0.0, 2.0]))
    r = np.where(nd["depth"] == 0)[0][0]
    assert nd["mass"][r] == 2.0 and nd["comX"][r] == 10.0 and nd["comY"][r] == 10.0


def test_quadtree_duplicates_terminate(oracle):
    # gvizQuadtreeTests.c:125-148: duplicates land in one overflow leaf
    d, _, _, _ = _leaves(oracle, [[2, 2], [2, 2], [2, 2]], [1, 1, 1])
    assert len(set(d.tolist())) == 1 and d[0] == 30  # halfSize 1 -> 2^-30 <= 1e-9


# --- golden fixtures made by the reference ------------------------------

@pytest.mark.parametrize("name", ["qt_uniform3000", "qt_duplicates"])
def test_oracle_quadtree_matches_golden(oracle, name):
    g = golden(name)
    for k in g["ks"]:
        d, hi, lo, _ = oracle.quadtree_leaves(g["pts"], g["mass"], int(k))
        assert np.array_equal(d, g[f"k{k}_leafDepth"])
        assert np.array_equal(hi, g[f"k{k}_pathHi"]) and np.array_equal(lo, g[f"k{k}_pathLo"])
        nd = oracle.quadtree_nodes(g["pts"], g["mass"], int(k))
        ref_keys = {(int(a), int(b), int(c)): i for i, (a, b, c) in
                    enumerate(zip(g[f"k{k}_node_depth"], g[f"k{k}_node_hi"], g[f"k{k}_node_lo"]))}
        assert len(ref_keys) == len(nd["depth"])
        for i, key in enumerate(zip(nd["depth"], nd["hi"], nd["lo"])):
            j = ref_keys[(int(key[0]), int(key[1]), int(key[2]))]
            assert nd["mass"][i] == g[f"k{k}_node_mass"][j]
            assert nd["comX"][i] == g[f"k{k}_node_comX"][j]
            assert nd["count"][i] == g[f"k{k}_node_count"][j]


@pytest.mark.parametrize("name", ["traj_grid32_fr_theta05", "traj_rc300_linlog_theta08_grav_overlap",
                                  "traj_rc200_fr_exact", "traj_rc500_linlog_theta12_k3"])
def test_oracle_trajectory_bit_exact_vs_golden(oracle, name):
    g = golden(name)
    c = golden_cfg(g)
    V = int(g["V"])
    row, col = csr_of(V, g["ea"], g["eb"])
    deg, mass = degree_mass(row, c["model"])
    p = oracle_params(c)
    pos = g["x0"].copy()
    sf = np.zeros(2 * V)
    ss = np.array([1.0, 1.0])
    for s in range(g["pos"].shape[0]):
        out = oracle.step((row, col), mass, deg, p, pos, sf, ss)
        assert out["maxDisp"] == g["maxDisp"][s]
        assert np.array_equal(pos, g["pos"][s])
        assert np.array_equal(sf, g["structForce"][s])
        assert np.array_equal(ss, g["speedState"][s])
        assert np.array_equal(out["stats"], g["stats"][s])


def test_oracle_vs_live_reference(oracle, ref):
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(2000, 3, 11)
    c = cfg(model=1, theta=0.9, gravity=0.5, radius_base=0.5, radius_per_degree=0.3,
            prevent_overlap=True)
    r = ref.create_edges(2000, a, b, 1)
    r.configure(oracle_params(c), 500.0)
    r.begin(13)
    row, col = r.csr()
    deg, mass = r.degree_mass()
    pos = r.positions().copy()
    sf = np.zeros(4000)
    ss = np.array([1.0, 1.0])
    for _ in range(10):
        r.step()
        oracle.step((row, col), mass, deg, oracle_params(c), pos, sf, ss)
    assert np.array_equal(pos, r.positions())
