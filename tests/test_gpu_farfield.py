"""The learned far-field correction: the BF16 tensor-core training and
inference kernels against the FP64 NumPy oracle (oracle/mlp_oracle.py, with
BF16 rounding emulated where the kernels store BF16), the harvested training
targets against the analytic quadrupole term, and what the trained network
gains over the same walk without it, judged against exact FP64 all-pairs
repulsion."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(seed=3):
    from grapher_b200.farfield import FarFieldModel
    return FarFieldModel(seed=seed)


def _batch(n=1000, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(0.0, 0.5, (n, 10)).astype(np.float32)
    T = rng.normal(0.0, 0.2, (n, 2)).astype(np.float32)
    W = rng.uniform(0.5, 2.0, n).astype(np.float32)
    return X, T, W


@pytest.mark.parametrize("tc", [True, False], ids=["tcgen05", "mma_sync"])
@pytest.mark.parametrize("n", [1, 17, 1000, 5000])
def test_gradient_matches_oracle(n, tc):
    """Both training paths (tcgen05 with TMEM accumulators, and mma.sync)
    against the FP64 oracle with BF16 rounding where the kernels round."""
    from oracle import mlp_oracle as MO
    m = _model()
    m.set_training_kernels(tc)
    w = m.weights().astype(np.float64)
    X, T, W = _batch(n)
    loss, g = m.gradient(X, T, W)
    lo, go = MO.loss_and_grad(w, X.astype(np.float64), T.astype(np.float64),
                              W.astype(np.float64), bf=True)
    # FP32 accumulation in a different order is the only difference left
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    cos = float(np.dot(g, go) / (np.linalg.norm(g) * np.linalg.norm(go)))
    assert cos > 0.99999
    assert np.linalg.norm(g - go) <= 2e-3 * np.linalg.norm(go)
    # padding entries of the master layout never receive gradient
    assert np.all(g[go == 0.0] == 0.0)


def test_training_paths_agree():
    """The tcgen05 and mma.sync gradients of one batch (several CTAs, a
    ragged last tile) agree up to FP32 summation order."""
    X, T, W = _batch(3000, 5)
    m = _model(2)
    m.set_training_kernels(True)
    l1, g1 = m.gradient(X, T, W)
    m.set_training_kernels(False)
    l2, g2 = m.gradient(X, T, W)
    assert abs(l1 - l2) <= 1e-5 * abs(l2)
    assert np.linalg.norm(g1 - g2) <= 1e-3 * np.linalg.norm(g2)


def test_gradient_unweighted_equals_unit_weights():
    m = _model()
    X, T, _ = _batch(300, 1)
    l1, g1 = m.gradient(X, T, None)
    l2, g2 = m.gradient(X, T, np.ones(300, np.float32))
    assert l1 == l2 and np.array_equal(g1, g2)


def test_inference_matches_oracle():
    from oracle import mlp_oracle as MO
    m = _model(5)
    X, _, _ = _batch(4099, 2)   # not a multiple of the 32-row tiles
    Y = m.infer(X)
    Yo, _ = MO.forward(m.weights().astype(np.float64), X.astype(np.float64), bf=True)
    assert np.max(np.abs(Y - Yo)) <= 1e-5 + 1e-4 * np.max(np.abs(Yo))


def test_weights_round_trip_and_validation():
    from grapher_b200._native import GvizCudaError
    m = _model()
    w = np.random.default_rng(4).normal(0, 0.1, m.nparams).astype(np.float32)
    m.set_weights(w)
    assert np.array_equal(m.weights(), w)
    with pytest.raises(GvizCudaError):
        m.gradient(np.zeros((0, 10), np.float32), np.zeros((0, 2), np.float32))


@pytest.mark.parametrize("tc", [True, False], ids=["tcgen05", "mma_sync"])
def test_training_fits_quadrupole_law(tc):
    """Adam over the tensor-core gradient learns the leading 1/r correction
    t = (f1, -f2) from random features."""
    m = _model(7)
    m.set_training_kernels(tc)
    rng = np.random.default_rng(8)
    X = rng.uniform(-0.3, 0.3, (20000, 10)).astype(np.float32)
    T = np.stack([X[:, 1], -X[:, 2]], 1).astype(np.float32)
    losses = m.train(X, T, None, epochs=30, batch=2048, lr=3e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.05 * losses[0]
    assert m.gradient(X, T)[0] < 1e-2 * float(np.mean(np.sum(T * T, 1)))


# ----------------------------------------------------------------- layouts
def _ba_layout(V=1 << 15, steps=20, theta=0.5):
    from grapher_b200 import ForceLayout, graphs
    a, b = graphs.barabasi_albert(V, 4, 7)
    row, col = graphs.to_csr(V, a, b)
    lay = ForceLayout(row, col, model=1)
    lay.set_params(theta=theta, gravityK=1.0, preventOverlap=0)
    lay.begin(0, positions=graphs.randomize_positions(V, 1000.0, 7))
    for _ in range(steps):
        lay.step()
    return lay


@pytest.fixture(scope="module")
def trained():
    """A 32K-vertex BA layout (LinLog + gravity) and a model trained on its
    own harvested pairs at theta = 1.2 from two snapshots."""
    from grapher_b200.farfield import harvest_training_set
    lay = _ba_layout()
    rng = np.random.default_rng(0)
    Xs, Ts, Ws = [], [], []
    for _ in range(2):
        for _ in range(5):
            lay.step()
        t = np.sort(rng.choice(lay.V, 4096, replace=False)).astype(np.uint32)
        X, T, W = harvest_training_set(lay, 1.2, t)
        Xs.append(X), Ts.append(T), Ws.append(W)
    m = _model(3)
    m.train(np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ws), epochs=40,
            batch=4096, lr=2e-3, seed=2)
    for _ in range(5):
        lay.step()
    targets = np.sort(rng.choice(lay.V, 2048, replace=False)).astype(np.uint32)
    return lay, m, targets, lay.exact_repulsion(targets)


def _nrms(lay, targets, exact):
    rep = lay.repulsion()[targets]
    return float(np.sqrt(np.sum((rep - exact) ** 2) / np.sum(exact ** 2)))


def test_harvest_targets_follow_quadrupole(trained):
    """For cells far away compared with their size the exact relative
    correction is the quadrupole term (f1, -f2) up to O((h/d)^3)."""
    from grapher_b200.farfield import harvest
    lay, _, targets, _ = trained
    X, T, M, Vx = harvest(lay, targets[:512], 1.2)
    assert len(X) > 512 and np.all(np.isfinite(X)) and np.all(np.isfinite(T))
    assert set(np.unique(Vx)) <= set(targets[:512].tolist())
    far = X[:, 0] < 0.25
    quad = np.stack([X[:, 1], -X[:, 2]], 1)
    res = np.sqrt(np.mean(np.sum((T[far] - quad[far]) ** 2, 1)))
    tr = np.sqrt(np.mean(np.sum(T[far] ** 2, 1)))
    assert res < 0.35 * tr
    assert np.all(M > 0)


def test_harvest_is_deterministic(trained):
    """Pairs come back in one canonical order (target vertex, then cell),
    whatever order the GPU found them in, so training on them is
    repeatable."""
    from grapher_b200.farfield import harvest
    lay, _, targets, _ = trained
    a = harvest(lay, targets[:256], 1.0)
    b = harvest(lay, targets[:256], 1.0, cap=7)   # too small: retried inside
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.all(np.diff(a[3].astype(np.int64)) >= 0)


def test_zero_model_is_the_plain_walk(trained):
    """With all weights zero the learned walk adds nothing; below
    theta = 1/sqrt(2) no cell can contain its target, so the per-target
    learned walk takes the same terms as the plain walk (the same count) and
    the forces agree up to the order of the compensated FP32 sums (the plain
    walk expands the tree in rounds, the per-target walk in preorder)."""
    lay, _, targets, _ = trained
    z = _model(1)
    z.set_weights(np.zeros(z.nparams, np.float32))
    lay.set_params(theta=0.6, farField=0)
    plain = lay.repulsion()
    n_plain = lay.count_interactions()[0]
    z.attach(lay)
    for spread in (0.0, 0.25):
        lay.set_params(theta=0.6, farField=1, farGroupSpread=spread)
        got = lay.repulsion()
        assert lay.count_interactions()[0] == n_plain
        d = np.linalg.norm(got - plain, axis=1)
        n = np.linalg.norm(plain, axis=1)
        assert float(np.max(d / np.maximum(n, 1e-30))) < 1e-5
    lay.set_params(farField=0)


@pytest.mark.parametrize("spread", [0.0, 0.25])
def test_learned_correction_beats_monopole(trained, spread):
    """The gain of the trained network: at theta = 1.2 its force error
    against exact FP64 repulsion is well below that of the same walk with
    the monopole alone."""
    lay, m, targets, exact = trained
    z = _model(1)
    z.set_weights(np.zeros(z.nparams, np.float32))
    z.attach(lay)
    lay.set_params(theta=1.2, farField=1, farGroupSpread=spread)
    e_mono = _nrms(lay, targets, exact)
    m.attach(lay)
    e_mlp = _nrms(lay, targets, exact)
    lay.set_params(farField=0)
    e_plain = _nrms(lay, targets, exact)
    assert e_mlp < 0.5 * e_mono, (e_mlp, e_mono)
    assert e_mlp < 0.5 * e_plain, (e_mlp, e_plain)


def test_group_rows_cut_evaluations(trained):
    lay, m, targets, exact = trained
    m.attach(lay)
    lay.set_params(theta=1.2, farField=1, farGroupSpread=0.0)
    g0, l0 = lay.count_far_rows()
    e0 = _nrms(lay, targets, exact)
    lay.set_params(farGroupSpread=0.25)
    g1, l1 = lay.count_far_rows()
    e1 = _nrms(lay, targets, exact)
    lay.set_params(farField=0)
    assert g0 == 0 and l0 > 0
    assert g1 > 0 and g1 + l1 < 0.75 * l0
    assert e1 < 1.5 * e0


def test_learned_steps_and_graph_replay(trained):
    """Steps with the correction on run inside the captured step graph and
    are deterministic: two layouts from the same state agree exactly."""
    from grapher_b200 import graphs
    _, m, _, _ = trained
    outs = []
    for _ in range(2):
        lay = _ba_layout(V=4096, steps=3)
        m.attach(lay)
        lay.set_params(theta=1.2, farField=1)
        for _ in range(5):
            lay.step()
        outs.append(lay.positions())
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])


# ------------------------------------------------------- cell-group walk
def test_cell_groups_partition_the_vertices(trained):
    """Every vertex is in exactly one group of 1..32 targets, and no vertex
    of another group lies strictly inside a group's bounding box: a group
    is a cell of the tree, or sibling cells whose quadrant rectangle holds
    no other sibling."""
    lay, _, _, _ = trained
    gof, n = lay.far_groups()
    assert n > 0 and np.all(gof < n)
    sizes = np.bincount(gof, minlength=n)
    assert sizes.min() >= 1 and sizes.max() <= 32
    assert sizes.sum() == lay.V
    x = lay.positions().reshape(-1, 2)
    lo = np.full((n, 2), np.inf)
    hi = np.full((n, 2), -np.inf)
    np.minimum.at(lo, gof, x)
    np.maximum.at(hi, gof, x)
    bad = 0
    for s0 in range(0, lay.V, 2048):
        p = x[s0:s0 + 2048, None, :]
        inside = np.all((p > lo[None]) & (p < hi[None]), axis=2)
        inside[np.arange(inside.shape[0]), gof[s0:s0 + 2048]] = False
        bad += int(inside.sum())
    assert bad == 0


def test_cell_group_walk_is_exact_without_acceptance(trained):
    """With a zero model and theta so small that no cell is accepted, each
    target sums the pair terms of every other vertex: the exact repulsion
    up to the rounding of plain FP32 sums of 32K terms, so every node is
    reached from every group."""
    lay, _, targets, exact = trained
    z = _model(1)
    z.set_weights(np.zeros(z.nparams, np.float32))
    z.attach(lay)
    lay.set_params(theta=1e-4, farField=1, farCellGroups=1)
    e = _nrms(lay, targets, exact)
    lay.set_params(theta=1.0, farField=0, farCellGroups=0)
    assert e < 2e-4, e


def test_cell_group_correction_beats_monopole(trained):
    """The trained network's gain in the cell-group walk at theta = 1.0:
    well below the same walk with the monopole alone, and below the plain
    walk at the same theta."""
    lay, m, targets, exact = trained
    z = _model(1)
    z.set_weights(np.zeros(z.nparams, np.float32))
    z.attach(lay)
    lay.set_params(theta=1.0, farField=1, farCellGroups=1)
    e_mono = _nrms(lay, targets, exact)
    m.attach(lay)
    e_mlp = _nrms(lay, targets, exact)
    g, _, why = lay.count_far_rows(causes=True)
    lay.set_params(farField=0, farCellGroups=0)
    e_plain = _nrms(lay, targets, exact)
    assert e_mlp < 0.6 * e_mono, (e_mlp, e_mono)
    assert e_mlp < 0.6 * e_plain, (e_mlp, e_plain)
    assert g > 0 and why[2] == lay.V   # one row per accepted cell; every target walked


def test_cell_group_steps_are_deterministic(trained):
    """Steps of the cell-group walk run in the captured step graph and do
    not depend on which warp drew which group."""
    _, m, _, _ = trained
    outs = []
    for _ in range(2):
        lay = _ba_layout(V=8192, steps=3)
        m.attach(lay)
        lay.set_params(theta=1.0, farField=1, farCellGroups=1)
        for _ in range(5):
            lay.step()
        outs.append(lay.positions())
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("theta", [1.0, 1e-4])
def test_cell_walk_in_place_subtrees_agree(trained, theta):
    """The expanding cell-group walk with a stack too small for its pushes
    walks those subtrees in place: the same decisions and the same terms, so
    the forces agree up to the order of the compensated FP32 sums, and the
    fallback really ran."""
    lay, m, targets, exact = trained
    m.attach(lay)
    lay.set_params(theta=theta, farField=1, farCellGroups=1)
    lay.set_walk_stack_cap(0)
    full = lay.repulsion()
    _, _, why_full = lay.count_far_rows(causes=True)
    lay.set_walk_stack_cap(32)
    try:
        small = lay.repulsion()
        g, _, why_small = lay.count_far_rows(causes=True)
    finally:
        lay.set_walk_stack_cap(0)
        lay.set_params(theta=1.0, farField=0, farCellGroups=0)
    assert why_small[1] > 0 and why_small[2] == lay.V and why_full[2] == lay.V
    d = np.linalg.norm(small - full, axis=1)
    n = np.linalg.norm(full, axis=1)
    assert np.all(np.isfinite(small))
    assert float(np.sqrt(np.sum(d * d) / np.sum(n * n))) < 1e-6
    assert float(np.max(d / np.maximum(n, 1e-30))) < 1e-4


def _heaviest(lay, k):
    """The k heaviest vertices (LinLog mass deg + 1, ties to the lower id)."""
    deg = np.diff(lay.row).astype(np.int64)
    return np.sort(np.lexsort((np.arange(lay.V), -deg))[:k])


def test_hub_targets_take_the_plain_walk(trained):
    """farHubTargets: the heaviest vertices' repulsion is the plain monopole
    walk's (at farHubTheta == theta the opening test is the same one; only
    the order of the FP32 sums differs) and every other vertex keeps the
    learned walk's result bit for bit."""
    lay, m, _, _ = trained
    m.attach(lay)
    k = 300
    hubs = _heaviest(lay, k)
    lay.set_params(theta=1.2, farField=1, farCellGroups=1, farHubTargets=0)
    learned = lay.repulsion()
    lay.set_params(farField=0, farCellGroups=0)
    plain = lay.repulsion()
    lay.set_params(farField=1, farCellGroups=1, farHubTargets=k, farHubTheta=1.2)
    mixed = lay.repulsion()
    again = lay.repulsion()
    lay.set_params(theta=1.0, farField=0, farCellGroups=0, farHubTargets=0)
    rest = np.ones(lay.V, bool)
    rest[hubs] = False
    assert np.array_equal(mixed[rest], learned[rest])
    d = np.linalg.norm(mixed[hubs] - plain[hubs], axis=1)
    # both sums are Kahan-compensated FP32; the hubs' terms cancel heavily
    assert np.all(d <= 1e-4 * np.linalg.norm(plain[hubs], axis=1)), d.max()
    assert not np.array_equal(mixed[hubs], learned[hubs])
    assert np.array_equal(mixed, again)   # deterministic sums


def test_hub_targets_in_a_batch(trained):
    """In a batch of layouts every hub walks its own graph's tree only: the
    heaviest vertices over the batch take the plain walk's repulsion of
    their own graph, the rest keep the learned walk's."""
    from grapher_b200 import ForceLayout, graphs
    _, m, _, _ = trained
    parts, offs, n = [], [0], 0
    for V, seed in ((3000, 11), (5000, 12)):
        a, b = graphs.barabasi_albert(V, 4, seed)
        parts.append((a + n, b + n))
        n += V
        offs.append(n)
    a = np.concatenate([p[0] for p in parts])
    b = np.concatenate([p[1] for p in parts])
    row, col = graphs.to_csr(n, a, b)
    lay = ForceLayout(row, col, model=1, graph_offsets=np.array(offs, np.uint64))
    lay.set_params(theta=1.2, gravityK=1.0)
    lay.begin(0, positions=graphs.randomize_positions(n, 1000.0, 7))
    for _ in range(5):
        lay.step()
    m.attach(lay)
    hubs = _heaviest(lay, 40)
    assert hubs.min() < offs[1] <= hubs.max()   # hubs in both graphs
    lay.set_params(farField=1, farCellGroups=1, farHubTargets=0)
    learned = lay.repulsion()
    lay.set_params(farField=0, farCellGroups=0)
    plain = lay.repulsion()
    lay.set_params(farField=1, farCellGroups=1, farHubTargets=40, farHubTheta=1.2)
    mixed = lay.repulsion()
    rest = np.ones(n, bool)
    rest[hubs] = False
    assert np.array_equal(mixed[rest], learned[rest])
    d = np.linalg.norm(mixed[hubs] - plain[hubs], axis=1)
    assert np.all(d <= 1e-4 * np.linalg.norm(plain[hubs], axis=1)), d.max()
    lay.close()


def test_hub_walk_without_acceptance_is_exact(trained):
    """At a tiny farHubTheta no cell is accepted: every hub sums the pair
    terms of all other vertices, so its frontier outgrows the block's
    shared memory and the entries beyond it are walked by their threads."""
    lay, m, targets, exact = trained
    m.attach(lay)
    hubs = _heaviest(lay, 64)
    ex = lay.exact_repulsion(hubs.astype(np.uint32))
    lay.set_params(theta=1.2, farField=1, farCellGroups=1, farHubTargets=64,
                   farHubTheta=1e-4)
    rep = lay.repulsion()[hubs]
    lay.set_params(theta=1.0, farField=0, farCellGroups=0, farHubTargets=0)
    d = np.linalg.norm(rep - ex, axis=1)
    n = np.linalg.norm(ex, axis=1)
    assert np.sqrt(np.sum(d * d) / np.sum(n * n)) < 1e-4
    assert np.all(d <= 1e-3 * n), (d / n).max()


def test_hub_targets_cut_the_weighted_error(trained):
    """The hubs carry most of LinLog's force, so a tight walk for the
    heaviest 1/64 of the vertices lowers the force-weighted error of the
    learned walk at theta = 1.2."""
    lay, m, targets, exact = trained
    m.attach(lay)
    lay.set_params(theta=1.2, farField=1, farCellGroups=1, farHubTargets=0)
    e0 = _nrms(lay, targets, exact)
    lay.set_params(farHubTargets=lay.V // 64, farHubTheta=0.35)
    e1 = _nrms(lay, targets, exact)
    lay.set_params(theta=1.0, farField=0, farCellGroups=0, farHubTargets=0)
    assert e1 < 0.9 * e0, (e1, e0)


def test_hub_steps_are_deterministic(trained):
    """Steps with the hub walk forked beside the learned walk in the
    captured step graph give the same positions on every run."""
    _, m, _, _ = trained
    outs = []
    for _ in range(2):
        lay = _ba_layout(V=8192, steps=3)
        m.attach(lay)
        lay.set_params(theta=1.2, farField=1, farCellGroups=1, farHubTargets=128,
                       farHubTheta=0.35)
        for _ in range(5):
            lay.step()
        outs.append(lay.positions())
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])


def test_far_field_argument_checks(trained):
    from grapher_b200._native import GvizCudaError
    lay = _ba_layout(V=512, steps=1)
    with pytest.raises(GvizCudaError):      # no model attached
        lay.set_params(farField=1)
    lay.set_params(farField=0)
    _, m, _, _ = trained
    m.attach(lay)
    with pytest.raises(GvizCudaError):      # the correction is FP32 only
        lay.set_params(farField=1, precision=1)
    lay.set_params(farField=0, precision=0)
    with pytest.raises(GvizCudaError):
        lay.set_params(farField=1, farGroupSpread=-1.0)
    lay.set_params(farField=0, farGroupSpread=1.0)
    with pytest.raises(GvizCudaError):
        lay.set_params(farCellGroups=2)
    lay.set_params(farCellGroups=0)
    with pytest.raises(GvizCudaError):
        lay.set_params(farHubTargets=-1)
    lay.set_params(farHubTargets=0)
    with pytest.raises(GvizCudaError):
        lay.set_params(farHubTargets=8, farHubTheta=0.0)
    lay.set_params(farHubTargets=0, farHubTheta=0.35)
    lay.set_params(farHubTargets=1 << 30)   # more than the vertices: all of them
    lay.set_params(farHubTargets=0)


# ------------------------------------------------------------ the judge
def test_judge_keeps_a_good_network_and_drops_a_bad_one(trained):
    """gvizCudaForceJudgeFarField: the learned walk is judged against the
    plain walk on sampled vertices, both against exact FP64 repulsion. The
    trained network at theta = 1.0 beats the plain walk at the same theta and
    stays on; a network with large random weights does not and the handle
    falls back to the plain walk (farField 0, later steps plain)."""
    from grapher_b200 import _native as N
    lay, m, targets, exact = trained
    m.attach(lay)
    lay.set_params(theta=1.0, farField=1, farCellGroups=1)
    lay.set_far_judge(every=0, samples=2048, plain_theta=1.0, slack=1.0, seed=5)
    le, pe, fell = lay.judge_far_field()
    assert not fell and 0 < le < pe, (le, pe)
    p = N.ForceParams()
    lay.L.gvizCudaForceGetParams(lay.h, C.byref(p))
    assert p.farField == 1
    bad = _model(9)
    bad.set_weights(np.random.default_rng(1).normal(0, 3.0, bad.nparams).astype(np.float32))
    bad.attach(lay)
    le2, pe2, fell2 = lay.judge_far_field()
    lay.L.gvizCudaForceGetParams(lay.h, C.byref(p))
    n, l_last, p_last, fell_any = lay.far_judge_status()
    lay.set_far_judge()
    lay.set_params(theta=1.0, farField=0, farCellGroups=0)
    assert fell2 and le2 > pe2 and p.farField == 0
    assert n >= 2 and fell_any and l_last == le2 and p_last == pe2
    assert abs(pe2 - pe) <= 1e-12 * pe   # the plain walk's error does not depend on the model


def test_judge_every_n_steps_falls_back_to_the_plain_walk(trained):
    """Automatic checks: with every = 3 the first learned step is checked;
    a bad network is dropped there, and the steps that follow are exactly
    the plain walk's steps from the same state."""
    lay, _, _, _ = trained
    x_s, (sf, sp, ef) = lay.positions(), lay.fa2_state()
    bad = _model(11)
    bad.set_weights(np.random.default_rng(2).normal(0, 3.0, bad.nparams).astype(np.float32))
    bad.attach(lay)
    lay.set_params(theta=0.5, farField=1, farCellGroups=1)
    lay.set_far_judge(every=3, samples=1024, plain_theta=0.5, slack=1.0, seed=3)
    for _ in range(4):
        lay.step()
    judged = lay.positions()
    n, _, _, fell = lay.far_judge_status()
    lay.set_far_judge()
    lay.set_positions(x_s)
    lay.set_fa2_state(sf, sp, ef)
    lay.set_params(theta=0.5, farField=0, farCellGroups=0)
    for _ in range(4):
        lay.step()
    plain = lay.positions()
    lay.set_positions(x_s)
    lay.set_fa2_state(sf, sp, ef)
    lay.set_params(theta=1.0)
    assert fell and n >= 1
    assert np.array_equal(judged, plain)
