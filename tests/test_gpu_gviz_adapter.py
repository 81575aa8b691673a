"""The drop-in switch, end to end: a real gviz embedder (the reference built
from source) gets gvizCudaForceAttach, then front-end style
gvizEmbeddedGraphInvokeAction("forceEmbedder.step") calls step on the GPU.
A twin embedder with the same graph, configuration and seed steps on the CPU;
both must stay together (FP64 path: 1e-9 relative; FP32: layout-level)."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "grapher_b200", "lib", "libgvizcuda_gviz.so")


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32),
                ("syncScratch", C.c_int32), ("strictReductions", C.c_int32)]


@pytest.fixture(scope="module")
def glue(ref):
    if not os.path.exists(ADAPTER):
        pytest.skip("gviz glue was not built (needs gviz's headers at build time)")
    lib = C.CDLL(ADAPTER)
    lib.gvizCudaForceAttach.argtypes = [C.c_void_p, C.POINTER(Options)]
    lib.gvizCudaForceEmbedderStep.restype = C.c_double
    lib.gvizCudaForceEmbedderStep.argtypes = [C.c_void_p]
    lib.gvizCudaForceEmbedderRun.argtypes = [C.c_void_p, C.c_size_t, C.c_double]
    lib.gvizCudaForceDetach.argtypes = [C.c_void_p]
    lib.gvizCudaForceEmbedderLastError.argtypes = [C.c_void_p]
    lib.gvizCudaForceEmbedderRunBatch.argtypes = [C.POINTER(C.c_void_p), C.c_size_t,
                                                  C.c_size_t, C.c_double,
                                                  C.POINTER(Options),
                                                  C.POINTER(C.c_uint64)]
    return lib


def twins(ref, model, params, box, seed, n=400):
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(n, 3, 21) if model == 1 else graphs.random_connected(n, 0.01, 4)
    cpu = ref.create_edges(n, a, b, model)
    gpu = ref.create_edges(n, a, b, model)
    for r in (cpu, gpu):
        r.configure(params, box)
        r.begin(seed)
    return cpu, gpu


@pytest.mark.parametrize("model", [0, 1])
def test_action_registry_switch_fp64(ref, glue, model):
    from oracle.bindings import make_params
    p = make_params(model=model, theta=0.8, gravity=0.5 if model else 0.0,
                    radius_base=0.5, radius_per_degree=0.3, prevent_overlap=bool(model))
    cpu, gpu = twins(ref, model, p, 50.0, 9)
    opt = Options(0, 1, 1, 1)
    assert glue.gvizCudaForceAttach(gpu.state_ptr(), C.byref(opt)) == 0
    for s in range(12):
        if s == 6:  # live toggle through the other action, on both
            cpu.invoke_toggle_overlap()
            gpu.invoke_toggle_overlap()
        if s >= 6:
            # with overlap prevention on, a pair whose gap sits at zero takes
            # the saturated branch in one twin and not the other, and free
            # runs then part ways chaotically: each step starts the GPU twin
            # from the CPU twin's positions and FA2 state instead
            sc = cpu.state()
            gpu.set_positions(cpu.positions())
            gpu.set_fa2_state(sc["structForce"], sc["speed"], sc["efficiency"])
        assert cpu.invoke_step_action() == 0 and gpu.invoke_step_action() == 0
        # free-running twins: last-bit centre-of-mass differences grow a few
        # bits per step, so the bound loosens after the first steps
        pc, pg = cpu.positions(), gpu.positions()
        scale = np.abs(pc).max()
        if s < 6:
            assert np.abs(pc - pg).max() <= (1e-9 if s < 5 else 1e-6) * scale, s
        else:
            d = np.abs(pc - pg) / scale
            assert np.median(d) <= 1e-12 and np.quantile(d, 0.999) <= 1e-9, s
    sc, sg = cpu.state(), gpu.state()
    assert sc["iteration"] == sg["iteration"] == 12
    assert abs(sc["speed"] - sg["speed"]) <= 1e-3 * sc["speed"]
    assert abs(sc["lastMaxDisp"] - sg["lastMaxDisp"]) <= 1e-3 * sc["lastMaxDisp"]
    fs = np.abs(sg["structForce"] - sc["structForce"]) / np.abs(sc["structForce"]).max()
    assert np.median(fs) <= 1e-8 and np.quantile(fs, 0.99) <= 1e-3
    hc, hg = cpu.stats(), gpu.stats()
    assert hc.shape == hg.shape == (12, 5)
    np.testing.assert_allclose(hg[:5], hc[:5], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(hg, hc, rtol=1e-3, atol=1e-12)
    # restart through Begin, then keep stepping through the action
    cpu.begin(5)
    gpu.begin(5)
    for _ in range(3):
        cpu.invoke_step_action()
        gpu.invoke_step_action()
    assert np.abs(cpu.positions() - gpu.positions()).max() <= 1e-9 * np.abs(cpu.positions()).max()
    assert glue.gvizCudaForceEmbedderLastError(gpu.state_ptr()) == 0
    # Run on the device (the loop stays resident) against the reference's
    # Run from the same state: a few rounds follow the reference; longer
    # free runs part ways (see above), so those only keep the bookkeeping
    sc = cpu.state()
    gpu.set_positions(cpu.positions())
    gpu.set_fa2_state(sc["structForce"], sc["speed"], sc["efficiency"])
    rc = cpu.run(3, 1e-12)
    rg = glue.gvizCudaForceEmbedderRun(gpu.state_ptr(), 3, 1e-12)
    assert rc == rg == 3
    pc, pg = cpu.positions(), gpu.positions()
    dp = np.abs(pc - pg) / np.abs(pc).max()
    assert np.median(dp) <= 1e-9 and np.quantile(dp, 0.99) <= 1e-6
    rc = cpu.run(40, 1e-12)
    rg = glue.gvizCudaForceEmbedderRun(gpu.state_ptr(), 40, 1e-12)
    assert rc == rg == 40
    assert cpu.state()["iteration"] == gpu.state()["iteration"]
    assert cpu.stats().shape == gpu.stats().shape
    # detach hands the action back to the CPU step
    glue.gvizCudaForceDetach(gpu.state_ptr())
    before = gpu.positions()
    gpu.invoke_step_action()
    assert np.any(gpu.positions() != before)
    cpu.close()
    gpu.close()


def test_action_registry_switch_fp32(ref, glue):
    from oracle.bindings import make_params
    p = make_params(model=1, theta=0.8, gravity=1.0, radius_base=1.0, radius_per_degree=0.5,
                    prevent_overlap=True)
    cpu, gpu = twins(ref, 1, p, 100.0, 3, n=2000)
    opt = Options(0, 0, 0, 0)
    assert glue.gvizCudaForceAttach(gpu.state_ptr(), C.byref(opt)) == 0
    x0 = cpu.positions()
    cpu.invoke_step_action()
    gpu.invoke_step_action()
    d_c = (cpu.positions() - x0).reshape(-1, 2)
    d_g = (gpu.positions() - x0).reshape(-1, 2)
    e = np.linalg.norm(d_c - d_g, axis=1) / np.linalg.norm(d_c, axis=1)
    assert np.median(e) <= 1e-5 and np.quantile(e, 0.99) <= 1e-3
    assert gpu.state()["iteration"] == 1 and gpu.stats().shape == (1, 5)
    glue.gvizCudaForceDetach(gpu.state_ptr())
    cpu.close()
    gpu.close()


def _forest(ref, params, seeds):
    """Reference embedders of several small graphs (random trees, grids,
    ER), configured alike and begun."""
    from grapher_b200 import graphs
    out = []
    for i, seed in enumerate(seeds):
        kind = i % 3
        if kind == 0:
            V = 150 + 40 * i
            a, b = graphs.random_connected(V, 0.0, seed)
        elif kind == 1:
            a, b = graphs.grid(9 + i, 9 + i)
            V = (9 + i) ** 2
        else:
            V = 300
            a, b = graphs.erdos_renyi(V, 600, seed)
        r = ref.create_edges(V, a, b, 0)
        r.configure(params, 0.0)
        r.begin(seed)
        out.append(r)
    return out


@pytest.mark.parametrize("prec", [0, 1])
def test_run_batch_matches_single_runs(ref, glue, prec):
    """gvizCudaForceEmbedderRunBatch lays n embedders out in one handle and
    writes back what n separate Runs write; per-graph trees, speeds and
    convergence make it equal, bit for bit, to attaching each one alone."""
    from oracle.bindings import make_params
    p = make_params(model=0, theta=0.7)
    seeds = [11, 12, 13, 14, 15]
    batch, single = _forest(ref, p, seeds), _forest(ref, p, seeds)
    opt = Options(0, prec, 1, 0)
    ptrs = (C.c_void_p * len(batch))(*[r.state_ptr() for r in batch])
    rounds = (C.c_uint64 * len(batch))()
    assert glue.gvizCudaForceEmbedderRunBatch(ptrs, len(batch), 25, 1e-9, C.byref(opt),
                                              rounds) == 0
    assert list(rounds) == [25] * len(batch)
    for r, b in zip(single, batch):
        assert glue.gvizCudaForceAttach(r.state_ptr(), C.byref(opt)) == 0
        n = glue.gvizCudaForceEmbedderRun(r.state_ptr(), 25, 1e-9)
        glue.gvizCudaForceDetach(r.state_ptr())
        sb, ss = b.state(), r.state()
        assert n == 25
        assert np.array_equal(b.positions(), r.positions())
        assert sb["iteration"] == ss["iteration"] == 25
        assert sb["speed"] == ss["speed"] and sb["lastMaxDisp"] == ss["lastMaxDisp"]
        assert np.array_equal(sb["structForce"], ss["structForce"])
        assert b.stats().shape == (25, 5) and np.array_equal(b.stats(), r.stats())
    for r in batch + single:
        r.close()


def test_run_batch_follows_the_cpu(ref, glue):
    """FP64 batch against the reference's own Run on twins: the first steps
    agree to 1e-9."""
    from oracle.bindings import make_params
    p = make_params(model=0, theta=0.7)
    seeds = [21, 22, 23]
    gpu, cpu = _forest(ref, p, seeds), _forest(ref, p, seeds)
    opt = Options(0, 1, 1, 1)
    ptrs = (C.c_void_p * len(gpu))(*[r.state_ptr() for r in gpu])
    assert glue.gvizCudaForceEmbedderRunBatch(ptrs, len(gpu), 3, 1e-12, C.byref(opt),
                                              None) == 0
    for g, c in zip(gpu, cpu):
        c.run(3, 1e-12)
        pc, pg = c.positions(), g.positions()
        assert np.abs(pc - pg).max() <= 1e-9 * np.abs(pc).max()
        np.testing.assert_allclose(g.stats(), c.stats(), rtol=1e-9, atol=1e-12)
        assert g.state()["iteration"] == c.state()["iteration"] == 3
    for r in gpu + cpu:
        r.close()


def test_run_batch_rejects_mixed_configurations(ref, glue):
    from oracle.bindings import make_params
    a = _forest(ref, make_params(model=0, theta=0.7), [31])
    b = _forest(ref, make_params(model=0, theta=0.9), [32])
    ptrs = (C.c_void_p * 2)(a[0].state_ptr(), b[0].state_ptr())
    assert glue.gvizCudaForceEmbedderRunBatch(ptrs, 2, 5, 1e-9, None, None) < 0
    assert a[0].state()["iteration"] == 0
    for r in a + b:
        r.close()


def test_grip_action_switch_bit_identical(ref, glue):
    """gvizCudaGripAttach takes over "grip.refineRound": a GRIP state refined
    through the action on the GPU (strict reductions) stays bit-identical to
    a twin refined by the reference on the CPU, across every layer (gviz's
    own NextStage places each layer and builds its k-nearest lists), with the
    same lastRoundStats and round counter; after detach, CPU rounds on it
    continue identically (the decorators were written back).

    The check runs in a fresh process (tests/grip_glue_check.py), apart
    from the glue's attach registry of the other tests. Both twins clear the
    BFS stamps the reference allocates without clearing
    (src/embedders/gvizGRIPEmbedder.c:253) before Begin, so they build the
    same filtration (tests/test_grip_ref.py pins that)."""
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "grip_glue_check.py")],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().splitlines()[-1] == "OK", out.stdout[-2000:]


def test_learned_walk_through_the_action(ref, glue):
    """The learned walk behind the drop-in switch: the caller turns it on
    through the attached handle and "forceEmbedder.step" runs it; the
    embedder's own Barnes-Hut toggle (gvizForceEmbedderSetBarnesHutEnabled)
    holds it off while Barnes-Hut is off (an exact step, no error) and it
    comes back with Barnes-Hut; once the handle's judge falls back to the
    plain walk, it stays off."""
    from oracle.bindings import make_params

    from grapher_b200 import _native as N
    from grapher_b200.farfield import FarFieldModel
    L = N.lib()
    glue.gvizCudaForceEmbedderHandle.restype = C.c_void_p
    glue.gvizCudaForceEmbedderHandle.argtypes = [C.c_void_p]
    p = make_params(model=1, theta=1.0, gravity=1.0)
    lrn, pln = twins(ref, 1, p, 100.0, 3, n=3000)
    opt = Options(0, 0, 0, 0)
    assert glue.gvizCudaForceAttach(lrn.state_ptr(), C.byref(opt)) == 0
    assert glue.gvizCudaForceAttach(pln.state_ptr(), C.byref(opt)) == 0
    h = C.c_void_p(glue.gvizCudaForceEmbedderHandle(lrn.state_ptr()))
    model = FarFieldModel(seed=4)
    model.set_weights(np.random.default_rng(6).normal(0, 0.05, model.nparams).astype(np.float32))
    assert L.gvizCudaForceSetFarFieldModel(h, model.h) == 0

    def far_field():
        q = N.ForceParams()
        assert L.gvizCudaForceGetParams(h, C.byref(q)) == 0
        return q

    q = far_field()
    q.farField, q.farCellGroups = 1, 1
    assert L.gvizCudaForceSetParams(h, C.byref(q)) == 0
    x0 = lrn.positions()
    lrn.invoke_step_action()
    pln.invoke_step_action()
    d_l = (lrn.positions() - x0).reshape(-1, 2)
    d_p = (pln.positions() - x0).reshape(-1, 2)
    e = np.linalg.norm(d_l - d_p, axis=1) / np.linalg.norm(d_p, axis=1)
    assert np.all(np.isfinite(d_l)) and glue.gvizCudaForceEmbedderLastError(lrn.state_ptr()) == 0
    assert far_field().farField == 1 and lrn.state()["iteration"] == 1
    assert 0.0 < np.median(e) < 0.05, np.median(e)   # the learned walk ran, close to plain
    lrn.set_barnes_hut(False)
    before = lrn.positions()
    lrn.invoke_step_action()
    assert glue.gvizCudaForceEmbedderLastError(lrn.state_ptr()) == 0
    assert far_field().farField == 0 and np.any(lrn.positions() != before)
    lrn.set_barnes_hut(True)
    lrn.invoke_step_action()
    assert far_field().farField == 1
    # a judge that no network can satisfy sends the layout back to the plain walk
    assert L.gvizCudaForceSetFarJudge(h, 1, 256, 1.0, 1e-9, 1) == 0
    lrn.invoke_step_action()
    assert far_field().farField == 0
    lrn.set_barnes_hut(False)
    lrn.invoke_step_action()
    lrn.set_barnes_hut(True)
    lrn.invoke_step_action()
    assert far_field().farField == 0 and glue.gvizCudaForceEmbedderLastError(lrn.state_ptr()) == 0
    assert lrn.state()["iteration"] == 6
    for r in (lrn, pln):
        glue.gvizCudaForceDetach(r.state_ptr())
    model.close()
    lrn.close()
    pln.close()
