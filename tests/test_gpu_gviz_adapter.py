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
        assert cpu.invoke_step_action() == 0 and gpu.invoke_step_action() == 0
        # free-running twins: last-bit centre-of-mass differences grow a few
        # bits per step, so the bound loosens after the first steps
        pc, pg = cpu.positions(), gpu.positions()
        scale = np.abs(pc).max()
        assert np.abs(pc - pg).max() <= (1e-9 if s < 5 else 1e-6) * scale, s
    sc, sg = cpu.state(), gpu.state()
    assert sc["iteration"] == sg["iteration"] == 12
    assert abs(sc["speed"] - sg["speed"]) <= 1e-6 * sc["speed"]
    assert abs(sc["lastMaxDisp"] - sg["lastMaxDisp"]) <= 1e-6 * sc["lastMaxDisp"]
    np.testing.assert_allclose(sg["structForce"], sc["structForce"], rtol=1e-5, atol=1e-8)
    hc, hg = cpu.stats(), gpu.stats()
    assert hc.shape == hg.shape == (12, 5)
    np.testing.assert_allclose(hg[:5], hc[:5], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(hg, hc, rtol=1e-6, atol=1e-12)
    # restart through Begin, then keep stepping through the action
    cpu.begin(5)
    gpu.begin(5)
    for _ in range(3):
        cpu.invoke_step_action()
        gpu.invoke_step_action()
    assert np.abs(cpu.positions() - gpu.positions()).max() <= 1e-9 * np.abs(cpu.positions()).max()
    assert glue.gvizCudaForceEmbedderLastError(gpu.state_ptr()) == 0
    # Run on the device (the loop stays resident) against the reference's Run
    rc = cpu.run(40, 1e-12)
    rg = glue.gvizCudaForceEmbedderRun(gpu.state_ptr(), 40, 1e-12)
    assert rc == rg == 40
    # 40 free-running steps amplify last-bit differences: compare statistically
    pc, pg = cpu.positions(), gpu.positions()
    dp = np.abs(pc - pg) / np.abs(pc).max()
    assert np.median(dp) <= 1e-6 and dp.max() <= 1e-2
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
