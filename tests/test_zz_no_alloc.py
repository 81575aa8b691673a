"""The allocation-free speed update (gvizCudaFa2SpeedUpdateNoAlloc) against
the handle-based step it is a variant of.

It serves callers that must not allocate device memory while they run, e.g.
a render loop stepping the layout every frame, or a program whose GPU memory
belongs to another allocator. The handle-based step sums swing and traction
in a buffer it allocated; this entry point keeps those partial sums in an
array built into the library. Same inputs, same arithmetic, same order of
the sums, so the results must be bit-identical to the FP64 step's, on two
calls in a row (the second call reuses the array the first one left
behind).
This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from helpers import cfg, csr_of, make_layout

pytestmark = pytest.mark.gpu


def test_speed_update_without_allocation_matches_step():
    import torch

    from grapher_b200 import _native as N
    from grapher_b200 import graphs

    a, b = graphs.barabasi_albert(20000, 3, 5)
    V = 20000
    row, col = csr_of(V, a, b)
    c = cfg(model=1, theta=0.8, gravity=1.0, precision="fp64")
    lay = make_layout(row, col, c)
    lay.begin(3)
    for _ in range(3):
        lay.step()
    sf_prev, speed0, eff0 = lay.fa2_state()
    lay.step()
    sf_new, speed1, eff1 = lay.fa2_state()
    swing_ref = lay.forces()["swing"]
    lay.close()

    dev = torch.device("cuda:0")
    d_sf = torch.tensor(sf_new, dtype=torch.float64, device=dev)
    d_old = torch.tensor(sf_prev, dtype=torch.float64, device=dev)
    mass = 1.0 + np.diff(row).astype(np.float64)
    d_mass = torch.tensor(mass, dtype=torch.float64, device=dev)
    d_swing = torch.zeros(V, dtype=torch.float64, device=dev)
    lib = N.lib()
    for call in range(2):
        d_state = torch.tensor([speed0[0], eff0[0]], dtype=torch.float64, device=dev)
        d_swing.zero_()
        torch.cuda.synchronize()
        rc = lib.gvizCudaFa2SpeedUpdateNoAlloc(
            C.c_void_p(d_sf.data_ptr()), C.c_void_p(d_old.data_ptr()),
            C.c_void_p(d_mass.data_ptr()), V, 1.0, C.c_void_p(d_swing.data_ptr()),
            C.c_void_p(d_state.data_ptr()), None)
        assert rc == 0, N.lib().gvizCudaErrorString(rc)
        torch.cuda.synchronize()
        got = d_state.cpu().numpy()
        assert got[0] == speed1[0] and got[1] == eff1[0], (call, got, speed1, eff1)
        assert np.array_equal(d_swing.cpu().numpy(), swing_ref), call


def test_speed_update_without_allocation_rejects_oversize():
    from grapher_b200 import _native as N
    lib = N.lib()
    # beyond 4096 chunks of 2048 vertices: refused before touching memory
    rc = lib.gvizCudaFa2SpeedUpdateNoAlloc(C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                           4096 * 2048 + 1, 1.0, None, C.c_void_p(16), None)
    assert rc == -9  # GVIZ_CUDA_ERR_LIMIT
