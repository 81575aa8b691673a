"""gvizCudaForceRunHost: n steps end to end over a host position buffer, the
positions copied to the device before every step and back after it, with the
copies of consecutive steps pipelined. Its results must be those of n
gvizCudaForceStepHost calls, bit for bit, from page-locked and from pageable
host memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _layout(precision):
    from grapher_b200 import ForceLayout, graphs
    a, b = graphs.grid(180, 180)  # 32,400 vertices: every copy is cut in pieces
    V = 180 * 180
    row, col = graphs.to_csr(V, a, b)
    lay = ForceLayout(row, col, model=1)
    lay.set_params(theta=0.8, precision=precision, gravityK=1.0)
    lay.begin(0, positions=graphs.randomize_positions(V, 1000.0, 11))
    return lay


def _stats(lay):
    s = lay.last_stats[0]
    return (s.maxDisp, s.speed, s.meanAttractive, s.meanRepulsive, s.meanGravity)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("pinned", [True, False])
def test_run_host_matches_step_host(precision, pinned):
    import torch
    steps = 6
    ref = _layout(precision)
    x_ref = ref.positions()
    for _ in range(steps):
        md_ref = ref.step_host(x_ref)
    st_ref = _stats(ref)

    lay = _layout(precision)
    x0 = lay.positions()
    if pinned:
        buf = torch.empty(x0.size, dtype=torch.float64, pin_memory=True)
        xy = buf.numpy()
    else:
        xy = np.empty_like(x0)
    xy[:] = x0
    md = lay.run_host(xy, steps)
    assert md == md_ref
    assert _stats(lay) == st_ref
    assert np.array_equal(xy, x_ref)
    assert np.array_equal(lay.positions(), x_ref)
    ref.close()
    lay.close()


def test_run_host_zero_steps_keeps_positions():
    lay = _layout(0)
    xy = lay.positions().copy()
    before = xy.copy()
    lay.run_host(xy, 0)
    assert np.array_equal(xy, before)
    assert np.array_equal(lay.positions(), before)
    lay.close()
