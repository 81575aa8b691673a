"""Pins the MLP oracle (oracle/mlp_oracle.py) before it judges the GPU
kernels: its analytic gradient against central finite differences."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(3)
    w = M.random_weights(1)
    X = rng.normal(0, 1, (40, M.IN))
    T = rng.normal(0, 0.3, (40, M.OUT))
    Wt = rng.uniform(0.5, 2.0, 40)
    loss, g = M.loss_and_grad(w, X, T, Wt)
    real = [i for i in range(M.PAD) if g[i] != 0.0]
    assert len(real) > 4000
    for i in rng.choice(real, 60, replace=False):
        e = np.zeros(M.PAD)
        e[i] = 1e-6
        lp, _ = M.loss_and_grad(w + e, X, T, Wt)
        lm, _ = M.loss_and_grad(w - e, X, T, Wt)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    from oracle.mlp_oracle import bf16
    assert bf16(1.0) == 1.0
    assert bf16(1.0 + 2 ** -9) == 1.0          # below half an ulp (2^-7)
    assert bf16(1.0 + 3 * 2 ** -9) == 1.0 + 2 ** -7
    assert bf16(-3.14159) == -3.140625
