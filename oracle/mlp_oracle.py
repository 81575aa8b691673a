"""FP64 NumPy restatement of the far-field MLP (10 -> 64 -> 64 -> 2, ReLU),
its weighted mean squared error and the gradient, in the padded master
layout of libgvizcuda (w1t[64][16], b1[64], w2t[64][64], b2[64], w3t[8][64],
b3[8]).

TEST INFRASTRUCTURE ONLY: the checker for the tensor-core training and
inference kernels. With bf16=True it rounds weights, inputs and the hidden
activations (and the backward activation gradients) to BF16 where the
kernels store them in BF16, and keeps everything else in FP64, so the
remaining difference to the GPU is its FP32 accumulation order.
"""
from __future__ import annotations

import numpy as np

IN, INP, HID, OUT, OUTP = 10, 16, 64, 2, 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * INP
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUTP * HID
PAD = OFF_B3 + OUTP


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    W1 = w[OFF_W1:OFF_B1].reshape(HID, INP)[:, :IN]      # [64][10]
    b1 = w[OFF_B1:OFF_W2]
    W2 = w[OFF_W2:OFF_B2].reshape(HID, HID)              # [out][in]
    b2 = w[OFF_B2:OFF_W3]
    W3 = w[OFF_W3:OFF_B3].reshape(OUTP, HID)[:OUT]       # [2][64]
    b3 = w[OFF_B3:OFF_B3 + OUT]
    return W1, b1, W2, b2, W3, b3


def forward(w, X, bf=False):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    X = r(X)
    W1, W2, W3 = r(W1), r(W2), r(W3)
    H1 = r(np.maximum(X @ W1.T + b1, 0.0))
    H2 = r(np.maximum(H1 @ W2.T + b2, 0.0))
    Y = H2 @ W3.T + b3
    return Y, (X, H1, H2, W1, W2, W3)


def loss_and_grad(w, X, T, Wt=None, bf=False):
    """Weighted mean squared error and its gradient in the padded layout."""
    n = X.shape[0]
    Wt = np.ones(n) if Wt is None else np.asarray(Wt, dtype=np.float64)
    scale = 1.0 / Wt.sum()
    Y, (Xr, H1, H2, W1, W2, W3) = forward(w, X, bf)
    E = Y - T
    loss = scale * np.sum(Wt[:, None] * E * E)
    r = bf16 if bf else (lambda a: a)
    dY = r(2.0 * scale * Wt[:, None] * E)
    g = np.zeros(PAD)
    g[OFF_B3:OFF_B3 + OUT] = dY.sum(0)
    dW3 = dY.T @ H2
    g[OFF_W3:OFF_B3].reshape(OUTP, HID)[:OUT] = dW3
    dH2 = r((dY @ W3) * (H2 > 0))
    g[OFF_B2:OFF_W3] = dH2.sum(0)
    g[OFF_W2:OFF_B2] = (dH2.T @ H1).reshape(-1)
    dH1 = r((dH2 @ W2) * (H1 > 0))
    g[OFF_B1:OFF_W2] = dH1.sum(0)
    g[OFF_W1:OFF_B1].reshape(HID, INP)[:, :IN] = dH1.T @ Xr
    return loss, g


def random_weights(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, scale, PAD)
    w[OFF_W1:OFF_B1].reshape(HID, INP)[:, IN:] = 0.0
    w[OFF_W3:OFF_B3].reshape(OUTP, HID)[OUT:] = 0.0
    w[OFF_B3 + OUT:] = 0.0
    return w
