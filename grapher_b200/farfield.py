"""The learned far-field correction, end to end over libgvizcuda:

    model = FarFieldModel(seed=1)
    X, T, W = harvest_training_set(layout, theta=1.2, targets=..., snapshots=...)
    model.train(X, T, W, epochs=40)
    model.attach(layout)             # the walk now applies the correction
    layout.set_params(theta=1.2, farField=1)
    errors = force_error(layout, targets)   # judged against exact FP64 forces

Training pairs are harvested from the layout's own tree (gvizCudaForce-
HarvestFarField): exact FP64 force of every accepted cell's points against
its monopole. The network predicts that relative correction in units of
s^2 = (h/d)^2, its leading order, and the walk multiplies its output by s^2.
Sample weights (|F_mono| / |F_v|)^2 s^4 make the loss the sum of squared
per-cell contributions to each target's relative force error.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

IN = 10


class FarFieldModel:
    def __init__(self, seed=1, device=0):
        self.L = N.lib()
        h = C.c_void_p()
        N.check(self.L.gvizCudaMlpCreate(C.byref(h), device, seed), "gvizCudaMlpCreate")
        self.h = h
        self.nparams = int(self.L.gvizCudaMlpParamCount())

    def set_training_kernels(self, tcgen05=True):
        """Gradient and training kernels: tcgen05 (default) or mma.sync."""
        N.check(self.L.gvizCudaMlpSetTrainingKernels(self.h, 1 if tcgen05 else 0),
                "gvizCudaMlpSetTrainingKernels")

    def weights(self):
        w = np.zeros(self.nparams, np.float32)
        N.check(self.L.gvizCudaMlpGetWeights(self.h, N.ptr(w, C.c_float)), "gvizCudaMlpGetWeights")
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        N.check(self.L.gvizCudaMlpSetWeights(self.h, N.ptr(w, C.c_float)), "gvizCudaMlpSetWeights")

    @staticmethod
    def _prep(X, T=None, W=None):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, IN)
        T = None if T is None else np.ascontiguousarray(T, dtype=np.float32).reshape(-1, 2)
        W = None if W is None else np.ascontiguousarray(W, dtype=np.float32)
        return X, T, W

    def gradient(self, X, T, W=None):
        X, T, W = self._prep(X, T, W)
        g = np.zeros(self.nparams, np.float32)
        loss = C.c_float()
        N.check(self.L.gvizCudaMlpGradient(self.h, N.ptr(X, C.c_float), N.ptr(T, C.c_float),
                                           N.ptr(W, C.c_float), X.shape[0],
                                           N.ptr(g, C.c_float), C.byref(loss)),
                "gvizCudaMlpGradient")
        return loss.value, g

    def train(self, X, T, W=None, epochs=30, batch=4096, lr=2e-3, seed=7):
        X, T, W = self._prep(X, T, W)
        losses = np.zeros(epochs, np.float32)
        N.check(self.L.gvizCudaMlpTrain(self.h, N.ptr(X, C.c_float), N.ptr(T, C.c_float),
                                        N.ptr(W, C.c_float), X.shape[0], epochs, batch, lr,
                                        seed, N.ptr(losses, C.c_float)), "gvizCudaMlpTrain")
        return losses

    def infer(self, X):
        X, _, _ = self._prep(X)
        Y = np.zeros((X.shape[0], 2), np.float32)
        N.check(self.L.gvizCudaMlpInfer(self.h, N.ptr(X, C.c_float), X.shape[0],
                                        N.ptr(Y, C.c_float)), "gvizCudaMlpInfer")
        return Y

    def attach(self, layout):
        N.check(self.L.gvizCudaForceSetFarFieldModel(layout.h, self.h),
                "gvizCudaForceSetFarFieldModel")

    def close(self):
        if getattr(self, "h", None):
            self.L.gvizCudaMlpDestroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def harvest(layout, targets, theta, cap=None):
    """(features, targets, |F_mono|, vertex) of every cell the learned walk
    accepts for the listed target vertices at the current positions."""
    L = N.lib()
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    cap = cap or 256 * max(1, t.shape[0])
    while True:
        X = np.zeros((cap, IN), np.float32)
        T = np.zeros((cap, 2), np.float32)
        M = np.zeros(cap, np.float32)
        V = np.zeros(cap, np.uint32)
        n = L.gvizCudaForceHarvestFarField(layout.h, N.ptr(t, C.c_uint32), t.shape[0], theta,
                                           N.ptr(X, C.c_float), N.ptr(T, C.c_float),
                                           N.ptr(M, C.c_float), N.ptr(V, C.c_uint32), cap)
        N.check(int(n), "gvizCudaForceHarvestFarField")
        if n <= cap:
            return X[:n], T[:n], M[:n], V[:n]
        cap = int(n)


def harvest_training_set(layout, theta, targets):
    """Training set for the network of the learned walk, which predicts the
    relative correction in units of s^2 = (h/d)^2 (feature 8) and has its
    output multiplied by s^2 in the walk: features, targets T / s^2 and
    weights W s^4 with W = (|F_mono| / |F_v|)^2 and F_v the exact FP64
    repulsion of the sample's target vertex, so that the loss is the sum of
    squared per-cell contributions to each target's relative force error."""
    X, T, M, V = harvest(layout, targets, theta)
    exact = layout.exact_repulsion(targets)
    fv = dict(zip(np.asarray(targets, np.uint32).tolist(), np.linalg.norm(exact, axis=1)))
    den = np.array([fv[int(v)] for v in V])
    W = (M / np.maximum(den, 1e-30)) ** 2
    s2 = np.maximum(X[:, 8].astype(np.float64), 1e-12)
    return X, (T / s2[:, None]).astype(np.float32), (W * s2 * s2).astype(np.float32)


def force_error(layout, targets, exact=None):
    """Per-target relative error of the layout's current repulsion (its
    configuration as set: plain or learned, any theta) against exact FP64
    all-pairs repulsion: returns (rms, max, per-target errors)."""
    t = np.asarray(targets, dtype=np.uint32)
    if exact is None:
        exact = layout.exact_repulsion(t)
    rep = layout.repulsion()[t]
    e = np.linalg.norm(rep - exact, axis=1) / np.maximum(np.linalg.norm(exact, axis=1), 1e-300)
    return float(np.sqrt(np.mean(e * e))), float(e.max()), e
