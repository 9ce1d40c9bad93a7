"""CPU oracle of the parameter-predictor network (test infrastructure only).

A float64 numpy restatement of the 16 -> 64 -> 64 -> 5 GELU perceptron of
vortexpasta.jl_b200/csrc/mlp.cu with the same flat parameter layout
[W1 (64x16), b1, W2 (64x64), b2, W3 (5x64), b3] and the same loss
sum_o w_o (y_o - t_o)^2 averaged over the batch.  Used by the tests to check the CUDA forward
pass and the CUDA gradients (and, through finite differences, this module's own backward pass).
The network has no counterpart in the reference; the GELU is 0.5 z (1 + erf(z / sqrt 2))
(Hendrycks & Gimpel 2016).
"""

from __future__ import annotations

import math

import numpy as np

IN, HID, OUT = 16, 64, 5
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)), ("b3", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)

_erf = np.vectorize(math.erf)


def unpack(p):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    Z1 = X @ w["W1"].T + w["b1"]
    H1 = gelu(Z1)
    Z2 = H1 @ w["W2"].T + w["b2"]
    H2 = gelu(Z2)
    Y = H2 @ w["W3"].T + w["b3"]
    return Y, (X, Z1, H1, Z2, H2)


def loss_and_grad(p, X, T, wts=None):
    """Loss and its gradient (flat, same layout as the parameters)."""
    w = unpack(p)
    wts = np.ones(OUT) if wts is None else np.asarray(wts, dtype=np.float64)
    Y, (X, Z1, H1, Z2, H2) = forward(p, X)
    n = X.shape[0]
    D = Y - np.asarray(T, dtype=np.float64)
    loss = float((wts * D * D).sum() / n)
    dY = 2.0 * wts * D / n
    g = {"W3": dY.T @ H2, "b3": dY.sum(0)}
    dZ2 = (dY @ w["W3"]) * gelu_grad(Z2)
    g["W2"], g["b2"] = dZ2.T @ H1, dZ2.sum(0)
    dZ1 = (dZ2 @ w["W2"]) * gelu_grad(Z1)
    g["W1"], g["b1"] = dZ1.T @ X, dZ1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])
