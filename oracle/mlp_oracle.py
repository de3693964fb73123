"""FP64 restatement of the learned closure's network and features.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the GPU training
kernels (gradients) and the tensor-core inference against plain numpy.  It is
not part of the product and is never executed on the product path.

The network and features have no counterpart in the reference; they follow
cudalbm_b200/csrc/lbm_mlp.cuh (16 -> 32 -> 32 -> 1, GELU in its tanh form
0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) (Hendrycks & Gimpel 2016), features =
10 stored moments + 6 strain-rate components 3 (u_a u_b - m_ab) / (2 scale tau0),
standardised as (f - in_mean) * in_scale).
"""
from __future__ import annotations

import math

import numpy as np

WEIGHTS = ("w1", "b1", "w2", "b2", "w3", "b3")
_A, _B = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(_A * (z + _B * z ** 3)))


def gelu_grad(z):
    t = np.tanh(_A * (z + _B * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _A * (1.0 + 3.0 * _B * z * z)


def params_of(mlp) -> dict:
    """numpy views (float64) of an _lib.MLP structure."""
    p = {name: np.array(getattr(mlp, name), dtype=np.float64) for name, _ in mlp._fields_}
    p["w1"] = p["w1"].reshape(32, 16)
    p["w2"] = p["w2"].reshape(32, 32)
    return p


def features(m, tau0):
    """Features [n][16] of stored moments m [10][n], in float32 arithmetic with
    every product and difference rounded separately (as the device does)."""
    m = np.asarray(m, dtype=np.float32)
    f32 = np.float32
    r_ii = f32(1.0) / (f32(2.0) * f32(4.5) * f32(tau0))
    r_ij = f32(1.0) / (f32(2.0) * f32(9.0) * f32(tau0))
    u, v, w = m[1], m[2], m[3]
    uu = [u * u, u * v, u * w, v * v, v * w, w * w]
    r = [r_ii, r_ij, r_ij, r_ii, r_ij, r_ii]
    s = [(f32(3.0) * (uu[c] - m[4 + c])) * r[c] for c in range(6)]
    return np.concatenate([m, np.stack(s)], axis=0).T.astype(np.float32)


def _h(a):
    """Round to FP16 with saturation to the largest finite value."""
    return np.clip(np.asarray(a, np.float64), -65504.0, 65504.0).astype(np.float16).astype(np.float64)


def forward(p, feats, fp16=False):
    """Network output y [n]; fp16=True follows the tensor-core path's
    roundings (accumulation in FP64): standardised inputs and the weights of
    the two hidden layers in FP16, biases added in FP32, each hidden layer's
    pre-activation rounded to FP16 before the GELU and its activation rounded
    to FP16 after it, the output layer in FP32.  (The device evaluates the
    GELU in FP16 arithmetic, which this model rounds only once.)"""
    x = (np.asarray(feats, np.float64) - p["in_mean"]) * p["in_scale"]
    w1, w2, w3, b1, b2, b3 = p["w1"], p["w2"], p["w3"], p["b1"], p["b2"], p["b3"]
    if not fp16:
        h1 = gelu(x @ w1.T + b1)
        return gelu(h1 @ w2.T + b2) @ w3 + b3
    h1 = _h(gelu(_h(_h(x) @ _h(w1).T + b1)))
    h2 = _h(gelu(_h(h1 @ _h(w2).T + b2)))
    return h2 @ w3 + b3


def gradient(p, feats, targets):
    """Mean squared error on standardised targets clip(t)/out_scale and its
    gradient with respect to w1, b1, w2, b2, w3, b3."""
    x = (np.asarray(feats, np.float64) - p["in_mean"]) * p["in_scale"]
    t = np.clip(np.asarray(targets, np.float64), p["dtau_lo"], p["dtau_hi"]) / p["out_scale"]
    n = x.shape[0]
    z1 = x @ p["w1"].T + p["b1"]
    h1 = gelu(z1)
    z2 = h1 @ p["w2"].T + p["b2"]
    h2 = gelu(z2)
    y = h2 @ p["w3"] + p["b3"]
    e = y - t
    dy = 2.0 * e / n
    g = {"w3": h2.T @ dy, "b3": np.array(dy.sum())}
    dz2 = dy[:, None] * p["w3"][None, :] * gelu_grad(z2)
    g["w2"] = dz2.T @ h1
    g["b2"] = dz2.sum(axis=0)
    dz1 = (dz2 @ p["w2"]) * gelu_grad(z1)
    g["w1"] = dz1.T @ x
    g["b1"] = dz1.sum(axis=0)
    return g, float(np.mean(e * e))
