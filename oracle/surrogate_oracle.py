"""Oracle of the settling surrogate (test infrastructure only): the library's MLP
restated in numpy — Fourier features, hidden layers Linear + SiLU, linear output, MSE —
with its forward pass and hand-derived backward pass. With ``bf16=True`` it rounds to
BF16 (round-to-nearest-even) exactly where the library's tensor-core path stores BF16:
the features, the hidden-layer weights, the hidden activations and the back-propagated
pre-activation gradients; sums are then formed in float64, so the library's FP32
accumulation differs from it only by rounding. With ``bf16=False`` everything is float64,
which a finite-difference test checks the backward pass against."""
from __future__ import annotations

import numpy as np

N_IN, N_OUT, N_FEAT = 5, 3, 128   # default inputs, outputs, first-layer width of 5 inputs


def feature_width(nin: int, bands: int) -> int:
    """First layer's input width: nin * (1 + 2 bands) rounded up to a multiple of 128."""
    return max(128, -(-nin * (1 + 2 * bands) // 128) * 128)


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def features(u: np.ndarray, bands: int, bf16: bool = True) -> np.ndarray:
    """u_i, then sin(2^f pi u_i), cos(2^f pi u_i) for f < bands (f-major, i, sin before
    cos), zero padding to feature_width."""
    u = np.asarray(u, np.float32)
    n, nin = u.shape
    x = np.zeros((n, feature_width(nin, bands)), np.float32)
    x[:, :nin] = u
    for f in range(bands):
        a = np.float32(2.0 ** f * 3.14159265358979) * u
        for i in range(nin):
            x[:, nin + 2 * nin * f + 2 * i] = np.sin(a[:, i])
            x[:, nin + 2 * nin * f + 2 * i + 1] = np.cos(a[:, i])
    return bf16_round(x) if bf16 else x.astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(params: dict, layers: int, u, targets, bands: int, bf16: bool = True):
    """Loss and gradients (dict of the same keys as params) of the MSE on these rows."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    f64 = np.float64
    x = features(u, bands, bf16).astype(f64)
    acts, zs = [x], []
    for l in range(layers):
        W = rnd(params[f"W{l}"]).astype(f64)
        z = acts[-1] @ W.T + params[f"b{l}"].astype(f64)
        if bf16:
            z = z.astype(np.float32).astype(f64)
        zs.append(z)
        acts.append(rnd(_silu(z)).astype(f64))
    Wo = params["Wo"].astype(f64)
    y = acts[-1] @ Wo.T + params["bo"].astype(f64)
    t = np.asarray(targets, f64)
    n = y.shape[0]
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / (n * N_OUT)
    g = {"Wo": dy.T @ acts[-1], "bo": dy.sum(0)}
    dz = rnd(((dy @ Wo) * _silu_grad(zs[-1]))).astype(f64)
    for l in range(layers - 1, -1, -1):
        g[f"W{l}"] = dz.T @ acts[l]
        g[f"b{l}"] = dz.sum(0)
        if l > 0:
            W = rnd(params[f"W{l}"]).astype(f64)
            dz = rnd(((dz @ W) * _silu_grad(zs[l - 1]))).astype(f64)
    return loss, g, y


def predict(params: dict, layers: int, u, bands: int, bf16: bool = True) -> np.ndarray:
    t = np.zeros((np.asarray(u).shape[0], N_OUT))
    return forward_backward(params, layers, u, t, bands, bf16)[2]
