"""TEST INFRASTRUCTURE ONLY: numpy forward/backward of the proposal network, for checking the
library's hand-written CUDA kernels (float64 arithmetic, weights rounded to BF16 as the library's
working copy is)."""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params, L, H):
    o = 0
    out = {}
    for name, shape in (("W1", (H, L)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (L, H)), ("b3", (L,))):
        n = int(np.prod(shape))
        out[name] = params[o:o + n].reshape(shape).astype(np.float64)
        o += n
    return out


def gelu(z):
    return 0.5 * z * (1 + erf(z / np.sqrt(2)))


def gelu_grad(z):
    return 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def forward(params, L, H, X):
    """Logits of the network in float64 with BF16-rounded weights."""
    P = unpack(params, L, H)
    W1, W2, W3 = (bf16(P[k].astype(np.float32)).astype(np.float64) for k in ("W1", "W2", "W3"))
    h1 = gelu(X.astype(np.float64) @ W1.T + P["b1"])
    h2 = gelu(h1 @ W2.T + P["b2"])
    return h2 @ W3.T + P["b3"]


def loss_and_grads(params, L, H, X, y):
    P = unpack(params, L, H)
    W1, W2, W3 = (bf16(P[k].astype(np.float32)).astype(np.float64) for k in ("W1", "W2", "W3"))
    X = X.astype(np.float64)
    B = X.shape[0]
    z1 = X @ W1.T + P["b1"]
    h1 = gelu(z1)
    z2 = h1 @ W2.T + P["b2"]
    h2 = gelu(z2)
    lg = h2 @ W3.T + P["b3"]
    mx = lg.max(1, keepdims=True)
    lse = mx[:, 0] + np.log(np.exp(lg - mx).sum(1))
    loss = float(np.mean(lse - lg[np.arange(B), y]))
    p = np.exp(lg - lse[:, None])
    p[np.arange(B), y] -= 1
    d = p / B
    g = {"W3": d.T @ h2, "b3": d.sum(0)}
    dz2 = (d @ W3) * gelu_grad(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    g["W1"], g["b1"] = dz1.T @ X, dz1.sum(0)
    flat = np.concatenate([g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3")])
    return loss, flat
