"""FP64 CPU oracle of the warm-start network (6 -> 64 -> 64 -> 1, SiLU).

TEST INFRASTRUCTURE ONLY: checks the device forward/backward kernels (lp_mlp.cu).  Same flat
weight layout as lp_mlp.cuh; loss = mean over samples of (out - y)^2.
"""

from __future__ import annotations

import numpy as np

IN, H = 6, 64
W1 = 0
B1 = W1 + H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NW = B3 + 1


def unpack(w: np.ndarray):
    w = np.asarray(w, dtype=np.float64)
    return (w[W1:B1].reshape(H, IN), w[B1:W2], w[W2:B2].reshape(H, H), w[B2:W3], w[W3:B3], w[B3])


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(w: np.ndarray, x: np.ndarray) -> np.ndarray:
    w1, b1, w2, b2, w3, b3 = unpack(w)
    h1 = silu(x @ w1.T + b1)
    h2 = silu(h1 @ w2.T + b2)
    return h2 @ w3 + b3


def bf16(a) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward_bf16(w: np.ndarray, x: np.ndarray) -> np.ndarray:
    """The tensor-core inference of lp_mlp.cuh with its roundings made explicit and the rest in
    FP64: inputs split into BF16 hi + lo, W1 and W2 in BF16, the first hidden layer rounded to
    BF16 after SiLU, the second hidden layer and the output layer unrounded."""
    w32 = np.asarray(w, dtype=np.float32)
    x32 = np.asarray(x, dtype=np.float32)
    hi = bf16(x32)
    lo = bf16(x32 - hi)
    w1 = bf16(w32[W1:B1]).astype(np.float64).reshape(H, IN)
    w2 = bf16(w32[W2:B2]).astype(np.float64).reshape(H, H)
    b1, b2 = w32[B1:W2].astype(np.float64), w32[B2:W3].astype(np.float64)
    w3, b3 = w32[W3:B3].astype(np.float64), float(w32[B3])
    z1 = hi.astype(np.float64) @ w1.T + lo.astype(np.float64) @ w1.T + b1
    h1 = bf16(silu(z1).astype(np.float32)).astype(np.float64)
    h2 = silu(h1 @ w2.T + b2)
    return h2 @ w3 + b3


def loss_grad(w: np.ndarray, x: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(w)
    n = len(y)
    z1 = x @ w1.T + b1
    h1 = silu(z1)
    z2 = h1 @ w2.T + b2
    h2 = silu(z2)
    out = h2 @ w3 + b3
    e = out - y
    loss = float(np.mean(e * e))
    g3 = 2.0 * e / n
    dz2 = (g3[:, None] * w3[None, :]) * silu_grad(z2)
    dz1 = (dz2 @ w2) * silu_grad(z1)
    g = np.zeros(NW)
    g[W1:B1] = (dz1.T @ x).ravel()
    g[B1:W2] = dz1.sum(0)
    g[W2:B2] = (dz2.T @ h1).ravel()
    g[B2:W3] = dz2.sum(0)
    g[W3:B3] = h2.T @ g3
    g[B3] = g3.sum()
    return loss, g


def finite_difference(w: np.ndarray, x: np.ndarray, y: np.ndarray, idx, eps: float = 1e-6) -> np.ndarray:
    w = np.asarray(w, dtype=np.float64)
    out = []
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        out.append((loss_grad(wp, x, y)[0] - loss_grad(wm, x, y)[0]) / (2 * eps))
    return np.array(out)
