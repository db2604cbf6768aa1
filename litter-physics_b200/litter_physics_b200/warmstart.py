"""Learned warm start of the Herschel-Bulkley return: data collection and device training.

The plain Newton solver logs (trial stress, yield stress, consistency, flow index, shear
modulus, dt) -> returned stress for every yielded particle while a simulation runs
(`Simulation.enable_newton_log`).  Training turns each record into the network's six features
(the device feature map of lp_mlp.cuh, restated in numpy) and the target logit(t) with
t = (sigma - sigma_y) / (sigma_tr - sigma_y), then runs the library's own forward/backward/Adam
kernels (`lp_mlp_train`).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

NW = 4673


def features(raw: np.ndarray) -> np.ndarray:
    """Six features per return problem; raw columns: trial, yield, K, n, mu, dt (any float dtype)."""
    r = raw.astype(np.float64)
    trial, ys, k, n, mu, dt = (r[:, i] for i in range(6))
    a = np.maximum((trial - ys) / k, 1e-300)
    b = np.maximum(3.0 * mu * dt / k, 1e-300)
    la, lb = np.log(a), np.log(b)
    f = np.stack([la / 8.0, lb / 8.0, n, (lb + (1.0 / n - 1.0) * la) / 8.0, 1.0 / (3.0 * n), np.log(n)], axis=1)
    return f.astype(np.float32)


def targets(raw: np.ndarray, sigma: np.ndarray) -> np.ndarray:
    """logit of the root fraction t in (0, 1)."""
    r = raw.astype(np.float64)
    t = (sigma.astype(np.float64) - r[:, 1]) / (r[:, 0] - r[:, 1])
    t = np.clip(t, 1e-6, 1.0 - 1e-6)
    return np.log(t / (1.0 - t)).astype(np.float32)


def valid(raw: np.ndarray, sigma: np.ndarray) -> np.ndarray:
    r = raw.astype(np.float64)
    ok = np.isfinite(r).all(axis=1) & np.isfinite(sigma) & (r[:, 0] > r[:, 1]) & (r[:, 2] > 0)
    t = (sigma - r[:, 1]) / np.where(r[:, 0] > r[:, 1], r[:, 0] - r[:, 1], 1.0)
    return ok & (t > 0.0) & (t < 1.0)


def init_weights(seed: int = 0) -> np.ndarray:
    w = np.zeros(NW, dtype=np.float32)
    check(lib().lp_mlp_init(w.ctypes.data_as(C.POINTER(C.c_float)), NW, seed))
    return w


def train(x: np.ndarray, y: np.ndarray, epochs: int = 8, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          weights: np.ndarray | None = None) -> tuple[np.ndarray, float]:
    """Train on (features, logit targets) with the device kernels; returns (weights, final loss)."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(y))
    xs = np.ascontiguousarray(x[order], dtype=np.float32)
    ys = np.ascontiguousarray(y[order], dtype=np.float32)
    w = init_weights(seed) if weights is None else np.ascontiguousarray(weights, dtype=np.float32).copy()
    loss = C.c_float()
    F = C.POINTER(C.c_float)
    check(lib().lp_mlp_train(w.ctypes.data_as(F), NW, xs.ctypes.data_as(F), ys.ctypes.data_as(F), len(ys), epochs,
                             batch, lr, C.byref(loss)))
    return w, float(loss.value)


def predict(w: np.ndarray, x: np.ndarray, tensor_cores: bool = False) -> np.ndarray:
    """Network output per feature row: the FP32 training arithmetic, or (tensor_cores) the BF16
    tensor-core inference the solver's warm start runs."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.zeros(len(x), dtype=np.float32)
    F = C.POINTER(C.c_float)
    fn = lib().lp_mlp_forward_mma if tensor_cores else lib().lp_mlp_forward
    check(fn(np.ascontiguousarray(w, dtype=np.float32).ctypes.data_as(F), NW, x.ctypes.data_as(F), len(x),
             y.ctypes.data_as(F)))
    return y


def loss_grad(w: np.ndarray, x: np.ndarray, y: np.ndarray) -> tuple[float, np.ndarray]:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    g = np.zeros(NW, dtype=np.float32)
    loss = C.c_float()
    F = C.POINTER(C.c_float)
    check(lib().lp_mlp_loss_grad(np.ascontiguousarray(w, dtype=np.float32).ctypes.data_as(F), NW,
                                 x.ctypes.data_as(F), y.ctypes.data_as(F), len(y), C.byref(loss),
                                 g.ctypes.data_as(F)))
    return float(loss.value), g


def collect(sim, steps: int, capacity: int = 4_000_000) -> tuple[np.ndarray, np.ndarray]:
    """Run `steps` substeps of `sim` with the Newton log on; returns (raw inputs, returned stress)."""
    sim.enable_newton_log(capacity)
    t = sim.time + steps * sim.spec.max_dt
    sim.advance_to(t)
    raw, sigma = sim.read_newton_log(capacity)
    sim.enable_newton_log(0)
    return raw, sigma


def dataset(raw: np.ndarray, sigma: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    ok = valid(raw, sigma)
    return features(raw[ok]), targets(raw[ok], sigma[ok])
