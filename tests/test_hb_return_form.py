"""The device's form of the Herschel-Bulkley return, restated in numpy, against the oracle's
restatement of the reference solver (constitutive.rs:280-362).

The device iterates on the excess stress x = sigma - yield and, once a Newton step's relative
change q is small, updates the flow power (x/K)^(1/n) by the factor (1 - q)^(1/n) from two short
Taylor series instead of a logarithm and an exponential.  This checks, on the CPU, that the form
is the reference's solver: the same iteration counts and the same returned stress to the
tolerance, and that the series factor is the FP64 power to rounding.
"""

from __future__ import annotations

import numpy as np

SMALL = 2.0**-7


def pow_one_minus_small(q: np.ndarray, a: np.ndarray) -> np.ndarray:
    """(1 - q)^a = exp(a log1p(-q)) from the series cut after the eighth power (FP64 FMA-free
    evaluation; the device uses FMAs, which only rounds differently)."""
    s = np.full_like(q, 1.0 / 8.0)
    for j in range(7, 0, -1):
        s = s * q + 1.0 / j
    t = -a * q * s
    e = np.full_like(q, 1.0 / 40320.0)  # 1/8!
    for k in range(7, 0, -1):
        e = e * t + 1.0 / float(np.prod(np.arange(1, k + 1)))
    return e * t + 1.0


def device_form(trial, ys, k, n, mu, dt, tol):
    """Vectorised restatement of hb_return_d: returns (sigma, iterations)."""
    vs = 3.0 * mu * dt
    ex = 1.0 / n
    lk = np.log(k)
    c1 = vs * ex
    span = trial - ys
    small_q = SMALL / np.maximum(ex, 1.0)
    lo, hi = np.zeros_like(span), span.copy()
    x = 0.5 * span
    tl = tol * np.maximum(trial, 1.0)
    pw = np.where(x > 0, np.exp(ex * (np.log(np.maximum(x, 1e-300)) - lk)), 0.0)
    last = x - span + vs * pw
    its = np.zeros(len(trial), dtype=np.int64)
    done = np.zeros(len(trial), dtype=bool)
    for it in range(1, 201):
        conv = ~done & ((np.abs(last) <= tl) | ((hi - lo) <= tl))
        its[conv] = it
        done |= conv
        if done.all():
            break
        act = ~done
        hi = np.where(act & (last > 0), x, hi)
        lo = np.where(act & ~(last > 0), x, lo)
        q = np.where(x > 0, last / (x + c1 * pw), 0.0)
        xn = x - q * x
        newton = (x > 0) & np.isfinite(xn) & (xn > lo) & (xn < hi)
        cheap = newton & (np.abs(q) <= small_q)
        full_x = np.where(newton, xn, 0.5 * (lo + hi))
        full_pw = np.where(full_x > 0, np.exp(ex * (np.log(np.maximum(full_x, 1e-300)) - lk)), 0.0)
        new_pw = np.where(cheap, pw * pow_one_minus_small(q, ex), full_pw)
        x = np.where(act, full_x, x)
        pw = np.where(act, new_pw, pw)
        last = np.where(act, x - span + vs * pw, last)
    return ys + x, its


def test_series_factor_is_the_power_to_rounding():
    rng = np.random.default_rng(0)
    a = rng.uniform(0.1, 10.0, 200_000)
    q = rng.uniform(-1.0, 1.0, a.size) * SMALL / np.maximum(a, 1.0)
    ref = np.power(1.0 - q.astype(np.longdouble), a.astype(np.longdouble))
    got = pow_one_minus_small(q, a)
    err = np.abs((got - ref) / ref).astype(np.float64)
    assert err.max() <= 4e-16


def test_device_form_matches_reference_solver(oracle_mod):
    rng = np.random.default_rng(5)
    n_prob = 4000
    ys = rng.uniform(10, 300, n_prob)
    trial = ys * rng.uniform(1.0001, 3.0, n_prob)
    k = rng.uniform(1, 40, n_prob)
    nn = rng.uniform(0.3, 1.5, n_prob)
    mu = rng.uniform(5e3, 5e4, n_prob)
    dt = rng.uniform(1e-5, 1e-3, n_prob)
    for tol in (1e-10, 1e-12):
        sigma, its = device_form(trial, ys, k, nn, mu, dt, tol)
        ref = np.array([oracle_mod.hb_return(trial[i], ys[i], k[i], nn[i], mu[i], dt[i], tol) for i in range(n_prob)])
        assert (ref[:, 0] == 0).all()
        same = its == ref[:, 3].astype(np.int64)
        assert same.mean() >= 0.999, same.mean()
        assert np.all(np.abs(sigma - ref[:, 1]) <= tol * np.maximum(trial, 1.0))
