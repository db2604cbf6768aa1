"""Learned warm start: CPU checks of the oracle network and the feature map, GPU checks of the
device forward/backward kernels against the FP64 oracle, training, and the gain of the trained
network over the midpoint start at equal tolerance."""

from __future__ import annotations

import numpy as np
import pytest


def test_oracle_gradient_matches_finite_differences():
    import mlp_oracle as M

    rng = np.random.default_rng(0)
    w = rng.normal(scale=0.3, size=M.NW)
    x = rng.normal(size=(64, 6))
    y = rng.normal(size=64)
    _, g = M.loss_grad(w, x, y)
    idx = [0, 5, M.B1 + 3, M.W2 + 100, M.W2 + 4000, M.B2 + 7, M.W3 + 10, M.B3]
    fd = M.finite_difference(w, x, y, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_feature_map_matches_device_definition():
    import ctypes as C

    from litter_physics_b200 import _lib, warmstart

    _lib.build()
    raw = np.array([[120.0, 86.6, 11.4, 0.5, 2e4, 1e-4], [300.0, 40.0, 3.0, 0.9, 5e3, 1e-3]])
    f = warmstart.features(raw)
    for i in range(len(raw)):
        out = (C.c_float * 6)()
        _lib.lib().lp_hb_features(*[float(v) for v in raw[i]], out)
        assert np.allclose(np.array(out), f[i], rtol=1e-6, atol=1e-7)


def test_targets_invert_to_the_root():
    from litter_physics_b200 import warmstart

    raw = np.array([[120.0, 86.6, 11.4, 0.5, 2e4, 1e-4]])
    sigma = np.array([100.0])
    t = 1.0 / (1.0 + np.exp(-warmstart.targets(raw, sigma).astype(np.float64)))
    assert abs(86.6 + t[0] * (120.0 - 86.6) - 100.0) < 1e-3


@pytest.mark.gpu
def test_device_gradient_matches_fp64_oracle():
    import mlp_oracle as M

    from litter_physics_b200 import _lib, warmstart

    _lib.build()
    rng = np.random.default_rng(1)
    w = warmstart.init_weights(seed=7)
    x = rng.normal(size=(2048, 6)).astype(np.float32)
    y = rng.normal(size=2048).astype(np.float32)
    loss, g = warmstart.loss_grad(w, x, y)
    rloss, rg = M.loss_grad(w.astype(np.float64), x, y)
    assert abs(loss - rloss) <= 1e-5 * abs(rloss)
    assert np.abs(g - rg).max() <= 1e-4 * np.abs(rg).max()
    yp = warmstart.predict(w, x[:100])
    assert np.allclose(yp, M.forward(w, x[:100]), rtol=1e-4, atol=1e-5)


@pytest.fixture(scope="module")
def trained():
    """Network trained by the device kernels on the pairs the plain Newton logs in a slump."""
    from litter_physics_b200 import _lib, configs, warmstart
    from litter_physics_b200.sim import Simulation

    _lib.build()
    sim = Simulation(configs.slump(32, (8, 8, 16), seed=3, yield_range=(20.0, 100.0)))
    raw, sigma = warmstart.collect(sim, 150, capacity=1_000_000)
    x, y = warmstart.dataset(raw, sigma)
    assert len(y) > 1000
    w, loss = warmstart.train(x, y, epochs=20, batch=1024, lr=2e-3)
    assert loss < 0.05
    return w, x


@pytest.mark.gpu
def test_tensor_core_inference_matches_oracle(trained):
    """The solver's BF16 mma.sync forward pass against the FP64 oracle: error within the BF16
    budget (1% of the output scale), and closer to the oracle's explicit-BF16-rounding forward
    than to the unrounded one (the gap is rounding, not a fragment-layout error)."""
    import mlp_oracle as M

    from litter_physics_b200 import warmstart

    w, x_train = trained
    rng = np.random.default_rng(5)
    x = np.concatenate([x_train[rng.choice(len(x_train), 3000, replace=False)],
                        rng.normal(size=(997, 6)).astype(np.float32)])  # 3997 rows: a ragged last warp
    y = warmstart.predict(w, x, tensor_cores=True).astype(np.float64)
    y64 = M.forward(w.astype(np.float64), x)
    yb = M.forward_bf16(w, x)
    scale = max(1.0, float(np.abs(y64).max()))
    err64 = np.abs(y - y64)
    errb = np.abs(y - yb)
    print(f"max |mma - fp64| {err64.max():.3e}, mean {err64.mean():.3e}; mean |mma - bf16 oracle| {errb.mean():.3e}")
    assert err64.max() <= 1e-2 * scale
    assert errb.mean() <= 0.5 * err64.mean()
    # rows are independent of their warp neighbours
    y_sub = warmstart.predict(w, x[7:40], tensor_cores=True).astype(np.float64)
    assert np.array_equal(y_sub, y[7:40])


@pytest.mark.gpu
def test_warm_table_matches_network(trained):
    """The solver's logit table (one tensor-core pass per instance and dt over the la8 nodes)
    against the network evaluated directly: equal at the nodes up to feature rounding, and the
    linear interpolation half-way between nodes within the BF16 budget of the FP64 network."""
    import mlp_oracle as M

    from litter_physics_b200 import _abi, configs, warmstart
    from litter_physics_b200.sim import Simulation

    w, _ = trained
    spec = configs.slump(32, (8, 8, 16), seed=11, yield_range=(20.0, 100.0))
    sim = Simulation(spec)
    assert sim.warm_table()[0] is None
    sim.set_warm_start(w)
    sim.run_substeps(2)
    tab, dt = sim.warm_table()
    assert tab is not None and 0.0 < dt <= spec.max_dt
    mat = spec.material
    k, n, mu = mat.consistency, mat.flow_index, mat.shear_modulus

    def rows(la8):
        # return problems whose log(a)/8 is la8: trial - yield = K exp(8 la8)
        la8 = np.asarray(la8, dtype=np.float64)
        ys = np.zeros(la8.shape)  # a yield of 0 keeps trial - yield exact down to a = 1e-37
        raw = np.stack([k * np.exp(8.0 * la8), ys, np.full(la8.shape, k), np.full(la8.shape, n),
                        np.full(la8.shape, mu), np.full(la8.shape, dt)], axis=1)
        return warmstart.features(raw).astype(np.float32)

    j = np.arange(_abi.MLP_TAB_N)
    nodes = (np.float32(_abi.MLP_TAB_LO) + j.astype(np.float32) * np.float32(_abi.MLP_TAB_H)).astype(np.float64)
    assert nodes[0] < np.log(1e-37) / 8 and nodes[-1] > np.log(np.finfo(np.float32).max) / 8
    # the la8 range of real problems (a from 1e-6 to 1e4) and a spread over the whole table
    sel = np.unique(np.concatenate([np.flatnonzero((nodes > -1.8) & (nodes < 1.2)), j[::16]]))
    sel = sel[sel < _abi.MLP_TAB_N - 1]
    direct = warmstart.predict(w, rows(nodes[sel]), tensor_cores=True).astype(np.float64)
    scale = max(1.0, float(np.abs(direct).max()))
    assert np.abs(tab[sel] - direct).max() <= 1e-3 * scale
    mid = 0.5 * (nodes[sel] + nodes[sel + 1])
    interp = 0.5 * (tab[sel].astype(np.float64) + tab[sel + 1])
    y64 = M.forward(w.astype(np.float64), rows(mid))
    err = np.abs(interp - y64)
    print(f"table: max |node - mma| {np.abs(tab[sel] - direct).max():.3e}; "
          f"mid-node |interp - fp64| max {err.max():.3e}, mean {err.mean():.3e}")
    assert err.max() <= 1e-2 * scale


@pytest.mark.gpu
def test_batch_warm_tables_per_member(trained):
    """Each batch member's warm-start table comes from its own material and dt: it equals the
    table of a single simulation of the same spec, members with different flow indices get
    different tables, and a weight upload marks every table stale until the next attempt."""
    from litter_physics_b200 import configs
    from litter_physics_b200.sim import Batch, Simulation

    w, _ = trained
    spec_a = configs.slump(16, (4, 4, 8), seed=1, yield_range=(20.0, 100.0))
    spec_b = configs.slump(16, (4, 4, 8), seed=2, yield_range=(20.0, 100.0))
    spec_b.material.flow_index = 0.8
    batch = Batch([spec_a, spec_b])
    batch.set_warm_start(w)
    batch.run_substeps(2)
    batch.sync()
    ta, dta = batch.warm_table(0)
    tb, dtb = batch.warm_table(1)
    assert ta is not None and tb is not None and dta > 0.0 and dtb > 0.0
    assert not np.array_equal(ta, tb)
    one = Simulation(spec_a)
    one.set_warm_start(w)
    one.run_substeps(2)
    one.sync()
    t1, dt1 = one.warm_table()
    assert dt1 == dta and np.array_equal(t1, ta)
    batch.set_warm_start(w)  # a new upload: every table is rebuilt on the next attempt
    assert batch.warm_table(0)[0] is None and batch.warm_table(1)[0] is None
    batch.run_substeps(1)
    batch.sync()
    ta2, dta2 = batch.warm_table(0)
    assert ta2 is not None and (dta2 != dta or np.array_equal(ta2, ta))
    with pytest.raises(Exception):
        batch.warm_table(2)


@pytest.mark.gpu
def test_warm_started_slump_matches_oracle(trained):
    """Warm start inside the solver (G2P's tensor-core network pass): the slump after 100
    substeps stays within the parity bars of the plain solver against the FP64 oracle, with
    fewer Newton iterations."""
    import oracle
    from litter_physics_b200 import configs
    from litter_physics_b200.sim import Simulation

    w, _ = trained
    spec = configs.slump(32, (8, 8, 16), seed=11, yield_range=(20.0, 100.0))
    steps = 100
    ref = oracle.OracleSim(spec)
    ref.advance_to(steps * spec.max_dt)
    r = ref.particles()
    order_r = np.argsort(r["id"])
    out = {}
    for name, weights in (("plain", None), ("warm", w)):
        sim = Simulation(spec)
        sim.set_warm_start(weights)
        sim.advance_to(steps * spec.max_dt)
        p = sim.particles()
        o = np.argsort(p["id"])
        assert np.array_equal(p["id"][o], r["id"][order_r])
        dx = float(np.abs(p["position"][o] - r["position"][order_r]).max()) / max(spec.domain)
        dv = float(np.linalg.norm(p["velocity"][o] - r["velocity"][order_r])) / float(
            np.linalg.norm(r["velocity"]))
        out[name] = (dx, dv, sim.counters.newton_iterations, sim.counters.yielded_particles)
    print(out)
    for name in out:
        assert out[name][0] <= 1e-5 and out[name][1] <= 1e-5, (name, out[name])
    assert out["warm"][3] > 0
    assert out["warm"][2] < 0.8 * out["plain"][2]


@pytest.mark.gpu
def test_trained_network_cuts_newton_iterations_at_equal_tolerance(trained):
    """Solve fresh return problems with and without the warm start (tensor-core inference):
    same residual tolerance, fewer iterations."""
    import ctypes as C

    from litter_physics_b200 import _lib, configs, warmstart
    from litter_physics_b200.sim import Simulation

    w, _ = trained
    # fresh problems from a different slump
    sim2 = Simulation(configs.slump(32, (8, 8, 16), seed=9, yield_range=(20.0, 100.0)))
    raw2, _ = warmstart.collect(sim2, 120, capacity=200_000)
    r = raw2.astype(np.float64)
    n = len(r)
    D = C.POINTER(C.c_double)
    cols = [np.ascontiguousarray(r[:, i]) for i in range(6)]
    res = {}
    for name, weights in (("plain", None), ("warm", w)):
        out = np.zeros((n, 3))
        st = np.zeros(n, dtype=np.int32)
        wp = weights.ctypes.data_as(C.POINTER(C.c_float)) if weights is not None else None
        _lib.check(_lib.lib().lp_hb_return_batch(n, *[c.ctypes.data_as(D) for c in cols], 1e-10, wp,
                                                  warmstart.NW if weights is not None else 0,
                                                  out.ctypes.data_as(D), st.ctypes.data_as(C.POINTER(C.c_int32))))
        assert (st == 0).all()
        res[name] = out
    # equal residual tolerance: both meet the stopping rule; the returned stress agrees to it
    tol = 1e-10 * np.maximum(r[:, 0], 1.0)
    assert np.all(np.abs(res["plain"][:, 0] - res["warm"][:, 0]) <= 10 * tol + 1e-9 * r[:, 0])
    it_plain, it_warm = res["plain"][:, 2].mean(), res["warm"][:, 2].mean()
    print(f"mean Newton iterations: plain {it_plain:.3f}, warm {it_warm:.3f}")
    assert it_warm < 0.8 * it_plain
