"""GPU parity against the FP64 oracle, through the C ABI.

Bars (north-star parity contract):
  * particle positions: max_p |x_gpu - x_ref| / L_domain <= 1e-5 after 100 substeps;
  * particle velocities: ||v_gpu - v_ref||_2 / ||v_ref||_2 <= 1e-5 after 100 substeps
    (particles matched by id, since both sides reorder them).  The hydrostatic column at rest
    has reference velocities that are discretisation noise, not a velocity scale; there the
    bar is absolute, per particle, in m/s (see the test);
  * grid mass and momentum after P2G equal the particle totals to 1e-10 relative (the P2G
    tile totals are exact by construction), and node by node the deposit and the wall
    reactions agree with the oracle's FP64 grid to 1e-6 of the grid's scale;
  * ledger totals: relative agreement stated per field below (FP32 device arithmetic against
    FP64 reference arithmetic).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_request

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
VEL_TOL = 1e-5


@pytest.fixture(scope="module")
def lib_built():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


def by_id(p: dict) -> dict:
    order = np.argsort(p["id"])
    return {k: v[order] for k, v in p.items()}


def compare(gpu: dict, ref: dict, length: float) -> dict:
    g, r = by_id(gpu), by_id(ref)
    assert np.array_equal(g["id"], r["id"])
    x_err = float(np.max(np.abs(g["position"] - r["position"]))) / length
    v_ref = float(np.linalg.norm(r["velocity"]))
    dv = float(np.linalg.norm(g["velocity"] - r["velocity"]))
    return {"x": x_err, "v": dv / max(v_ref, 1e-300), "v_norm": v_ref}


def run_pair(spec, steps: int):
    import oracle
    from litter_physics_b200.sim import Simulation

    target = steps * spec.max_dt
    ref = oracle.OracleSim(spec)
    ref.advance_to(target)
    gpu = Simulation(spec)
    gpu.advance_to(target)
    return gpu, ref


def small_slump():
    from litter_physics_b200 import configs

    # config-0 material on a 32^3 grid (column 8x8x16 cells, 8192 particles)
    return configs.slump(32, (8, 8, 16), seed=0)


def test_initial_state_matches_oracle(lib_built):
    import oracle
    from litter_physics_b200.sim import Simulation

    spec = small_slump()
    gpu = Simulation(spec).particles()
    ref = oracle.OracleSim(spec).particles()
    d = compare(gpu, ref, 1.0)
    assert d["x"] < 1e-7
    assert np.allclose(by_id(gpu)["mass"], by_id(ref)["mass"], rtol=1e-7)


@pytest.mark.parametrize("name", ["slump32", "research_slump", "research_hydrostatic_water", "dam_break",
                                  "research_coupled_patch"])
def test_100_substeps_match_oracle(lib_built, name):
    from litter_physics_b200 import configs, research

    if name == "slump32":
        spec = small_slump()
    elif name == "dam_break":
        spec = configs.dam_break(32, (16, 8, 16), seed=1)
    else:
        spec = research.spec_from_request(load_request(name))
    gpu, ref = run_pair(spec, 100)
    length = max(spec.domain)
    pg, pr = gpu.particles(), ref.particles()
    d = compare(pg, pr, length)
    gc, rc = gpu.counters, ref.counters()
    assert gc.step_count == rc.step_count and gc.rejected_steps == rc.rejected_steps
    assert d["x"] <= POS_TOL, d
    if name == "research_hydrostatic_water":
        # A column at rest: the reference velocities are the residual of gravity against the
        # pressure gradient, not a physical velocity scale, so the bar is absolute.  Per step,
        # FP32 rounding of positions and stress (relative 2^-23) perturbs each particle's
        # acceleration by about (h / dx) 2^-23 |g|, the pressure-gradient cancellation of a
        # column of h / dx cells; over n steps that is n (h / dx) 2^-23 |g| dt.  The bar is 8
        # times that bound, per particle.
        g = math.sqrt(sum(v * v for v in spec.gravity))
        cells_high = spec.initial_size[2] / spec.grid_spacing
        bar = 8.0 * gc.step_count * cells_high * 2.0**-23 * g * spec.max_dt
        gv, rv = by_id(pg)["velocity"], by_id(pr)["velocity"]
        err = np.linalg.norm(gv - rv, axis=1)
        print(name, d, f"max |dv| {err.max():.3e} m/s, rms {np.sqrt(np.mean(err**2)):.3e} m/s, bar {bar:.3e} m/s")
        assert err.max() <= bar, (err.max(), bar)
    else:
        print(name, d)
        assert d["v"] <= VEL_TOL, d


def test_ledgers_match_oracle(lib_built):
    spec = small_slump()
    gpu, ref = run_pair(spec, 100)
    lg, lr = gpu.ledger, ref.ledger()
    assert lg.initial_mass == pytest.approx(lr.initial_mass, rel=1e-7)
    for f in ("gravity_impulse", "wall_impulse"):
        a, b = np.array(getattr(lg, f)), np.array(getattr(lr, f))
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), f
    for f, rel in (("wall_normal_projection_energy", 1e-3), ("wall_friction_dissipation", 1e-3),
                   ("wall_normal_traction_energy", 1e-3), ("plastic_dissipation", 1e-3)):
        a, b = getattr(lg, f), getattr(lr, f)
        assert abs(a - b) <= rel * max(abs(b), 1e-30), (f, a, b)


def test_grid_conserves_mass_and_momentum(lib_built):
    from litter_physics_b200.sim import Simulation

    spec = small_slump()
    sim = Simulation(spec)
    sim.advance_to(30 * spec.max_dt)
    t = sim.grid_totals(spec.max_dt)
    assert abs(t["grid_mass"] - t["particle_mass"]) <= 1e-10 * t["particle_mass"]
    scale = np.linalg.norm(t["particle_momentum"])
    assert np.linalg.norm(t["grid_momentum"] - t["particle_momentum"]) <= 1e-10 * scale


def random_state(p: dict, spec, rng) -> dict:
    """A developed state made generic: positions jittered by up to 0.3 cells (kept inside the
    domain), random velocities, affine fields and symmetric Kirchhoff stresses, every value
    rounded to FP32 so that the device and the oracle start from the same numbers."""
    q = {k: v.copy() for k, v in p.items()}
    n = len(q["id"])
    dx = spec.grid_spacing
    lo, hi = 0.25 * dx, np.array(spec.domain) - 0.25 * dx
    q["position"] = np.clip(q["position"] + rng.uniform(-0.3 * dx, 0.3 * dx, (n, 3)), lo, hi)
    q["velocity"] = q["velocity"] + rng.normal(scale=0.05, size=(n, 3))
    q["affine"] = q["affine"] + rng.normal(scale=2.0, size=(n, 3, 3))
    s = rng.normal(scale=200.0, size=(n, 3, 3))
    q["kirchhoff"] = q["kirchhoff"] + 0.5 * (s + s.transpose(0, 2, 1))
    for k in ("position", "velocity", "affine", "kirchhoff"):
        q[k] = np.ascontiguousarray(q[k].astype(np.float32).astype(np.float64))
    return q


@pytest.mark.parametrize("name", ["slump32", "dam_break"])
def test_p2g_and_traction_match_oracle_node_by_node(lib_built, name):
    """P2G (solver.rs:632-661, grid.rs:254-263) and the wall traction (solver.rs:725-819,
    grid.rs:279-295) of one generic state, node by node against the oracle's FP64 grid: mass,
    momentum before the reactions and the signed reaction impulses, including the wall shell."""
    import oracle
    from litter_physics_b200 import configs
    from litter_physics_b200.sim import Simulation

    spec = small_slump() if name == "slump32" else configs.dam_break(32, (16, 8, 16), seed=1)
    sim = Simulation(spec)
    sim.advance_to(30 * spec.max_dt)
    state = random_state(sim.particles(), spec, np.random.default_rng(3))
    sim.set_particles(state)
    ref = oracle.OracleSim(spec)
    ref.set_particles(state)
    dt = spec.max_dt
    gm, gp, gr = sim.grid_dump(dt)
    rm, rp, rr = ref.probe_grid(dt, len(gm))
    m_scale, p_scale = rm.max(), np.abs(rp).max()
    r_scale = np.abs(rr).max()
    assert m_scale > 0 and p_scale > 0 and r_scale > 0  # the case has deposits and wall reactions
    m_err = np.abs(gm - rm).max() / m_scale
    p_err = np.abs(gp - rp).max() / p_scale
    r_err = np.abs(gr - rr).max() / r_scale
    walls = np.count_nonzero(np.any(rr != 0.0, axis=1))
    print(name, f"nodes {np.count_nonzero(rm)}, wall nodes {walls}, mass {m_err:.2e}, momentum {p_err:.2e}, "
          f"reaction {r_err:.2e}")
    assert m_err <= 1e-6 and p_err <= 1e-6 and r_err <= 1e-6
    # the probe leaves the committed state untouched
    after = sim.particles()
    assert np.array_equal(by_id(after)["position"], by_id(state)["position"])


def test_runs_are_bitwise_repeatable(lib_built):
    from litter_physics_b200.sim import Simulation

    spec = small_slump()
    out = []
    for _ in range(2):
        sim = Simulation(spec)
        sim.advance_to(50 * spec.max_dt)
        led = sim.ledger
        p = by_id(sim.particles())
        out.append((bytes(led), p["position"].tobytes(), p["velocity"].tobytes()))
    assert out[0] == out[1]


def test_rejected_trial_preserves_state(lib_built):
    """solver.rs:1714-1740: an oversized step is rejected before any commit."""
    from litter_physics_b200 import research
    from litter_physics_b200.sim import Simulation

    spec = research.spec_from_request(load_request("research_slump"))
    spec.initial_velocity[:] = [1.0, 0.0, -1.0]
    sim = Simulation(spec)
    sim.advance_to(2e-4)
    before = (bytes(sim.ledger), sim.particles()["position"].tobytes())
    ok, reason = sim.try_step(5e-3)
    assert not ok and reason
    after = (bytes(sim.ledger), sim.particles()["position"].tobytes())
    assert before == after


def test_constitutive_kernels_match_oracle(lib_built):
    import ctypes as C

    import oracle
    from litter_physics_b200 import _lib

    rng = np.random.default_rng(5)
    m = oracle.material_paste_shear(1200.0, 56250.0, 0.40625, 50.0, 5.0, 0.5)
    n = 512
    # small strains (series path) and large stretches (||F F^T - I|| > 0.25: eigen path)
    f = np.eye(3)[None] + rng.normal(scale=3e-3, size=(n, 3, 3))
    f[n // 2:] = np.diag([0.8, 1.15, 0.95])[None] + rng.normal(scale=2e-2, size=(n - n // 2, 3, 3))
    f = np.ascontiguousarray(f)
    dt = 1e-4
    fn, tau = np.zeros((n, 9)), np.zeros((n, 9))
    dep, diss, eq = np.zeros(n), np.zeros(n), np.zeros(n)
    st = np.zeros(n, dtype=np.int32)
    D = C.POINTER(C.c_double)
    _lib.check(_lib.lib().lp_update_paste_batch(n, f.ctypes.data_as(D), C.byref(m), dt, fn.ctypes.data_as(D),
                                                 tau.ctypes.data_as(D), dep.ctypes.data_as(D),
                                                 diss.ctypes.data_as(D), eq.ctypes.data_as(D),
                                                 st.ctypes.data_as(C.POINTER(C.c_int32))))
    assert (st == 0).all()
    yielded = 0
    for i in range(n):
        rs, rfn, rtau, rdep, rdiss, req = oracle.update_paste(f[i], m, dt)
        assert rs == 0
        scale = np.abs(rtau).max()
        assert np.abs(tau[i].reshape(3, 3) - rtau).max() <= 1e-4 * scale + 1e-3
        assert np.abs(fn[i].reshape(3, 3) - rfn).max() <= 2e-6 * max(1.0, np.abs(rfn).max())
        if rdep > 0:
            yielded += 1
            assert abs(eq[i] - req) <= 1e-4 * req
    assert yielded > 50


def test_hb_return_batch_matches_oracle(lib_built):
    import ctypes as C

    import oracle
    from litter_physics_b200 import _lib

    rng = np.random.default_rng(1)
    n = 2000
    ys = rng.uniform(10, 300, n)
    trial = ys * rng.uniform(1.0001, 3.0, n)
    k = rng.uniform(1, 40, n)
    nn = rng.uniform(0.3, 1.5, n)
    mu = rng.uniform(5e3, 5e4, n)
    dt = rng.uniform(1e-5, 1e-3, n)
    out = np.zeros((n, 3))
    st = np.zeros(n, dtype=np.int32)
    D = C.POINTER(C.c_double)
    args = [a.ctypes.data_as(D) for a in (trial, ys, k, nn, mu, dt)]
    _lib.check(_lib.lib().lp_hb_return_batch(n, *args, 1e-12, None, 0, out.ctypes.data_as(D),
                                              st.ctypes.data_as(C.POINTER(C.c_int32))))
    assert (st == 0).all()
    for i in range(0, n, 7):
        rs, sigma, dep, it = oracle.hb_return(trial[i], ys[i], k[i], nn[i], mu[i], dt[i])
        assert rs == 0 and it == int(out[i, 2])
        assert abs(out[i, 0] - sigma) <= 1e-12 * max(trial[i], 1.0) * 4


def test_liquid_kernel_matches_oracle(lib_built):
    import ctypes as C

    import oracle
    from litter_physics_b200 import _lib

    m = oracle.material_liquid(1000.0, 1e5, 0.2, 0.5)
    rng = np.random.default_rng(2)
    n = 256
    j = rng.uniform(0.98, 1.02, n)
    g = rng.normal(scale=2.0, size=(n, 3, 3))
    jn, tau, p = np.zeros(n), np.zeros((n, 9)), np.zeros(n)
    st = np.zeros(n, dtype=np.int32)
    D = C.POINTER(C.c_double)
    _lib.check(_lib.lib().lp_update_liquid_batch(n, j.ctypes.data_as(D), np.ascontiguousarray(g).ctypes.data_as(D),
                                                  C.byref(m), 1e-4, jn.ctypes.data_as(D), tau.ctypes.data_as(D),
                                                  p.ctypes.data_as(D), st.ctypes.data_as(C.POINTER(C.c_int32))))
    for i in range(n):
        rs, rj, rtau, rp = oracle.update_liquid(j[i], g[i], m, 1e-4)
        assert abs(jn[i] - rj) <= 1e-6
        assert abs(p[i] - rp) <= 1e-4 * abs(m.bulk_modulus) * 1e-2 + 1e-3 * abs(rp)


def test_batch_matches_single_instances(lib_built):
    from litter_physics_b200 import configs
    from litter_physics_b200.sim import Batch, Simulation

    specs = [configs.slump(16, (4, 4, 8), seed=s) for s in (11, 12)] + [configs.slump(24, (6, 6, 12), seed=13)]
    b = Batch(specs)
    b.advance_to(40 * 1e-4)
    for i, s in enumerate(specs):
        one = Simulation(s)
        one.advance_to(40 * 1e-4)
        pb, ps = by_id(b.particles(i)), by_id(one.particles())
        assert np.array_equal(pb["position"], ps["position"])
        assert bytes(b.ledger(i)) == bytes(one.ledger)


def test_export_in_place_matches_a_fresh_export(lib_built):
    """The export into a resident host particle set overwrites every field with what a fresh
    export returns."""
    from litter_physics_b200.sim import Simulation

    spec = small_slump()
    sim = Simulation(spec)
    sim.advance_to(10 * spec.max_dt)
    fresh = sim.particles()
    host = {k: np.full_like(v, 7) for k, v in fresh.items()}  # stale contents
    got = sim.particles(out=host)
    assert got is host
    for k, v in fresh.items():
        assert np.array_equal(host[k], v), k
    sim.close()


def test_large_strain_particles_take_the_eigen_pass(lib_built):
    """Particles whose trial strain is outside the series path (||F F^T - I|| > 0.25) are left by
    G2P to the eigen-decomposition pass: a developed slump where every fifth particle carries a
    large rotated stretch matches the oracle's update_paste (constitutive.rs:456-531, Jacobi
    373-425) for 5 substeps, and the run is bitwise repeatable (fixed-order tile partials)."""
    import oracle
    from litter_physics_b200.sim import Simulation

    spec = small_slump()
    sim = Simulation(spec)
    sim.advance_to(30 * spec.max_dt)
    state = sim.particles()
    n = len(state["id"])
    rng = np.random.default_rng(11)
    big = np.arange(0, n, 5)
    for i in big:
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        f = q @ np.diag(rng.uniform(1.15, 1.35, 3) * np.array([1.0, 0.8, 0.9])) @ q.T
        state["deformation"][i] = f.astype(np.float32).astype(np.float64).reshape(state["deformation"][i].shape)
    state["deformation"] = np.ascontiguousarray(state["deformation"])
    b = state["deformation"].reshape(-1, 3, 3)
    bn = np.linalg.norm(b[big] @ b[big].transpose(0, 2, 1) - np.eye(3), axis=(1, 2))
    assert bn.min() > 0.3  # all of them need the eigenvectors
    steps = 5
    runs = []
    for _ in range(2):
        g = Simulation(spec)
        g.set_particles(state)
        g.set_ledger(sim.ledger)
        g.set_counters(sim.counters)
        g.advance_to(sim.time + steps * spec.max_dt)
        runs.append(g)
    ref = oracle.OracleSim(spec)
    ref.set_particles(state)
    ref.set_ledger(sim.ledger)
    ref.set_counters(sim.counters)
    ref.advance_to(sim.time + steps * spec.max_dt)
    gp, rp = by_id(runs[0].particles()), by_id(ref.particles())
    assert runs[0].counters.step_count == ref.counters().step_count
    err = compare(gp, rp, float(spec.domain[0]))
    f_err = np.abs(gp["deformation"] - rp["deformation"]).max()
    print(f"large strain: x {err['x']:.2e}, v {err['v']:.2e}, F {f_err:.2e}")
    assert err["x"] <= POS_TOL and err["v"] <= VEL_TOL
    assert f_err <= 1e-5
    led_g, led_r = runs[0].ledger, ref.ledger()
    assert math.isclose(led_g.plastic_dissipation, led_r.plastic_dissipation, rel_tol=1e-4)
    again = by_id(runs[1].particles())
    for k in ("position", "velocity", "deformation", "kirchhoff", "plastic_strain"):
        assert np.array_equal(gp[k], again[k]), k
    assert bytes(runs[0].ledger) == bytes(runs[1].ledger)


def test_page_locked_import_and_export_match_the_staged_path(lib_built):
    """Export into and import from page-locked host arrays (lp_host_pin, moved by DMA) give
    bit for bit what the staged path gives for pageable arrays."""
    from litter_physics_b200.sim import PinnedParticles, Simulation

    spec = small_slump()
    sim = Simulation(spec)
    sim.advance_to(10 * spec.max_dt)
    fresh = sim.particles()
    host = {k: np.full_like(v, 7) for k, v in fresh.items()}
    with PinnedParticles(host) as pinned:
        sim.particles(out=pinned)
        for k, v in fresh.items():
            assert np.array_equal(pinned[k], v), k
        a, b = Simulation(spec), Simulation(spec)
        a.set_particles(fresh)
        b.set_particles(pinned)
        pa, pb = a.particles(), b.particles()
        for k in fresh:
            assert np.array_equal(pa[k], pb[k]), k
        a.advance_to(5 * spec.max_dt)
        b.advance_to(5 * spec.max_dt)
        assert np.array_equal(by_id(a.particles())["position"], by_id(b.particles())["position"])
    sim.close()
