"""Energy audit of one trial step (audit.rs, audit_tests.rs, examples/energy_audit.rs).

`audit_step(dt)` measures the endpoint energies (translation, APIC affine norm, elastic,
potential, pellet) before and after one trial step taken on a copy, the grid kinetic energy
after each stage of that step, the ledger increments, and the algebraic terms of the stage
telescope.  The simulation itself is unchanged.

The CPU tests restate the reference's analytic audit tests (core/src/mpm/audit_tests.rs)
against the oracle and pin it to the published light-body values (docs/energy-audit.md:150-160).
The GPU tests run the same cases through the C-ABI and compare every quantity with the
oracle at the FP32 particle-state tolerance."""

from __future__ import annotations

import math

import numpy as np
import pytest

# -------------------------------------------------------------------------- fixtures


def _spec(pellet: bool = False):
    """audit_tests.rs:13-35 `isolated()`: unit box, 0.1 m cells, paste, no gravity.  The
    fixture's own particle block is replaced by `_particles` below."""
    from litter_physics_b200 import _abi, research

    s = research.base_spec(fixture=_abi.LP_COUPLED_PATCH if pellet else _abi.LP_SLUMP, grid_spacing=0.1,
                           domain=[1.0, 1.0, 1.0], initial_size=[0.1, 0.1, 0.3], initial_velocity=[0.0, 0.0, 0.0],
                           seed=0, wall_friction=0.4, max_dt=1e-3, min_dt=1e-9, contact_stiffness=1000.0,
                           contact_restitution=0.2, contact_friction=0.4, gravity=[0.0, 0.0, 0.0])
    s.cfl = 0.3
    s.material = research.material_paste(1000.0, 1000.0, 0.3, 1e6, 0.0, 1.0)
    if pellet:
        # created at a resolvable size; `set_pellet` installs the tested geometry
        s.has_pellet, s.pellet_radius, s.pellet_length, s.pellet_density = 1, 0.16, 0.32, 1.0
    return s


def _particles(rows, yield_stress=1e6):
    """rows: (position, velocity, mass, volume0[, affine, kirchhoff, volume_ratio]); every
    point carries the material's yield stress."""
    from litter_physics_b200 import _abi

    arr, _ = _abi.particle_buffers(len(rows))
    for i, r in enumerate(rows):
        arr["id"][i] = i
        arr["position"][i] = r[0]
        arr["velocity"][i] = r[1]
        arr["mass"][i] = r[2]
        arr["volume0"][i] = r[3]
        arr["deformation"][i] = np.eye(3)
        arr["volume_ratio"][i] = r[6] if len(r) > 6 else 1.0
        arr["yield_stress"][i] = yield_stress
        if len(r) > 4 and r[4] is not None:
            arr["affine"][i] = r[4]
        if len(r) > 5 and r[5] is not None:
            arr["kirchhoff"][i] = r[5]
    return arr


def make_pellet(template, radius, length, density, position, quat):
    """`Pellet::new` (rigid.rs:115-175): cylinder mass and inertia, spheres at most one
    radius apart along the body x axis."""
    p = type(template)()
    mass = density * math.pi * radius * radius * length
    p.radius, p.length, p.mass = radius, length, mass
    p.inertia_body[:] = [0.5 * mass * radius * radius, mass * (3 * radius * radius + length * length) / 12.0,
                         mass * (3 * radius * radius + length * length) / 12.0]
    p.position[:] = list(position)
    p.orientation[:] = list(quat)
    p.velocity[:] = [0.0, 0.0, 0.0]
    p.angular_momentum[:] = [0.0, 0.0, 0.0]
    half = 0.5 * length - radius
    count = 1 if half <= 0.0 else int(math.ceil(2.0 * half / radius)) + 1
    p.sphere_count = count
    for i in range(count):
        p.sphere_offsets[i] = 0.0 if count == 1 else -half + 2.0 * half * i / (count - 1)
    return p


def light_body_sim(factory):
    """examples/energy_audit.rs:153-181: a 2 kg stress-free point moving up at 1 m/s under a
    stationary 1 kg/m^3 body (r 0.15 m, L 0.3 m); no gravity, friction or walls involved."""
    s = _spec(pellet=True)
    s.wall_friction, s.contact_friction, s.max_dt = 0.0, 0.0, 4e-5
    sim = factory(s)
    sim.set_particles(_particles([([0.5, 0.5, 0.5], [0.0, 0.0, 1.0], 2.0, 0.002)]))
    sim.set_pellet(make_pellet(sim.pellet(), 0.15, 0.3, 1.0, [0.5, 0.5, 0.65], [0.0, 0.0, 0.0, 1.0]))
    return sim


def isolated(factory, rows=None, pellet=False, gravity=0.0, material=None):
    s = _spec(pellet=pellet)
    s.gravity[2] = gravity
    if material is not None:
        s.material = material
    sim = factory(s)
    sim.set_particles(_particles(rows or [([0.47, 0.52, 0.55], [0.0, 0.0, 0.0], 2.0, 0.002)],
                                 s.material.yield_stress))
    return sim


def _get(sim, name):
    """`ledger` and `counters` are methods of the oracle and properties of the device simulation."""
    v = getattr(sim, name)
    return v() if callable(v) else v


def snapshot(sim) -> tuple:
    """Everything `audit_step` must leave untouched."""
    p = sim.particles()
    c = _get(sim, "counters")
    led = _get(sim, "ledger")
    pel = sim.pellet()
    key = (c.time, c.step_count, c.rejected_steps, c.limited_steps, c.dt_scale)
    ledger = bytes(memoryview(led))
    pellet = bytes(memoryview(pel)) if pel is not None else b""
    return key, ledger, pellet, {k: v.copy() for k, v in p.items()}


def same_snapshot(a, b) -> bool:
    return (a[0] == b[0] and a[1] == b[1] and a[2] == b[2] and a[3].keys() == b[3].keys()
            and all(np.array_equal(a[3][k], b[3][k]) for k in a[3]))


def oracle_factory(spec):
    import oracle

    return oracle.OracleSim(spec, threads=1)


def close(actual, expected, tol=2e-12):
    """audit_tests.rs:38-43: absolute tolerance for order-one energies."""
    assert abs(actual - expected) < tol, f"actual={actual!r}, expected={expected!r}"


# -------------------------------------------------------------------------- CPU (oracle)
def test_translation_and_affine_norm_are_analytic_and_nonmutating():
    """audit_tests.rs:45-66."""
    aff = np.array([[0.2, 0.3, -0.1], [0.5, -0.4, 0.7], [0.1, 0.2, 0.4]])
    sim = isolated(oracle_factory, [([0.47, 0.52, 0.55], [1.0, -2.0, 0.5], 2.0, 0.002, aff)])
    before = snapshot(sim)
    a = sim.audit_step(1e-4)
    close(a["before"]["translation"], 5.25)
    expected_affine = 0.0025 * float((aff * aff).sum())
    close(a["before"]["affine"], expected_affine)
    close(a["stages"]["grid_transport"], 5.25 + expected_affine)
    close(a["after"]["translation"], 5.25)
    close(a["after"]["affine"], expected_affine)
    close(a["terms"]["p2g_transfer_loss"], 0.0)
    close(a["terms"]["g2p_transfer_loss"], 0.0)
    close(a["terms"]["telescoping_error"], 0.0)
    assert same_snapshot(before, snapshot(sim))
    close(sim.energies()["kinetic"], a["before"]["translation"])


def test_colliding_velocities_have_exact_variance_loss():
    """audit_tests.rs:68-80: two coincident points at +-1 m/s deposit no momentum."""
    x = [0.47, 0.52, 0.55]
    sim = isolated(oracle_factory, [(x, [1.0, 0.0, 0.0], 2.0, 0.002), (x, [-1.0, 0.0, 0.0], 2.0, 0.002)])
    a = sim.audit_step(1e-4)
    close(a["before"]["translation"], 2.0)
    close(a["stages"]["grid_transport"], 0.0)
    close(a["terms"]["p2g_transfer_loss"], 2.0)
    close(a["terms"]["g2p_transfer_loss"], 0.0)


def test_transfers_match_independent_stencil_variance_identities():
    """audit_tests.rs:82-130: with no force the final grid velocity is the transport velocity,
    so both transfer losses are mass-weighted stencil variances, rebuilt here node by node."""
    import oracle

    rows = [([0.47, 0.52, 0.55], [0.7, -0.2, 0.3], 2.0, 0.002, np.eye(3) * 0.3),
            ([0.51, 0.49, 0.58], [-0.4, 0.8, -0.1], 3.0, 0.003,
             np.array([[0.1, -0.2, 0.3], [0.4, 0.2, -0.1], [0.0, 0.3, -0.2]]))]
    sim = isolated(oracle_factory, rows)
    a = sim.audit_step(1e-4)
    trial = isolated(oracle_factory, rows)
    ok, why = trial.try_step(1e-4)
    assert ok, why
    after = trial.particles()
    nodes = [13, 13, 13]  # 10 cells + 3 padding nodes per axis
    mass, mom, st = {}, {}, []
    for p, r in enumerate(rows):
        status, base, w, d = oracle.stencil(0.1, nodes, r[0])
        assert status == 0
        st.append((base, w, d))
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    key = (base[0] + i, base[1] + j, base[2] + k)
                    wt = w[0][i] * w[1][j] * w[2][k]
                    dist = np.array([d[0][i], d[1][j], d[2][k]])
                    v = np.array(r[1]) + r[4] @ dist
                    mass[key] = mass.get(key, 0.0) + wt * r[2]
                    mom[key] = mom.get(key, 0.0) + wt * r[2] * v
    p2g = g2p = 0.0
    for p, r in enumerate(rows):
        base, w, d = st[p]
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    key = (base[0] + i, base[1] + j, base[2] + k)
                    wt = w[0][i] * w[1][j] * w[2][k]
                    dist = np.array([d[0][i], d[1][j], d[2][k]])
                    grid_v = mom[key] / mass[key]
                    old = np.array(r[1]) + r[4] @ dist
                    new = after["velocity"][p] + after["affine"][p] @ dist
                    half = 0.5 * r[2] * wt
                    p2g += half * float(((old - grid_v) ** 2).sum())
                    g2p += half * float(((grid_v - new) ** 2).sum())
    assert p2g > 0.0 and g2p > 0.0
    close(a["terms"]["p2g_transfer_loss"], p2g)
    close(a["terms"]["g2p_transfer_loss"], g2p)


def test_freefall_has_semiimplicit_gravity_potential_defect():
    """audit_tests.rs:132-152: one-step gravity/potential defect -m g^2 dt^2 / 2."""
    sim = isolated(oracle_factory, gravity=-9.81)
    dt = 1e-3
    whole, half = sim.audit_step(dt), sim.audit_step(dt / 2.0)
    expected = -0.5 * 2.0 * 9.81**2 * dt * dt
    close(whole["terms"]["uncoupled_gravity_potential_mismatch"], expected)
    close(half["terms"]["uncoupled_gravity_potential_mismatch"], expected / 4.0)
    assert whole["terms"]["coupled_grid_gravity_total_potential_change"] is None


def test_resting_and_prestressed_material_expose_storage_mismatch():
    """audit_tests.rs:154-170."""
    from litter_physics_b200 import research

    rest = isolated(oracle_factory).audit_step(1e-4)
    close(rest["terms"]["augmented_energy_change"], 0.0)
    liquid = research.material_liquid(1000.0, 1000.0, 0.3, 0.0)
    tau = np.eye(3) * (liquid.bulk_modulus * (0.95 - 1.0))
    sim = isolated(oracle_factory, [([0.47, 0.52, 0.55], [0.0, 0.0, 0.0], 2.0, 0.002, None, tau, 0.95)],
                   material=liquid)
    a = sim.audit_step(1e-4)
    assert a["before"]["elastic"] > 0.0
    assert a["stages"]["grid_after_stress"] > a["stages"]["grid_transport"]
    assert abs(a["terms"]["stress_storage_plastic_mismatch"]) > 1e-10
    close(a["terms"]["telescoping_error"], 0.0)


def wall_rows(velocity):
    return [([0.47, 0.52, 0.025], velocity, 2.0, 0.002, None, np.eye(3) * -1000.0)]


def test_signed_wall_stages_match_existing_histories():
    """audit_tests.rs:172-203: floor projection, friction and traction stage jumps are the
    ledger increments."""
    sim = isolated(oracle_factory, wall_rows([0.1, 0.0, -0.5]), gravity=-9.81)
    a = sim.audit_step(1e-4)
    inc, t = a["increments"], a["terms"]
    assert inc["wall_normal_projection_energy"] < 0.0
    assert inc["wall_friction_dissipation"] > 0.0
    assert inc["wall_normal_traction_energy"] < 0.0
    close(t["traction_change"], inc["wall_normal_traction_energy"])
    close(t["walls_change"], inc["wall_normal_projection_energy"] - inc["wall_friction_dissipation"])
    close(t["telescoping_error"], 0.0)
    sim = isolated(oracle_factory, wall_rows([0.0, 0.0, 0.0]), gravity=-9.81)
    r = sim.audit_step(1e-4)
    assert r["increments"]["wall_normal_traction_energy"] > 0.0
    close(r["terms"]["traction_change"], r["increments"]["wall_normal_traction_energy"])


@pytest.mark.parametrize("density", [1.0, 500.0])
def test_coupled_stages_are_combined_not_fake_gravity_work(density):
    """audit_tests.rs:205-249, light and heavy bodies."""
    sim = isolated(oracle_factory, [([0.5, 0.5, 0.5], [0.0, 0.0, 1.0], 2.0, 0.002)], pellet=True, gravity=-9.81)
    sim.set_pellet(make_pellet(sim.pellet(), 0.15, 0.3, density, [0.5, 0.5, 0.65], [0.0, 0.0, 0.0, 1.0]))
    a = sim.audit_step(1e-4)
    t, inc = a["terms"], a["increments"]
    assert t["uncoupled_gravity_potential_mismatch"] is None
    assert t["coupled_grid_gravity_total_potential_change"] is not None
    assert inc["coupling_grid_energy"] < 0.0
    assert inc["coupling_pellet_energy"] > 0.0
    close(t["coupling_change"], inc["coupling_grid_energy"] + inc["coupling_pellet_energy"])
    close(t["pellet_integrator_combined_change"], a["after"]["pellet"] - a["stages"]["pellet_after_coupling"])
    close(t["telescoping_error"], 0.0)
    e0 = sim.energies()
    sim.advance_to(1e-4)
    e1 = sim.energies()
    # momentum minus the gravity impulse is unchanged by the step (audit_tests.rs:243-247)
    step = [e1[f"momentum_residual_{x}"] - e0[f"momentum_residual_{x}"] for x in "xyz"]
    assert np.linalg.norm(step) < 2e-12


def test_invalid_unstable_escaped_and_rejected_trials_do_not_mutate():
    """audit_tests.rs:251-277: every refused trial raises and leaves the state as it was."""
    from litter_physics_b200 import _abi

    sim = isolated(oracle_factory)
    before = snapshot(sim)
    for dt in (0.0, -1.0, math.nan, math.inf, 1e-12, 1.0):
        with pytest.raises(ValueError, match="audit `dt`"):
            sim.audit_step(dt)
        assert same_snapshot(before, snapshot(sim))
    limited = isolated(oracle_factory)
    c = _get(limited, "counters")
    c.dt_scale = 0.001
    limited.set_counters(c)
    with pytest.raises(ValueError):
        limited.audit_step(1e-4)
    x = [0.47, 0.52, 0.55]
    for rows in ([(x, [0.0] * 3, 2.0, 0.002, np.eye(3) * 1e200)],
                 [(x, [0.0] * 3, 2.0, 0.002, None, np.eye(3) * 1e20)]):
        bad = isolated(oracle_factory, rows)
        before = snapshot(bad)
        with pytest.raises(ValueError):
            bad.audit_step(1e-4)
        assert same_snapshot(before, snapshot(bad))
    assert _abi.EnergyAudit.TERMS[3] == "uncoupled_gravity_potential_mismatch"


def test_report_has_finite_measurements_and_optional_scope():
    """audit_tests.rs:279-289: exactly one of the two gravity terms is present."""
    a = isolated(oracle_factory).audit_step(1e-4)
    assert isinstance(a["before"]["affine"], float)
    assert a["terms"]["uncoupled_gravity_potential_mismatch"] is not None
    assert a["terms"]["coupled_grid_gravity_total_potential_change"] is None
    assert math.isfinite(a["increments"]["wall_normal_traction_energy"])


def plastic_sim(factory, ledger_plastic):
    from litter_physics_b200 import research

    aff = np.zeros((3, 3))
    aff[0, 1] = 50.0
    sim = isolated(factory, [([0.47, 0.52, 0.55], [0.0, 0.0, 0.0], 2.0, 0.002, aff)],
                   material=research.material_paste(1000.0, 1000.0, 0.3, 0.1, 0.0, 1.0))
    led = _get(sim, "ledger")
    led.plastic_dissipation = ledger_plastic
    sim.set_ledger(led)
    return sim


def test_plastic_increment_is_history_difference():
    """audit_tests.rs:291-311."""
    sim = plastic_sim(oracle_factory, 3.0)
    a = sim.audit_step(1e-3)
    sim.advance_to(1e-3)
    assert a["increments"]["plastic_dissipation"] > 0.0
    close(a["increments"]["plastic_dissipation"], _get(sim, "ledger").plastic_dissipation - 3.0)
    s = a["stages"]
    expected = (s["grid_after_stress"] - s["grid_transport"] + a["after"]["elastic"] - a["before"]["elastic"]
                + s["plastic_dissipation"])
    close(a["terms"]["stress_storage_plastic_mismatch"], expected)
    close(a["terms"]["telescoping_error"], 0.0)


def test_local_plastic_work_survives_cumulative_history_rounding():
    """audit_tests.rs:313-334: the ledger increment rounds to zero at 1e100, the stage sum does not."""
    sim = plastic_sim(oracle_factory, 1e100)
    before = snapshot(sim)
    a = sim.audit_step(1e-3)
    assert a["stages"]["plastic_dissipation"] > 0.0
    assert a["increments"]["plastic_dissipation"] == 0.0 and math.copysign(1.0, a["increments"]["plastic_dissipation"]) > 0
    assert same_snapshot(before, snapshot(sim))


def tilted_pellet_sim(factory):
    s_half = math.sin(0.015)
    sim = isolated(factory, pellet=True, gravity=-9.81)
    p = make_pellet(sim.pellet(), 0.1, 0.3, 500.0, [0.5, 0.5, 0.095], [0.0, s_half, 0.0, math.cos(0.015)])
    p.velocity[:] = [0.1, 0.0, -0.2]
    p.angular_momentum[:] = [0.01, 0.02, 0.03]
    sim.set_pellet(p)
    return sim


def test_rigid_gravity_contact_rotation_stay_one_combined_term():
    """audit_tests.rs:336-366: a tilted pellet touching the floor."""
    sim = tilted_pellet_sim(oracle_factory)
    before = snapshot(sim)
    a = sim.audit_step(1e-4)
    assert abs(a["increments"]["pellet_wall_work"]) > 0.0
    assert a["terms"]["uncoupled_gravity_potential_mismatch"] is None
    assert abs(a["terms"]["pellet_integrator_combined_change"]) > 0.0
    assert abs(a["terms"]["pellet_integrator_combined_change"] - a["increments"]["pellet_wall_work"]) > 1e-9
    close(a["terms"]["telescoping_error"], 0.0)
    assert same_snapshot(before, snapshot(sim))


def test_audit_matches_actual_advance_endpoint_and_existing_histories():
    """audit_tests.rs:368-381."""
    sim = isolated(oracle_factory, [([0.47, 0.52, 0.55], [0.1, -0.2, 0.3], 2.0, 0.002)], gravity=-9.81)
    a = sim.audit_step(1e-4)
    sim.advance_to(1e-4)
    e = sim.energies()
    close(a["after"]["translation"], e["kinetic"])
    close(a["after"]["elastic"], e["elastic"])
    close(a["after"]["potential"], e["potential"])
    close(a["increments"]["plastic_dissipation"], _get(sim, "ledger").plastic_dissipation)


# Published first-step figures of the light-body probe, docs/energy-audit.md:155-160.
LIGHT_BODY = {
    "grid_coupling_change": -0.079904513889,
    "pellet_coupling_change": 0.602205342991,
    "joint_coupling_change": 0.522300829103,
    "g2p_transfer_loss": 0.047207353380,
    "augmented_energy_change_dt_10us": 0.475093476868,
}


def light_body_figures(a) -> dict:
    st = a["stages"]
    return {
        "grid_coupling_change": st["grid_after_coupling"] - st["grid_after_walls"],
        "pellet_coupling_change": st["pellet_after_coupling"] - a["before"]["pellet"],
        "joint_coupling_change": a["terms"]["coupling_change"],
        "g2p_transfer_loss": a["terms"]["g2p_transfer_loss"],
    }


def test_light_body_probe_reproduces_published_figures():
    """The coupling figures agree with the published 12-digit values to their last digit and
    are the same at 40, 20 and 10 us.  The augmented endpoint gain at 10 us agrees to 1.4e-9
    relative: it also carries the step's elastic storage (5e-10 J here), which the published
    figure does not resolve further."""
    sim = light_body_sim(oracle_factory)
    before = snapshot(sim)
    audits = [sim.audit_step(4e-5 / d) for d in (1, 2, 4)]
    assert same_snapshot(before, snapshot(sim))
    for a in audits:
        got = light_body_figures(a)
        for k, v in got.items():
            assert abs(v - LIGHT_BODY[k]) <= 6e-13, (k, v)
        assert abs(a["terms"]["telescoping_error"]) < 1e-15
    aug = audits[2]["terms"]["augmented_energy_change"]
    assert abs(aug - LIGHT_BODY["augmented_energy_change_dt_10us"]) <= 2e-9 * LIGHT_BODY["augmented_energy_change_dt_10us"]
    # the joint gain is dt-independent: energy is created by the split coupling update
    joint = [a["terms"]["coupling_change"] for a in audits]
    assert max(joint) - min(joint) < 1e-15


# -------------------------------------------------------------------------- GPU
def sinking_bed(factory):
    """A 24-pellet bed (config-4 model at 7.8 mm cells) lowered 6 mm into its 2-cell paste layer
    and moving down at 0.3 m/s, so that many pellets couple to the grid in the audited step."""
    from test_pellet_bed import small_bed

    sim = factory(small_bed())
    moved = []
    for p in sim.pellets():
        p.position[2] -= 0.006
        p.velocity[:] = [0.0, 0.0, -0.3]
        moved.append(p)
    sim.set_pellets(moved)
    return sim


GPU_CASES = {
    "translation_affine": lambda f: isolated(f, [([0.47, 0.52, 0.55], [1.0, -2.0, 0.5], 2.0, 0.002,
                                                 np.array([[0.2, 0.3, -0.1], [0.5, -0.4, 0.7], [0.1, 0.2, 0.4]]))]),
    "collision": lambda f: isolated(f, [([0.47, 0.52, 0.55], [1.0, 0.0, 0.0], 2.0, 0.002),
                                        ([0.47, 0.52, 0.55], [-1.0, 0.0, 0.0], 2.0, 0.002)]),
    "freefall": lambda f: isolated(f, gravity=-9.81),
    "walls": lambda f: isolated(f, wall_rows([0.1, 0.0, -0.5]), gravity=-9.81),
    "plastic": lambda f: plastic_sim(f, 3.0),
    "light_body": light_body_sim,
    "tilted_pellet": tilted_pellet_sim,
    "pellet_bed": sinking_bed,
}
GPU_DT = {"freefall": 1e-3, "plastic": 1e-3, "light_body": 1e-5, "pellet_bed": 2e-5}


def test_sinking_bed_audit_couples_and_telescopes():
    """The pellet-bed extension inside the audit: every pellet's impulse is one coupling stage,
    and the stage telescope closes."""
    a = sinking_bed(oracle_factory).audit_step(2e-5)
    assert a["increments"]["coupling_grid_energy"] != 0.0
    assert a["increments"]["coupling_pellet_energy"] != 0.0
    close(a["terms"]["coupling_change"],
          a["increments"]["coupling_grid_energy"] + a["increments"]["coupling_pellet_energy"], 1e-12)
    close(a["terms"]["telescoping_error"], 0.0)
    assert a["terms"]["coupled_grid_gravity_total_potential_change"] is not None


@pytest.fixture(scope="module")
def built():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


def gpu_factory(spec):
    from litter_physics_b200.sim import Simulation

    return Simulation(spec)


def flat(a) -> dict:
    out = {}
    for group in ("before", "after", "stages", "increments", "terms"):
        for k, v in a[group].items():
            out[f"{group}.{k}"] = v
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(GPU_CASES))
def test_gpu_audit_matches_oracle(built, case):
    """Every audit quantity of the device path against the FP64 oracle on the same state.
    Particle state is FP32 on the device, so each quantity agrees to 2e-6 of the case's
    energy scale (the largest endpoint or stage energy); the optional gravity terms are
    present on the same side.  The device state is unchanged by the audit."""
    dt = GPU_DT.get(case, 1e-4)
    ref = GPU_CASES[case](oracle_factory)
    gpu = GPU_CASES[case](gpu_factory)
    before = snapshot(gpu)
    r, g = flat(ref.audit_step(dt)), flat(gpu.audit_step(dt))
    assert same_snapshot(before, snapshot(gpu))
    scale = max(abs(v) for k, v in r.items() if v is not None and k.split(".")[0] in ("before", "after", "stages"))
    scale = max(scale, 1e-12)
    bad = []
    for k, v in r.items():
        if v is None or g[k] is None:
            if (v is None) != (g[k] is None):
                bad.append((k, v, g[k]))
            continue
        if not abs(g[k] - v) <= 2e-6 * scale:
            bad.append((k, v, g[k]))
    assert not bad, bad


@pytest.mark.gpu
def test_gpu_audit_refuses_invalid_steps_without_mutation(built):
    sim = isolated(gpu_factory)
    before = snapshot(sim)
    for dt in (0.0, -1.0, math.nan, math.inf, 1e-12, 1.0):
        with pytest.raises(ValueError, match="audit `dt`"):
            sim.audit_step(dt)
    bad = isolated(gpu_factory, [([0.47, 0.52, 0.55], [0.0] * 3, 2.0, 0.002, None, np.eye(3) * 1e20)])
    b0 = snapshot(bad)
    with pytest.raises(ValueError, match="audit trial rejected"):
        bad.audit_step(1e-4)
    assert same_snapshot(before, snapshot(sim))
    assert same_snapshot(b0, snapshot(bad))
    # the simulation still steps normally afterwards
    bad2 = isolated(gpu_factory)
    bad2.audit_step(1e-4)
    bad2.advance_to(2e-4)
    assert _get(bad2, "counters").step_count >= 1
