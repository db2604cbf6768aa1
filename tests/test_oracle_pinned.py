"""Pin the FP64 oracle to the reference's own answers before trusting it.

Two kinds of pins:
  * end-to-end: the reference's published FP64 results of its shipped example requests
    (docs/validation.md:153-157, 232-236) reproduced to 10 significant digits;
  * known answers: restatements of the reference's unit tests (formal_examples.rs,
    constitutive.rs, grid.rs, solver.rs, rigid.rs, fixtures.rs tests) on the oracle.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_request, reference_values


def _quoted_half_ulp(value: float) -> float:
    """Half a unit in the last digit of the value as quoted (its shortest repr)."""
    text = repr(float(value)).lower()
    mantissa, _, exponent = text.partition("e")
    decimals = len(mantissa.split(".")[1]) if "." in mantissa else 0
    return 0.5 * 10.0 ** (-decimals) * 10.0 ** (int(exponent) if exponent else 0)


def _quoted_equal(ours: float, quoted: float) -> bool:
    return abs(ours - quoted) <= _quoted_half_ulp(quoted) * (1 + 1e-9)


@pytest.mark.parametrize("name", ["research_hydrostatic_water", "research_slump", "research_coupled_patch"])
def test_oracle_reproduces_published_example_results(oracle_mod, name):
    from litter_physics_b200 import research

    req = load_request(name)
    ref = reference_values()[name]
    sim = oracle_mod.OracleSim(research.spec_from_request(req))
    assert sim.advance_to(req["duration_s"])
    obs = sim.observables()
    for key, value in ref["observables"].items():
        if key in ("mass_residual_kg", "momentum_residual_kg_m_s"):
            assert obs[key] == pytest.approx(value, rel=1e-9, abs=1e-21), key
        else:
            assert _quoted_equal(obs[key], value), f"{key}: oracle {obs[key]!r} vs reference {value!r}"


def test_paste_return_known_answer(oracle_mod):
    """core/tests/formal_examples.rs:11-25."""
    ka = reference_values()["known_answers"]["paste_return"]
    m = oracle_mod.material_paste_shear(*ka["material_shear_rheology"])
    trial_stress = ka["trial_equivalent_stress"]
    strain = trial_stress / (2.0 * math.sqrt(3.0) * m.shear_modulus)
    f = np.diag([math.exp(strain), math.exp(-strain), 1.0])
    st, fn, tau, dep, diss, eq = oracle_mod.update_paste(f, m, ka["dt"])
    assert st == 0
    assert abs(eq - ka["equivalent_stress"]) < ka["equivalent_stress_tol"]
    assert abs(dep - ka["plastic_increment"]) < ka["plastic_increment_tol"]
    assert abs(np.linalg.det(fn) - 1.0) < 1e-12
    elastic_drop = (trial_stress**2 - eq**2) / (6.0 * m.shear_modulus)
    gap = 1.5 * m.shear_modulus * dep**2
    assert abs(elastic_drop - diss - gap) < 1e-12


def test_water_eos_known_answer(oracle_mod):
    """core/tests/formal_examples.rs:27-44."""
    ka = reference_values()["known_answers"]["water_eos"]
    m = oracle_mod.material_liquid(*ka["material_liquid"])
    ratio = math.exp(-m.density * ka["gravity"] * ka["depth"] / m.bulk_modulus)
    p = m.bulk_modulus * (1.0 / ratio - 1.0)
    assert abs(p - ka["pressure"]) < ka["pressure_tol"]
    st, j, tau, pressure = oracle_mod.update_liquid(1.0, -np.eye(3), m, 1e-3)
    assert st == 0 and abs(j - ka["volume_ratio_after"]) < 1e-14
    st, *_ = oracle_mod.update_liquid(1.0, -np.eye(3), m, 0.4)
    assert st == 1  # inverted


@pytest.mark.parametrize("n", [0.3, 0.6, 1.0, 1.5])
def test_hb_return_residual(oracle_mod, n):
    """constitutive.rs:617-633."""
    trial, ys, k, mu, dt = 500.0, 20.0, 5.0, 1.0e4, 1e-3
    st, sigma, dep, it = oracle_mod.hb_return(trial, ys, k, n, mu, dt)
    assert st == 0
    rate = ((sigma - ys) / k) ** (1.0 / n)
    assert abs(sigma - trial + 3.0 * mu * dt * rate) < 1e-8 * trial
    assert ys < sigma < trial
    assert abs(dep - rate * dt) < 1e-6 * rate * dt


def test_hb_return_edge_cases(oracle_mod):
    """constitutive.rs:610-645."""
    st, sigma, dep, it = oracle_mod.hb_return(10.0, 20.0, 5.0, 0.6, 1.0e4, 1e-3)
    assert st == 0 and dep == 0.0
    st, sigma, dep, it = oracle_mod.hb_return(500.0, 20.0, 0.0, 1.0, 1.0e4, 1e-3)
    assert st == 0 and sigma == 20.0
    st, *_ = oracle_mod.hb_return(float("nan"), 20.0, 5.0, 1.0, 1.0e4, 1e-3)
    assert st == 5  # non-finite


def test_jacobi_reconstructs(oracle_mod):
    """constitutive.rs:647-660."""
    m = np.array([[2.0, -1.0, 0.3], [-1.0, 3.0, 0.5], [0.3, 0.5, 1.5]])
    st, vals, vecs = oracle_mod.eigen3(m)
    assert st == 0
    assert np.linalg.norm(vecs @ np.diag(vals) @ vecs.T - m) < 1e-12
    assert np.linalg.norm(vecs @ vecs.T - np.eye(3)) < 1e-12
    near = np.eye(3) + np.array([[0, 1e-9, 0], [1e-9, 0, 0], [0, 0, 2e-9]])
    st, vals, vecs = oracle_mod.eigen3(near)
    assert np.linalg.norm(vecs @ np.diag(vals) @ vecs.T - near) < 1e-15
    st, *_ = oracle_mod.eigen3(np.eye(3) * float("nan"))
    assert st != 0


def test_paste_update_cases(oracle_mod):
    """constitutive.rs:662-723: inversion, hydrostatic Hencky, steady HB simple shear."""
    m = oracle_mod.material_paste(1000.0, 1.0e5, 0.3, 20.0, 5.0, 0.6)
    st, *_ = oracle_mod.update_paste(np.diag([-1.0, 1.0, 1.0]), m, 1e-3)
    assert st == 1
    stretch = 0.99
    st, fn, tau, dep, diss, eq = oracle_mod.update_paste(np.eye(3) * stretch, m, 1e-3)
    assert st == 0 and dep == 0.0
    expected = (2.0 * m.shear_modulus + 3.0 * m.lame_lambda) * math.log(stretch)
    assert abs(tau[0, 0] - expected) < 1e-9 * abs(expected)
    assert np.linalg.norm(fn - np.eye(3) * stretch) < 1e-12
    mat = oracle_mod.material_paste_shear(1000.0, 1.0e6, 0.3, 20.0, 5.0, 0.6)
    rate, dt = 2.0, 1e-4
    grad = np.zeros((3, 3))
    grad[0, 2] = rate
    f = np.eye(3)
    for _ in range(20_000):
        st, f, tau, dep, diss, eq = oracle_mod.update_paste((np.eye(3) + grad * dt) @ f, mat, dt)
        assert st == 0
    expected_shear = 20.0 + 5.0 * rate**0.6
    assert abs(eq - math.sqrt(3.0) * expected_shear) / (math.sqrt(3.0) * expected_shear) < 1e-6
    assert abs(tau[0, 2] - expected_shear) / expected_shear < 1e-6
    assert abs(dep / dt - rate / math.sqrt(3.0)) / (rate / math.sqrt(3.0)) < 1e-6


def test_liquid_cases(oracle_mod):
    """constitutive.rs:725-760."""
    m = oracle_mod.material_liquid(1000.0, 1.0e5, 0.2, 1e-3)
    st, j, tau, p = oracle_mod.update_liquid(1.0, -np.eye(3), m, 1e-3)
    assert abs(j - (1.0 - 3e-3)) < 1e-15
    assert abs(p - m.bulk_modulus * (1.0 / j - 1.0)) < 1e-9
    assert abs(tau[0, 0] + p * j) < 1e-9 and abs(tau[0, 1]) < 1e-15
    m = oracle_mod.material_liquid(1000.0, 1.0e5, 0.2, 0.5)
    g = np.zeros((3, 3))
    g[0, 2] = 4.0
    st, j, tau, p = oracle_mod.update_liquid(1.0, g, m, 1e-4)
    assert abs(tau[0, 2] - 2.0) < 1e-12 and abs(p) < 1e-12
    m = oracle_mod.material_liquid(1000.0, 1.0e5, 0.2, 0.0)
    st, *_ = oracle_mod.update_liquid(1.0, -np.eye(3) * 1.0e6, m, 1e-3)
    assert st == 1


def test_stencil_partition_of_unity(oracle_mod):
    """grid.rs:391-426."""
    nodes = [13, 13, 13]
    for x in ([0.0, 0.0, 0.0], [0.0031, 0.0177, 0.02], [0.0195, 0.0004, 0.011]):
        st, base, w, off = oracle_mod.stencil(0.002, nodes, x)
        assert st == 0
        total = 0.0
        centroid = np.zeros(3)
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    ww = w[0, a] * w[1, b] * w[2, c]
                    total += ww
                    node = (np.array([base[0] + a, base[1] + b, base[2] + c]) - 1.0) * 0.002
                    centroid += node * ww
                    d = np.array([off[0, a], off[1, b], off[2, c]])
                    assert np.linalg.norm(node - np.array(x) - d) < 1e-12
        assert abs(total - 1.0) < 1e-12 and np.linalg.norm(centroid - np.array(x)) < 1e-12
    assert oracle_mod.stencil(0.002, nodes, [-0.003, 0, 0])[0] != 0
    assert oracle_mod.stencil(0.002, nodes, [0, 0, 0.0231])[0] != 0


def test_splitmix_deterministic(oracle_mod):
    """rng.rs:55-67."""
    import ctypes

    a = ctypes.c_uint64(7)
    b = ctypes.c_uint64(7)
    for _ in range(1000):
        x = oracle_mod.lib().ora_splitmix_next_unit(ctypes.byref(a))
        assert x == oracle_mod.lib().ora_splitmix_next_unit(ctypes.byref(b)) and 0.0 <= x < 1.0
    assert a.value == b.value


def _grid_spec(gravity=(0.0, 0.0, 0.0), friction=0.4):
    from litter_physics_b200 import research

    return research.base_spec(grid_spacing=0.002, domain=[0.02] * 3, initial_size=[0.01] * 3,
                              wall_friction=friction, gravity=gravity, max_dt=1e-3, min_dt=1e-9)


def test_wall_decomposition_slide_stick_corner(oracle_mod):
    """solver.rs:1305-1358: per-node wall energy decomposition with exact node values."""
    spec = _grid_spec()
    mass = 1e-6
    cases = [((5, 5, 0), [1.0, 0.0, -0.5]), ((6, 5, 0), [0.1, 0.0, -0.5]), ((0, 5, 0), [-0.3, 0.2, -0.4]),
             ((7, 5, 0), [0.3, 0.0, 0.2])]
    trials = []
    for coords, v in cases:
        v = np.array(v)
        vel, imp, proj, fric = oracle_mod.grid_update_node(spec, coords, mass, v * mass, [0, 0, 0], 1e-3)
        jump = 0.5 * mass * (vel @ vel - v @ v)
        assert abs(jump - (proj - fric)) <= 1e-15 * max(abs(jump), 1e-12)
        assert proj <= 0.0 and fric >= 0.0
        assert np.linalg.norm((vel - v) * mass - imp) < 1e-20
        trials.append((vel, imp, proj, fric))
    assert abs(trials[0][2] + 0.5 * mass * 0.25) < 1e-20
    assert abs(trials[0][3] - 0.5 * mass * (1.0 - 0.8**2)) < 1e-20
    assert np.linalg.norm(trials[0][0] - np.array([0.8, 0, 0])) < 1e-15
    assert abs(trials[1][3] - 0.5 * mass * 0.01) < 1e-20 and np.all(trials[1][0] == 0.0)
    assert trials[2][0][0] == 0.0 and trials[2][0][2] == 0.0
    assert trials[3][2] == 0.0 and trials[3][3] == 0.0 and np.all(trials[3][1] == 0.0)


def test_pashias_and_hydrostatic_initial_state(oracle_mod):
    """fixtures.rs:671-684, 723-736."""
    from litter_physics_b200 import research

    liquid = research.material_liquid(1000.0, 1e5, 0.2, 1e-3)
    s = research.base_spec(fixture=1, grid_spacing=0.002, domain=[0.02] * 3, initial_size=[0.02, 0.02, 0.01],
                           wall_friction=0.4, max_dt=1e-3, min_dt=1e-9, seed=1, contact_stiffness=1000.0,
                           contact_restitution=0.2, contact_friction=0.4)
    s.material = liquid
    obs = oracle_mod.OracleSim(s).observables()
    assert obs["hydrostatic_max_relative_error"] < 1e-12 and abs(obs["mass_residual_kg"]) < 1e-18
    h0 = 0.02
    shear_yield = 0.1 * 1000.0 * 9.81 * h0
    s2 = research.base_spec(fixture=0, grid_spacing=0.002, domain=[0.02] * 3, initial_size=[0.01, 0.01, h0],
                            wall_friction=0.4, max_dt=1e-3, min_dt=1e-9, seed=1, contact_stiffness=1000.0,
                            contact_restitution=0.2, contact_friction=0.4)
    s2.material = research.material_paste(1000.0, 1e4, 0.3, shear_yield * math.sqrt(3.0), 1.0, 1.0)
    obs = oracle_mod.OracleSim(s2).observables()
    assert abs(obs["pashias_slump_m"] - h0 * (1.0 - 0.2 * (1.0 - math.log(0.2)))) < 1e-12
    assert abs(obs["dimensionless_yield_stress"] - 0.1) < 1e-12
