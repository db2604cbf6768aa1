"""The `_core` drop-in: `protocol_version` / `run_json` and the research driver (record loop,
checkpoint, checked restore), following the reference's own tests in
core/src/research/tests.rs and core/src/lib.rs:59-66.

CPU tests cover the wire parsing, request validation and the checkpoint JSON codecs; GPU tests
run the fixtures through the device simulation."""

from __future__ import annotations

import copy
import json
import math

import numpy as np
import pytest

from conftest import load_request


def small_request() -> dict:
    """research/tests.rs:4-22."""
    return {
        "schema_version": 1, "mode": "research", "seed": 3,
        "duration_s": 0.002, "dt_s": 0.0005, "record_interval_s": 0.001,
        "max_wall_time_s": 60.0, "boxes": [], "events": [],
        "materials": {
            "friction": 0.3, "restitution": 0.1, "normal_stiffness_n_m": 1000.0,
            "water_capacity_ratio": 3.0, "uptake_rate_s": 0.1,
            "breakdown_rate_s": 0.01, "evaporation_rate_s": 0.0,
        },
        "research": {
            "fixture": "slump", "grid_spacing_m": 0.005,
            "domain_m": [0.03, 0.03, 0.03], "material": "paste",
            "density_kg_m3": 1000.0, "young_modulus_pa": 1000.0,
            "poisson_ratio": 0.2, "yield_stress_pa": 30.0,
            "consistency_pa_s_n": 10.0, "flow_index": 0.6,
            "initial_size_m": [0.01, 0.01, 0.01], "initial_velocity_m_s": [0.0, 0.0, 0.0],
        },
    }


# ---------------------------------------------------------------------------- CPU
def test_protocol_is_versioned():
    from litter_physics_b200 import _core

    assert _core.protocol_version() == 1


@pytest.mark.parametrize("text,needle", [
    ("{", "invalid request JSON"),
    ('{"mode": "household"}', "household mode is not supported"),
    ('{"mode": "audit"}', "mode must be household or research"),
    ("[1, 2]", "mode must be household or research"),
    ('{"mode": "research", "x": NaN}', "invalid request JSON"),
])
def test_run_json_rejects_bad_envelopes(text, needle):
    from litter_physics_b200 import _core

    with pytest.raises(ValueError, match=needle):
        _core.run_json(text)


def test_run_json_input_cap(monkeypatch):
    from litter_physics_b200 import _core

    monkeypatch.setattr(_core, "MAX_JSON_BYTES", 16)
    with pytest.raises(ValueError, match="exceeds 256 MiB"):
        _core.run_json(json.dumps(small_request()))
    with pytest.raises(ValueError, match="exceeds 256 MiB"):
        _core.run_json("{}", "x" * 17)


@pytest.mark.parametrize("key,value", [
    ("material", "fines"),
    ("material", "unknown"),
    ("poisson_ratio", 0.5),
    ("flow_index", 0),
    ("grid_spacing_m", 1e-300),
    ("initial_size_m", [0.011, 0.01, 0.01]),
])
def test_unsupported_fines_and_bad_parameters_fail_closed(key, value):
    """research/tests.rs:84-101: refused before any device work."""
    from litter_physics_b200 import _core

    req = small_request()
    req["research"][key] = value
    with pytest.raises(ValueError):
        _core.run_json(json.dumps(req))


def test_unknown_top_level_field_is_refused():
    from litter_physics_b200 import _core

    req = small_request()
    req["unknown"] = 1
    with pytest.raises(ValueError, match="unknown field"):
        _core.run_json(json.dumps(req))


def test_grid_layout_follows_reference_rules():
    from litter_physics_b200 import research

    assert research.grid_layout([0.03, 0.03, 0.03], 0.005, 1_000_000) == [6, 6, 6]
    with pytest.raises(research.SpecError, match="not an integer multiple"):
        research.grid_layout([0.031, 0.03, 0.03], 0.005, 1_000_000)
    with pytest.raises(research.SpecError, match="at least two cells"):
        research.grid_layout([0.005, 0.03, 0.03], 0.005, 1_000_000)
    with pytest.raises(research.SpecError, match="exceeding the cap"):
        research.grid_layout([1.0, 1.0, 1.0], 0.005, 1_000_000)


def test_particle_json_uses_nalgebra_layout_and_round_trips():
    from litter_physics_b200 import research

    rng = np.random.default_rng(0)
    n = 5
    p = {
        "id": np.arange(n, dtype=np.uint32)[::-1].copy(),
        "position": rng.uniform(0.1, 0.2, (n, 3)),
        "velocity": rng.normal(size=(n, 3)),
        "affine": rng.normal(size=(n, 3, 3)),
        "deformation": np.eye(3)[None] + 1e-3 * rng.normal(size=(n, 3, 3)),
        "volume_ratio": np.ones(n),
        "kirchhoff": rng.normal(size=(n, 3, 3)),
        "plastic_strain": rng.uniform(0, 1e-3, n),
        "mass": rng.uniform(1e-6, 2e-6, n),
        "volume0": rng.uniform(1e-9, 2e-9, n),
    }
    d = research.particles_to_json(p)
    # column-major 3x3: element (row 0, column 1) is the 4th number
    assert d["affine"][2][3] == p["affine"][2][0, 1]
    assert d["affine"][2][1] == p["affine"][2][1, 0]
    back = research.particles_from_json(json.loads(json.dumps(d)))
    for k in p:
        assert np.array_equal(back[k], p[k]), k


@pytest.mark.parametrize("mutate,needle", [
    (lambda d: d["id"].__setitem__(1, d["id"][0]), "not unique"),
    (lambda d: d["mass"].__setitem__(0, -1.0), "non-positive mass"),
    (lambda d: d["volume_ratio"].__setitem__(0, 0.0), "invalid ratio"),
    (lambda d: d["position"].pop(), "has length"),
    (lambda d: d.__setitem__("extra", []), "unknown field"),
])
def test_corrupt_particle_arrays_are_refused(mutate, needle):
    from litter_physics_b200 import research

    n = 3
    d = {
        "id": [0, 1, 2], "position": [[0.1, 0.1, 0.1]] * n, "velocity": [[0.0, 0.0, 0.0]] * n,
        "affine": [[0.0] * 9] * n, "deformation": [[1, 0, 0, 0, 1, 0, 0, 0, 1]] * n,
        "volume_ratio": [1.0] * n, "kirchhoff": [[0.0] * 9] * n, "plastic_strain": [0.0] * n,
        "mass": [1e-3] * n, "volume0": [1e-6] * n,
    }
    d = copy.deepcopy(d)
    mutate(d)
    with pytest.raises(research.RunError, match=needle):
        research.particles_from_json(d)


# ---------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def built():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


@pytest.mark.gpu
def test_completes_a_real_fixture_without_claiming_validation(built):
    """research/tests.rs:24-56."""
    from litter_physics_b200 import _core

    out = json.loads(_core.run_json(json.dumps(small_request())))
    assert out["status"] == "completed"
    assert out["fidelity"] == "research_unvalidated"
    assert len(out["frames"]) == 3
    assert any("signed grid kinetic-energy diagnostic" in m and "energy closure remains open" in m
               for m in out["diagnostics"])
    traction = out["observables"]["wall_normal_traction_energy_j"]
    assert math.isfinite(traction) and traction != 0.0, traction
    assert out["checkpoint"]["state"]["ledger"]["wall_normal_traction_energy"] == traction
    assert abs(out["observables"]["mass_residual_kg"]) < 1e-12
    assert len(out["metrics"]) == 6
    assert {m["compartment"] for m in out["metrics"]} == {"domain", "outflow"}
    assert out["checkpoint"]["time_s"] == out["time_s"] == 0.002


@pytest.mark.gpu
def test_full_state_json_round_trip_matches_uninterrupted_trajectory(built):
    """research/tests.rs:103-129: a checkpoint taken at a record boundary, serialised and
    resumed, reproduces the uninterrupted run's final checkpoint and observables."""
    from litter_physics_b200 import research
    from litter_physics_b200.sim import Simulation

    req = small_request()
    req["dt_s"] = 0.002
    spec = research.spec_from_request(req)
    with Simulation(spec) as sim:
        sim.advance_to(0.001)
        checkpoint = {"schema_version": 1, "mode": "research", "request": req, "time_s": sim.time,
                      "state": research.snapshot(sim, 2)}
    restored = json.loads(json.dumps(checkpoint))
    resumed = research.run(req, restored)
    full = research.run(req)
    assert json.dumps(resumed["checkpoint"]) == json.dumps(full["checkpoint"])
    assert resumed["observables"] == full["observables"]
    assert full["observables"]["limited_steps"] > 0.0
    assert len(resumed["frames"]) == 1
    assert resumed["frames"][0] == full["frames"][2]


@pytest.mark.gpu
def test_corrupt_checkpoint_histories_and_requests_are_rejected(built):
    """research/tests.rs:131-189."""
    from litter_physics_b200 import _core

    req = small_request()
    full = json.loads(_core.run_json(json.dumps(req)))
    base = full["checkpoint"]

    def refused(cp, r=req):
        with pytest.raises(ValueError):
            _core.run_json(json.dumps(r), json.dumps(cp))

    for key, value in (("dt_scale", 0), ("next_record_index", 0), ("limited_steps", 2**64 - 1)):
        cp = copy.deepcopy(base)
        cp["state"][key] = value
        refused(cp)
    cp = copy.deepcopy(base)
    cp["state"]["particles"]["mass"][0] = -1
    refused(cp)
    cp = copy.deepcopy(base)
    cp["state"]["particles"]["position"][0] = [100.0, 0.0, 0.0]
    refused(cp)
    cp = copy.deepcopy(base)
    cp["state"]["ledger"]["initial_mechanical_energy"] = 1.0
    refused(cp)
    cp = copy.deepcopy(base)
    del cp["state"]["ledger"]["wall_normal_traction_energy"]
    refused(cp)
    cp = copy.deepcopy(base)
    cp["state"]["ledger"]["wall_normal_traction_energy"] = None
    refused(cp)
    changed = copy.deepcopy(req)
    changed["seed"] = 99
    refused(base, changed)
    # the untouched checkpoint resumes (time already at the end: nothing left to run)
    out = json.loads(_core.run_json(json.dumps(req), json.dumps(base)))
    assert out["status"] == "completed" and out["frames"] == []


@pytest.mark.gpu
def test_budget_expiry_and_restoration_are_explicit(built):
    """research/tests.rs:191-200."""
    from litter_physics_b200 import _core

    req = small_request()
    req["max_wall_time_s"] = 1e-12
    partial = json.loads(_core.run_json(json.dumps(req)))
    assert partial["status"] == "budget_exhausted"
    req["max_wall_time_s"] = 60
    complete = json.loads(_core.run_json(json.dumps(req), json.dumps(partial["checkpoint"])))
    assert complete["status"] == "completed"


@pytest.mark.gpu
def test_research_slump_observables_match_oracle(built):
    """The shipped research slump request through run_json against the FP64 oracle driven to the
    same time.  Counters agree exactly; lengths within 1e-5 of the domain; energies and energy
    residuals within 1e-3 of the mechanical-energy scale; masses within 1e-9 of the initial
    mass; other observables within 1e-3 relative (FP32 device state against FP64)."""
    import oracle

    from litter_physics_b200 import _core, research

    req = load_request("research_slump")
    req["duration_s"] = 0.01
    req["record_interval_s"] = 0.005
    out = json.loads(_core.run_json(json.dumps(req)))
    assert out["status"] == "completed"
    spec = research.spec_from_request(req)
    ref = oracle.OracleSim(spec)
    ref.advance_to(req["duration_s"])
    robs = ref.observables()
    gobs = out["observables"]
    assert set(robs) <= set(gobs)
    mech = max(abs(robs["mechanical_energy_j"]), 1e-30)
    mass = out["checkpoint"]["state"]["ledger"]["initial_mass"]
    length = max(spec.domain)
    impulse = mass * 9.81 * req["duration_s"]  # gravity impulse: the momentum scale
    bad = []
    for name, rv in robs.items():
        gv = gobs[name]
        if name.endswith("_steps") or name in ("particle_count", "step_count"):
            tol = 0.0
        elif name.endswith("_j"):
            tol = 1e-3 * mech
        elif "momentum" in name:
            tol = 1e-6 * impulse
        elif name.endswith("_kg"):
            tol = 1e-9 * mass + 1e-15
        elif name.endswith("_m"):
            tol = 1e-5 * length
        else:
            tol = 1e-3 * max(abs(rv), 1e-12)
        print(f"{name:40s} gpu {gv:+.9e} oracle {rv:+.9e} tol {tol:.2e}")
        if not abs(gv - rv) <= tol:
            bad.append((name, gv, rv, tol))
    assert not bad, bad
