"""Host-side request mapping (research.rs:137-305) and workload definitions, on CPU."""

from __future__ import annotations

import copy
import math

import pytest

from conftest import load_request


def test_examples_map_to_expected_specs():
    from litter_physics_b200 import _abi, research

    s = research.spec_from_request(load_request("research_slump"))
    assert s.fixture == _abi.LP_SLUMP and s.seed == 7 and s.max_dt == 1e-4
    assert s.material.yield_stress == pytest.approx(math.sqrt(3.0) * 30.0)
    assert s.material.consistency == pytest.approx(3 ** 0.8 * 10.0)
    assert research.particle_count(s) == 512
    h = research.spec_from_request(load_request("research_hydrostatic_water"))
    assert h.material.kind == _abi.LP_LIQUID and research.particle_count(h) == 4000
    c = research.spec_from_request(load_request("research_coupled_patch"))
    assert c.has_pellet == 1 and c.pellet_radius == 0.003 and research.particle_count(c) == 8000


@pytest.mark.parametrize(
    "mutate,message",
    [
        (lambda r: r.update(mode="household"), "mode=research"),
        (lambda r: r.update(dt_s=-1.0), "finite and positive"),
        (lambda r: r["research"].update(material="fines"), "Drucker-Prager"),
        (lambda r: r["research"].update(material="water"), "zero yield stress"),
        (lambda r: r["research"].update(poisson_ratio=0.5), "Poisson"),
        (lambda r: r["research"].update(fixture="tornado"), "unsupported research fixture"),
        (lambda r: r["research"].update(initial_size_m=[0.021, 0.02, 0.02]), "whole particle subcells"),
        (lambda r: r["research"].update(extra=1), "unknown field"),
        (lambda r: r.update(max_wall_time_s=4000.0), "3600"),
    ],
)
def test_invalid_requests_are_rejected(mutate, message):
    from litter_physics_b200 import research

    req = copy.deepcopy(load_request("research_slump"))
    mutate(req)
    with pytest.raises(research.SpecError, match=message):
        research.spec_from_request(req)


def test_particle_cap_is_enforced_before_allocation():
    from litter_physics_b200 import research

    req = copy.deepcopy(load_request("research_slump"))
    req["research"].update(grid_spacing_m=0.001, initial_size_m=[0.03, 0.03, 0.03], domain_m=[0.06] * 3)
    with pytest.raises(research.SpecError, match="exceeding the cap"):
        research.spec_from_request(req)


def test_benchmark_workloads_have_the_stated_sizes():
    from litter_physics_b200 import configs, research

    assert research.particle_count(configs.config0()) == 65_536
    assert research.particle_count(configs.config1()) == 1_048_576
    assert research.particle_count(configs.config2()) == 16_777_216
    batch = configs.config3()
    counts = [research.particle_count(s) for s in batch]
    assert len(batch) == 256 and min(counts) >= 4_000 and max(counts) <= 300_000
    assert [s.seed for s in batch] == list(range(100, 356))
    c0 = configs.config0()
    assert c0.face_mode_enabled == 1 and c0.face_sticky[4] == 1 and c0.face_friction[0] == 0.0
    e, nu = configs.young_poisson(2e4, 1e5)
    assert e == pytest.approx(56_250.0) and nu == pytest.approx(0.40625)


def test_oracle_runs_the_extensions(oracle_mod):
    """Extensions in the oracle: sticky floor + per-particle yield + Tait reduce to finite runs."""
    from litter_physics_b200 import configs

    s = configs.slump(16, (4, 4, 8), seed=3, yield_range=(20.0, 100.0))
    sim = oracle_mod.OracleSim(s)
    sim.advance_to(20 * s.max_dt)
    p = sim.particles()
    assert p["yield_stress"].min() >= math.sqrt(3) * 20.0 and p["yield_stress"].max() <= math.sqrt(3) * 100.0
    assert sim.counters().step_count == 20
    d = configs.dam_break(16, (8, 4, 8), seed=1)
    sim = oracle_mod.OracleSim(d)
    sim.advance_to(20 * d.max_dt)
    assert sim.counters().rejected_steps == 0
