"""Refinement studies on the batched launch (python/litter_physics/verification.py, tests/test_verification.py).

CPU tests restate the reference's study tests with an injected batch runner whose observables
converge like exact + c h^order + c_t dt: specification and grid-fit checks fail closed, the
per-observable verdicts, and whole studies that pass, stay unresolved, or fail the timestep
binding and fidelity gates.  The GPU test runs a real spatial study as one device batch and
checks each case against `research.run` of that case alone."""

from __future__ import annotations

import json
import math
from pathlib import Path

import pytest

from conftest import load_request
from test_research_run import small_request


def base_request() -> dict:
    return load_request("research_slump")


def spec_payload(base: str = "base.json", **overrides) -> dict:
    """test_verification.py:121-142."""
    payload = {
        "base_request": base,
        "label": "test",
        "spatial": {"grid_spacings_m": [0.01, 0.005, 0.0025], "dt_s": 0.0001},
        "temporal": {"grid_spacing_m": 0.01, "dt_values_s": [0.0004, 0.0002, 0.0001]},
        "observables": [{"name": "slump_m", "near_zero_scale": 0.0005}],
        "per_case_wall_budget_s": 60.0,
        "total_wall_budget_s": 300.0,
    }
    payload.update(overrides)
    return payload


def write_spec(tmp_path: Path, payload: dict, base: dict | None = None) -> Path:
    (tmp_path / "base.json").write_text(json.dumps(base or base_request()))
    path = tmp_path / "study.json"
    path.write_text(json.dumps(payload))
    return path


class RefinementFakeRunner:
    """test_verification.py:52-118 for a batch: observables converge like
    exact + c h^order + c_t dt and report the adaptive-step diagnostics as the kernel does."""

    def __init__(self, *, order=2.0, exact=0.01, coefficient=1.0, dt_coefficient=1.0, binding=True,
                 diagnostics=None, fidelity="research_unvalidated", fail_with=None):
        self.order, self.exact, self.coefficient, self.dt_coefficient = order, exact, coefficient, dt_coefficient
        self.binding, self.diagnostics, self.fidelity, self.fail_with = binding, diagnostics or {}, fidelity, fail_with
        self.calls: list = []

    def __call__(self, reqs: list) -> list:
        self.calls.append(len(reqs))
        if self.fail_with:
            return [ValueError(self.fail_with) for _ in reqs]
        out = []
        for r in reqs:
            h, dt = float(r["research"]["grid_spacing_m"]), float(r["dt_s"])
            obs = {"slump_m": self.exact + self.coefficient * h**self.order + self.dt_coefficient * dt,
                   "mass_residual_kg": 0.0, "max_dt_s": dt if self.binding else 0.5 * dt,
                   "step_count": float(round(r["duration_s"] / dt)), "rejected_steps": 0.0, "limited_steps": 0.0}
            for name, v in self.diagnostics.items():
                if v is None:
                    obs.pop(name)
                else:
                    obs[name] = v
            out.append({"status": "completed", "time_s": r["duration_s"], "fidelity": self.fidelity,
                        "observables": obs})
        return out


def test_spec_plans_six_grid_fitting_cases():
    """test_verification.py:156-169."""
    from litter_physics_b200.verification import plan_cases, validate_study

    spec = validate_study(spec_payload(spatial={"grid_spacings_m": [0.01, 0.005, 0.0025], "dt_s": 0.00005},
                                       temporal={"grid_spacing_m": 0.005, "dt_values_s": [0.0004, 0.0002, 0.0001]}))
    cases = plan_cases(spec, base_request())
    assert [c["axis"] for c in cases] == ["spatial"] * 3 + ["temporal"] * 3
    assert {c["request"]["dt_s"] for c in cases[:3]} == {0.00005}
    assert {c["request"]["research"]["grid_spacing_m"] for c in cases[3:]} == {0.005}
    assert {c["request"]["seed"] for c in cases} == {7}


@pytest.mark.parametrize("override, match", [
    ({"spatial": {"grid_spacings_m": [0.01, 0.005], "dt_s": 0.0001}}, "at least 3"),
    ({"spatial": {"grid_spacings_m": [0.005, 0.01, 0.0025], "dt_s": 0.0001}}, "decreasing"),
    ({"spatial": None, "temporal": None}, "needs"),
    ({"observables": [{"name": "slump_m", "near_zero_scale": 1.0}, {"name": "slump_m", "near_zero_scale": 1.0}]},
     "unique"),
    ({"max_relative_change": 0.1}, "less than or equal"),
    ({"per_case_wall_budget_s": 3601.0}, "less than or equal"),
    ({"observables": [{"name": "slump_m", "near_zero_scale": 0.0}]}, "greater than 0"),
])
def test_spec_validation(override, match):
    """test_verification.py:172-197."""
    from litter_physics_b200.verification import validate_study

    with pytest.raises(ValueError, match=match):
        validate_study(spec_payload(**override))


@pytest.mark.parametrize("path, value, match", [
    ("research.grid_spacing_m", 0.007, "integer multiple"),
    ("research.initial_size_m", [0.021, 0.02, 0.02], "subcells"),
    ("research.initial_size_m", [0.004, 0.02, 0.02], "at least one cell"),
    ("record_interval_s", 0.0001, "point samples"),
])
def test_grid_fit_fails_closed(path, value, match):
    """test_verification.py:200-217."""
    from litter_physics_b200.sweep import set_by_path
    from litter_physics_b200.verification import StudyPlanError, check_grid_fit

    payload = base_request()
    payload["dt_s"] = 0.0001
    set_by_path(payload, path, value)
    with pytest.raises(StudyPlanError, match=match):
        check_grid_fit(payload, "case")


def test_particle_cap_fails_closed():
    """test_verification.py:220-230."""
    from litter_physics_b200.verification import StudyPlanError, check_grid_fit

    payload = base_request()
    payload["research"]["domain_m"] = [0.12, 0.12, 0.12]
    payload["research"]["initial_size_m"] = [0.12, 0.12, 0.12]
    payload["research"]["grid_spacing_m"] = 0.004
    payload["record_interval_s"] = 0.5
    with pytest.raises(StudyPlanError, match="particles"):
        check_grid_fit(payload, "case")


def test_plan_rejects_non_research_base():
    """test_verification.py:270-274."""
    from litter_physics_b200.verification import StudyPlanError, plan_cases, validate_study

    household = {"schema_version": 1, "mode": "household", "seed": 1, "duration_s": 1.0}
    with pytest.raises(StudyPlanError, match="research request"):
        plan_cases(validate_study(spec_payload()), household)


def test_evaluate_observable_verdicts():
    """test_verification.py:277-302: pass, unresolved, uninformative, missing and nonfinite."""
    from litter_physics_b200.verification import evaluate_observable

    observable = {"name": "x", "near_zero_scale": 1e-3}
    h = [0.04, 0.02, 0.01]
    passed = evaluate_observable(observable, h, [1.16, 1.04, 1.01], 0.05)
    assert passed["outcome"] == "passed" and passed["trend"] == "decreasing"
    assert passed["observed_order"] is not None and math.isclose(passed["observed_order"], 2.0)
    assert passed["final_relative_change"] < 0.05
    unresolved = evaluate_observable(observable, h, [1.0, 1.2, 1.5], 0.05)
    assert unresolved["outcome"] == "unresolved" and unresolved["trend"] == "non_monotone"
    tiny = evaluate_observable(observable, h, [1e-5, 2e-6, 1e-6], 0.05)
    assert tiny["outcome"] == "uninformative" and tiny["near_zero"]
    missing = evaluate_observable(observable, h, [1.0, None, 1.0], 0.05)
    assert missing["outcome"] == "missing" and missing["observed_order"] is None
    nonfinite = evaluate_observable(observable, h, [1.0, math.nan, 1.0], 0.05)
    assert nonfinite["outcome"] == "nonfinite"
    boundary = evaluate_observable(observable, h, [1.0, 1.0, 1.06], 0.05)
    assert boundary["outcome"] == "unresolved"
    assert math.isclose(boundary["final_relative_change"], 0.06 / 1.06)
    assert evaluate_observable(observable, [0.04, 0.02, 0.015], [1.16, 1.04, 1.01], 0.05)["observed_order"] is None
    with pytest.raises(ValueError, match="at least 3"):
        evaluate_observable(observable, [0.1, 0.05], [1.0, 1.0], 0.05)
    # a small change in a large error is still a pass of the change criterion (test_verification.py:261-267)
    hydro = evaluate_observable({"name": "e", "near_zero_scale": 0.001}, [0.004, 0.002, 0.001], [0.31, 0.30, 0.299],
                                0.05)
    assert hydro["outcome"] == "passed" and hydro["values"][-1] == 0.299


def test_study_passes_in_one_batch_and_refuses_overwrite(tmp_path):
    """test_verification.py:305-322: a convergent kernel passes both axes; all six cases run
    in one batch; the study directory is write-once."""
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload())
    runner = RefinementFakeRunner(coefficient=0.1, dt_coefficient=0.1)
    report = run_study(spec, tmp_path / "study", runner=runner)
    assert runner.calls == [6]
    assert report["outcome"] == "passed" and report["study_complete"] and report["criterion_met"]
    assert report["fidelity"] == "research_unvalidated"
    assert [a["timestep_cap_binding"] for a in report["axes"]] == [True, True]
    assert report["omitted_gates"] and "validation" in report["claim"]
    written = json.loads((tmp_path / "study" / "study_report.json").read_text())
    assert written["outcome"] == "passed"
    assert (tmp_path / "study" / "cases" / "spatial" / "0002" / "output.json").is_file()
    assert (tmp_path / "study" / "study_spec.json").is_file()
    with pytest.raises(FileExistsError):
        run_study(spec, tmp_path / "study", runner=runner)


def test_study_unresolved_when_not_converged(tmp_path):
    """test_verification.py:325-334."""
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload(temporal=None))
    report = run_study(spec, tmp_path / "study", runner=RefinementFakeRunner(coefficient=200.0))
    assert report["study_complete"] and not report["criterion_met"] and report["outcome"] == "unresolved"
    verdict = report["axes"][0]["observables"][0]
    assert verdict["outcome"] == "unresolved" and math.isclose(verdict["observed_order"], 2.0)


def test_study_unresolved_when_cap_not_binding(tmp_path):
    """test_verification.py:337-344."""
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload(spatial=None))
    axis = run_study(spec, tmp_path / "study", runner=RefinementFakeRunner(binding=False))["axes"][0]
    assert axis["complete"] and axis["timestep_cap_binding"] is False and axis["outcome"] == "unresolved"
    assert any("does not equal `dt_s`" in r for r in axis["reasons"])


@pytest.mark.parametrize("diagnostics, match", [
    ({"limited_steps": None}, "`limited_steps` is None"),
    ({"limited_steps": 1.0}, "`limited_steps` 1 > 0"),
    ({"rejected_steps": 2.0}, "`rejected_steps` 2 > 0"),
    ({"step_count": 12.5}, "not a finite nonnegative integer"),
    ({"step_count": -1.0}, "not a finite nonnegative integer"),
    ({"step_count": 0.0}, "is zero"),
    ({"max_dt_s": None}, "`max_dt_s` None"),
])
def test_adaptive_diagnostics_fail_closed(tmp_path, diagnostics, match):
    """test_verification.py:347-370."""
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload(temporal=None))
    report = run_study(spec, tmp_path / "study", runner=RefinementFakeRunner(coefficient=0.1, diagnostics=diagnostics))
    axis = report["axes"][0]
    assert axis["complete"] and axis["timestep_cap_binding"] is False and axis["outcome"] == "unresolved"
    assert any(match in r for r in axis["reasons"]), axis["reasons"]
    assert report["outcome"] == "unresolved"


def test_non_research_fidelity_cannot_pass(tmp_path):
    """test_verification.py:373-383."""
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload(temporal=None))
    report = run_study(spec, tmp_path / "study",
                       runner=RefinementFakeRunner(coefficient=0.1, fidelity="preliminary_household"))
    assert report["study_complete"] and not report["criterion_met"] and report["outcome"] == "unresolved"
    assert report["fidelity"] == "preliminary_household"
    assert any("fidelity" in r for r in report["axes"][0]["reasons"])
    assert any("fidelity" in r for r in report["reasons"])


def test_failed_batch_leaves_study_incomplete(tmp_path):
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload())
    report = run_study(spec, tmp_path / "study", runner=RefinementFakeRunner(fail_with="fake kernel diverged"))
    assert report["outcome"] == "incomplete" and not report["study_complete"]
    assert all(c["status"] == "failed" and "diverged" in c["error"] for a in report["axes"] for c in a["cases"])


def test_exhausted_study_budget_starts_nothing(tmp_path):
    from litter_physics_b200.verification import run_study

    spec = write_spec(tmp_path, spec_payload(total_wall_budget_s=10.0))
    clock = {"now": 0.0}

    def fake_clock() -> float:
        clock["now"] += 9.0
        return clock["now"]

    runner = RefinementFakeRunner()
    report = run_study(spec, tmp_path / "study", runner=runner, clock=fake_clock)
    assert runner.calls == []
    assert report["outcome"] == "incomplete"
    assert {c["status"] for a in report["axes"] for c in a["cases"]} == {"not_started"}


# ---------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_real_study_runs_in_one_batch_and_matches_single_runs(tmp_path):
    """A spatial study of the small slump (three grids at one step cap) through the device batch:
    it completes with an honest verdict, and each case equals `research.run` of that case."""
    from litter_physics_b200 import _lib, research
    from litter_physics_b200.verification import plan_cases, run_study, validate_study

    _lib.build()
    payload = spec_payload(spatial={"grid_spacings_m": [0.01, 0.005, 0.0025], "dt_s": 0.00005}, temporal=None,
                           observables=[{"name": "slump_m", "near_zero_scale": 0.0001},
                                        {"name": "plastic_dissipation_j", "near_zero_scale": 1e-9}])
    spec = write_spec(tmp_path, payload, base=small_request())
    report = run_study(spec, tmp_path / "study")
    assert report["study_complete"], report["reasons"]
    assert report["outcome"] in ("passed", "unresolved")
    cases = plan_cases(validate_study(payload), small_request())
    for case, outcome in zip(cases, report["axes"][0]["cases"], strict=True):
        alone = json.loads(json.dumps(research.run(case["request"])))
        assert outcome["observables"] == alone["observables"], case["case_index"]
