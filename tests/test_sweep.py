"""Parameter sweeps on the batched launch (python/litter_physics/sweep.py, tests/test_sweep_benchmark.py).

CPU tests restate the reference's sweep tests with an injected runner in place of its fake
core: dotted-path errors, grid expansion with seed offsets, per-job statuses, the summary
files, the sweep budget, failure recording and up-front validation.  The GPU test runs a real
sweep as one device batch and checks every job's output against `research.run` of that job
alone: batched instances step exactly like single simulations, so they agree bit for bit."""

from __future__ import annotations

import json
from pathlib import Path

import pytest

from test_research_run import small_request


def write_sweep(tmp_path: Path, axes: list, seeds=(0, 1), base: dict | None = None) -> Path:
    (tmp_path / "base.json").write_text(json.dumps(base or small_request()))
    spec = {"base_request": "base.json", "label": "yield-and-flow", "seeds": list(seeds), "axes": axes}
    path = tmp_path / "sweep.json"
    path.write_text(json.dumps(spec))
    return path


AXES = [{"path": "research.yield_stress_pa", "values": [20.0, 40.0]},
        {"path": "research.flow_index", "values": [0.5, 0.8]}]


class FakeRunner:
    """Stands in for the device batch: one output per request, or a failure for each."""

    def __init__(self, fail_with: str | None = None):
        self.calls: list = []
        self.fail_with = fail_with

    def __call__(self, reqs: list) -> list:
        self.calls.append(len(reqs))
        if self.fail_with:
            return [RuntimeError(self.fail_with) for _ in reqs]
        return [{"status": "completed", "time_s": r["duration_s"],
                 "observables": {"yield": r["research"]["yield_stress_pa"], "seed": float(r["seed"])}}
                for r in reqs]


def test_set_by_path_errors():
    """test_sweep_benchmark.py:22-35."""
    from litter_physics_b200.sweep import set_by_path

    tree = {"a": {"b": [1, 2]}, "c": 1}
    set_by_path(tree, "a.b.1", 5)
    assert tree["a"]["b"] == [1, 5]
    with pytest.raises(KeyError):
        set_by_path(tree, "a.zzz", 1)
    with pytest.raises(TypeError):
        set_by_path(tree, "a.b.x", 1)
    with pytest.raises(TypeError):
        set_by_path(tree, "c.d", 1)
    with pytest.raises(IndexError):
        set_by_path(tree, "a.b.9", 1)


def test_expand_and_run_sweep(tmp_path):
    """test_sweep_benchmark.py:38-56: 2 x 2 grid points x 2 seeds; one batch for all eight."""
    from litter_physics_b200.sweep import expand_jobs, load_document, load_spec, read_summary, run_sweep

    path = write_sweep(tmp_path, AXES)
    spec = load_spec(path)
    jobs = expand_jobs(spec, load_document(tmp_path / "base.json"))
    assert len(jobs) == 8
    assert {job[1] for job in jobs} == {3, 4}
    assert [job[0]["research.yield_stress_pa"] for job in jobs] == [20.0] * 4 + [40.0] * 4
    assert [job[2]["research"]["flow_index"] for job in jobs][:4] == [0.5, 0.5, 0.8, 0.8]
    runner = FakeRunner()
    outcomes = run_sweep(path, tmp_path / "sweep", runner=runner)
    assert runner.calls == [8]
    assert all(o["status"] == "completed" for o in outcomes)
    assert [o["observables"]["seed"] for o in outcomes] == [3.0, 4.0] * 4
    table = read_summary(tmp_path / "sweep")
    assert table.num_rows == 8
    assert set(table.column_names) >= {"override:research.yield_stress_pa", "override:research.flow_index", "status"}
    summary = json.loads((tmp_path / "sweep" / "sweep_summary.json").read_text())
    assert summary["counts"] == {"completed": 8}
    assert (tmp_path / "sweep" / "jobs" / "0007" / "output.json").is_file()
    with pytest.raises(FileExistsError):
        run_sweep(path, tmp_path / "sweep", runner=runner)


def test_jobs_with_different_schedules_run_as_separate_batches(tmp_path):
    from litter_physics_b200.sweep import run_sweep

    path = write_sweep(tmp_path, [{"path": "duration_s", "values": [0.002, 0.003]},
                                  {"path": "research.yield_stress_pa", "values": [20.0, 40.0]}], seeds=[0])
    runner = FakeRunner()
    outcomes = run_sweep(path, tmp_path / "sweep", runner=runner)
    assert runner.calls == [2, 2]
    assert [o["time_s"] for o in outcomes] == [0.002, 0.002, 0.003, 0.003]


def test_sweep_total_budget_stops_starting_batches(tmp_path):
    """test_sweep_benchmark.py:59-72: a sweep budget marks unstarted jobs rather than shrinking
    running ones."""
    from litter_physics_b200.sweep import run_sweep

    path = write_sweep(tmp_path, [{"path": "duration_s", "values": [0.002, 0.003, 0.004]}], seeds=[0])
    clock = {"now": 0.0}

    def fake_clock() -> float:
        clock["now"] += 10.0
        return clock["now"]

    outcomes = run_sweep(path, tmp_path / "sweep", runner=FakeRunner(), total_wall_budget_s=25.0, clock=fake_clock)
    statuses = [o["status"] for o in outcomes]
    assert "not_started" in statuses and statuses[0] == "completed"


def test_sweep_records_failures(tmp_path):
    """test_sweep_benchmark.py:75-79."""
    from litter_physics_b200.sweep import run_sweep

    path = write_sweep(tmp_path, AXES)
    outcomes = run_sweep(path, tmp_path / "sweep", runner=FakeRunner(fail_with="solver diverged"))
    assert all(o["status"] == "failed" for o in outcomes)
    assert outcomes[0]["error"] is not None and "solver diverged" in outcomes[0]["error"]
    summary = json.loads((tmp_path / "sweep" / "sweep_summary.json").read_text())
    assert summary["counts"] == {"failed": 8}


def test_invalid_sweep_value_rejected(tmp_path):
    """test_sweep_benchmark.py:82-93: grid points are validated before any job starts."""
    from litter_physics_b200.sweep import run_sweep

    path = write_sweep(tmp_path, [{"path": "research.poisson_ratio", "values": [0.7]}])
    with pytest.raises(ValueError, match="invalid"):
        run_sweep(path, tmp_path / "sweep", runner=FakeRunner())
    assert not (tmp_path / "sweep").exists()


@pytest.mark.parametrize("doc, needle", [
    ({"base_request": "b.json", "axes": [], "label": "x"}, "at least one axis"),
    ({"base_request": "b.json", "axes": [{"path": "seed", "values": [1]}], "extra": 1}, "unknown fields"),
    ({"base_request": "b.json", "axes": [{"path": "", "values": [1]}]}, "non-empty"),
    ({"base_request": "b.json", "axes": [{"path": "seed", "values": []}]}, "at least one value"),
    ({"axes": [{"path": "seed", "values": [1]}]}, "base_request"),
])
def test_spec_validation(doc, needle):
    from litter_physics_b200.sweep import validate_spec

    with pytest.raises(ValueError, match=needle):
        validate_spec(doc)


def test_job_cap(tmp_path):
    from litter_physics_b200 import sweep

    spec = sweep.validate_spec({"base_request": "b.json", "axes": [{"path": "seed", "values": list(range(101))}],
                                "seeds": list(range(100))})
    with pytest.raises(ValueError, match="above the cap"):
        sweep.expand_jobs(spec, small_request())


# ---------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_batched_sweep_matches_single_runs(tmp_path):
    """Four slump jobs (two yield stresses x two seeds) in one device batch: each job's frames,
    metrics, observables and checkpoint equal `research.run` of that job alone."""
    from litter_physics_b200 import _lib, research
    from litter_physics_b200.sweep import expand_jobs, load_document, load_spec, run_sweep

    _lib.build()
    path = write_sweep(tmp_path, [{"path": "research.yield_stress_pa", "values": [20.0, 60.0]}])
    outcomes = run_sweep(path, tmp_path / "sweep")
    assert [o["status"] for o in outcomes] == ["completed"] * 4
    jobs = expand_jobs(load_spec(path), load_document(tmp_path / "base.json"))
    for k, (_, _, req) in enumerate(jobs):
        alone = research.run(req)
        batched = json.loads((tmp_path / "sweep" / "jobs" / f"{k:04d}" / "output.json").read_text())
        alone = json.loads(json.dumps(alone))
        for key in ("status", "time_s", "frames", "metrics", "observables", "checkpoint"):
            assert batched[key] == alone[key], (k, key)
    # different yield stresses give different results
    assert outcomes[0]["observables"] != outcomes[2]["observables"]
