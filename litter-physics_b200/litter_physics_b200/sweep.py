"""Parameter sweeps on the batched launch (python/litter_physics/sweep.py).

A sweep specification names a base research request and dotted-path overrides; the grid
product times the seed offsets gives one job per combination, validated before anything runs
(`expand_jobs`, sweep.py:170-203).  The reference runs the jobs one after another
(`run_sweep`, sweep.py:206-262).  Here every group of jobs that shares the record schedule
(`duration_s`, `record_interval_s`) and the fixture kind runs as ONE device batch
(`research.run_batch`): all of its instances advance in the same launch sequence with their own
dt control, and each job's output is what `research.run` returns for that job alone.  The
summary files keep the reference's names and columns.

Budgets: the reference gives every job its own wall budget and a sweep budget that only stops
STARTING jobs.  A batch starts all of its jobs together, so the sweep budget stops starting
groups, and a group runs under the smallest `max_wall_time_s` of its jobs.
"""

from __future__ import annotations

import copy
import itertools
import json
import os
import time
from pathlib import Path
from typing import Any, Callable

MAX_SWEEP_JOBS = 10_000
SUMMARY_FILE = "sweep_summary.json"
SUMMARY_TABLE = "sweep_summary.parquet"
JOBS_DIR = "jobs"

_SPEC_KEYS = {"base_request", "axes", "seeds", "label"}


def validate_spec(doc: Any) -> dict:
    """`SweepSpec` (sweep.py:55-66): base_request, axes (>= 1 of {path, values}), seeds
    (default [0]), label (default "sweep"); unknown keys are refused."""
    if not isinstance(doc, dict):
        raise ValueError("sweep specification must be a mapping")
    extra = set(doc) - _SPEC_KEYS
    if extra:
        raise ValueError(f"sweep specification has unknown fields {sorted(extra)}")
    base = doc.get("base_request")
    if not isinstance(base, str):
        raise ValueError("sweep specification needs a `base_request` path")
    axes = doc.get("axes")
    if not isinstance(axes, list) or not axes:
        raise ValueError("sweep specification needs at least one axis")
    out_axes = []
    for axis in axes:
        if not isinstance(axis, dict) or set(axis) - {"path", "values"}:
            raise ValueError("each sweep axis has exactly `path` and `values`")
        path, values = axis.get("path"), axis.get("values")
        if not isinstance(path, str) or not path:
            raise ValueError("sweep axis `path` must be a non-empty string")
        if not isinstance(values, list) or not values:
            raise ValueError(f"sweep axis '{path}' needs at least one value")
        out_axes.append({"path": path, "values": list(values)})
    seeds = doc.get("seeds", [0])
    if not isinstance(seeds, list) or not all(isinstance(s, int) and not isinstance(s, bool) for s in seeds):
        raise ValueError("sweep `seeds` must be a list of integers")
    label = doc.get("label", "sweep")
    if not isinstance(label, str):
        raise ValueError("sweep `label` must be a string")
    return {"base_request": base, "axes": out_axes, "seeds": list(seeds), "label": label}


def load_document(path: Path) -> Any:
    """YAML or JSON document."""
    text = Path(path).read_text()
    if str(path).endswith(".json"):
        return json.loads(text)
    import yaml

    return yaml.safe_load(text)


def load_spec(path: Path) -> dict:
    """sweep.py:158-167."""
    return validate_spec(load_document(path))


def _list_index(part: str, path: str) -> int:
    if not part.isdigit():
        raise TypeError(f"path '{path}' indexes a list with non-integer '{part}'")
    return int(part)


def _descend(node: Any, part: str, path: str) -> Any:
    if isinstance(node, list):
        return node[_list_index(part, path)]
    if isinstance(node, dict):
        if part not in node:
            raise KeyError(f"path '{path}' names unknown key '{part}'")
        return node[part]
    raise TypeError(f"path '{path}' descends into a scalar at '{part}'")


def set_by_path(payload: dict, path: str, value: Any) -> None:
    """Assign into a nested JSON-like tree by dotted path (sweep.py:88-116): KeyError for an
    unknown key, IndexError for an index past the end, TypeError for a non-integer list index
    or a path through a scalar."""
    parts = path.split(".")
    node: Any = payload
    for part in parts[:-1]:
        node = _descend(node, part, path)
    last = parts[-1]
    if isinstance(node, list):
        node[_list_index(last, path)] = value
    elif isinstance(node, dict):
        if last not in node:
            raise KeyError(f"path '{path}' names unknown key '{last}'")
        node[last] = value
    else:
        raise TypeError(f"path '{path}' descends into a scalar at '{last}'")


def expand_jobs(spec: dict, base: dict) -> list:
    """sweep.py:170-203: (overrides, seed, request) per grid point and seed offset, in
    `itertools.product` order with seeds innermost; every request is validated first."""
    from . import research

    combos = list(itertools.product(*[axis["values"] for axis in spec["axes"]]))
    total = len(combos) * len(spec["seeds"])
    if total > MAX_SWEEP_JOBS:
        raise ValueError(f"sweep expands to {total} jobs, above the cap {MAX_SWEEP_JOBS}")
    jobs = []
    for combo in combos:
        for seed_offset in spec["seeds"]:
            payload = copy.deepcopy(base)
            overrides = {axis["path"]: value for axis, value in zip(spec["axes"], combo, strict=True)}
            for path, value in overrides.items():
                set_by_path(payload, path, value)
            seed = int(base["seed"]) + seed_offset
            payload["seed"] = seed
            try:
                research.spec_from_request(payload)
            except (ValueError, KeyError, TypeError) as e:
                raise ValueError(f"sweep job with overrides {overrides} is invalid: {e}") from e
            jobs.append((overrides, seed, payload))
    return jobs


def group_jobs(jobs: list) -> list:
    """Job indices grouped by (duration, record interval, fixture), in order of first job."""
    groups: dict = {}
    for k, (_, _, req) in enumerate(jobs):
        key = (float(req["duration_s"]), float(req["record_interval_s"]), req["research"]["fixture"])
        groups.setdefault(key, []).append(k)
    return list(groups.values())


def _outcome(job_index: int, run_dir: Path, overrides: dict, seed: int, status: str, time_s, wall_time_s,
             observables: dict, error) -> dict:
    """`JobOutcome` (sweep.py:69-85)."""
    return {"job_index": job_index, "run_dir": str(run_dir), "overrides": overrides, "seed": seed,
            "status": status, "time_s": time_s, "wall_time_s": wall_time_s, "observables": observables,
            "error": error}


def _write_atomic(path: Path, text: str) -> None:
    tmp = path.with_name(path.name + ".tmp")
    tmp.write_text(text)
    os.replace(tmp, path)


def _write_summary(root: Path, spec: dict, outcomes: list) -> None:
    """sweep.py:319-352: JSON summary with status counts and a Parquet table."""
    payload = {
        "label": spec["label"],
        "axes": spec["axes"],
        "jobs": outcomes,
        "counts": {status: sum(1 for o in outcomes if o["status"] == status)
                   for status in sorted({o["status"] for o in outcomes})},
    }
    _write_atomic(root / SUMMARY_FILE, json.dumps(payload, indent=1))
    import pyarrow as pa
    import pyarrow.parquet as pq

    rows: dict = {
        "job_index": [o["job_index"] for o in outcomes],
        "seed": [o["seed"] for o in outcomes],
        "status": [o["status"] for o in outcomes],
        "time_s": [o["time_s"] for o in outcomes],
        "wall_time_s": [o["wall_time_s"] for o in outcomes],
        "run_dir": [o["run_dir"] for o in outcomes],
    }
    for axis in spec["axes"]:
        rows[f"override:{axis['path']}"] = [str(o["overrides"].get(axis["path"])) for o in outcomes]
    table_path = root / SUMMARY_TABLE
    if table_path.exists():
        raise FileExistsError(f"refusing to overwrite '{table_path}'")
    pq.write_table(pa.table(rows), table_path)


def run_sweep(spec_path: Path, sweep_dir: Path, *, runner: Callable[[list], list] | None = None,
              total_wall_budget_s: float | None = None, write_outputs: bool = True,
              clock: Callable[[], float] = time.monotonic) -> list:
    """Run every job, one device batch per group of jobs with a shared record schedule.

    `runner(requests)` returns one research output (or exception) per request; the default is
    `research.run_batch`.  Each job's output goes to `jobs/NNNN/output.json` when
    `write_outputs`.  Raises FileExistsError when `sweep_dir` already has content, and
    ValueError (before creating anything) when a job is invalid."""
    from . import research

    runner = runner or research.run_batch
    started = clock()
    spec = load_spec(spec_path)
    base_path = (Path(str(spec_path)).resolve().parent / spec["base_request"]).resolve()
    base = load_document(base_path)
    jobs = expand_jobs(spec, base)
    root = Path(str(sweep_dir)).resolve()
    if root.exists() and any(root.iterdir()):
        raise FileExistsError(f"Sweep directory '{root}' is not empty; refusing to overwrite")
    root.mkdir(parents=True, exist_ok=True)
    outcomes: list = [None] * len(jobs)
    for group in group_jobs(jobs):
        if total_wall_budget_s is not None and clock() - started >= total_wall_budget_s:
            for k in group:
                overrides, seed, _ = jobs[k]
                outcomes[k] = _outcome(k, root / JOBS_DIR / f"{k:04d}", overrides, seed, "not_started", None, None,
                                       {}, None)
            continue
        t0 = clock()
        try:
            results = runner([jobs[k][2] for k in group])
        except (ValueError, RuntimeError) as e:
            results = [e] * len(group)
        wall = clock() - t0
        for k, result in zip(group, results, strict=True):
            overrides, seed, _ = jobs[k]
            run_dir = root / JOBS_DIR / f"{k:04d}"
            if isinstance(result, BaseException):
                outcomes[k] = _outcome(k, run_dir, overrides, seed, "failed", None, None, {}, str(result))
                continue
            if write_outputs:
                run_dir.mkdir(parents=True, exist_ok=True)
                _write_atomic(run_dir / "output.json", json.dumps(result))
            outcomes[k] = _outcome(k, run_dir, overrides, seed, str(result["status"]), result["time_s"], wall,
                                   dict(result["observables"]), None)
    _write_summary(root, spec, outcomes)
    return outcomes


def read_summary(root: Path):
    """sweep.py:355-364."""
    import pyarrow.parquet as pq

    return pq.read_table(Path(str(root)).resolve() / SUMMARY_TABLE)
