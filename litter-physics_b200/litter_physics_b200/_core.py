"""Drop-in for the reference's compiled extension `litter_physics._core` (core/src/lib.rs:11-57,
python/litter_physics/_core.pyi): `protocol_version()` and `run_json(request_json, resume_json)`.

Research mode runs on the GPU through `research.run`; household mode (the DEM litter model) is
not part of the GPU substep and is refused with ValueError, as the reference refuses any request it cannot run.
Every failure surfaces as ValueError, like the PyO3 binding's `PyValueError`.
"""

from __future__ import annotations

import json

PROTOCOL_VERSION = 1
MAX_JSON_BYTES = 256 * 1024 * 1024  # lib.rs:25


def protocol_version() -> int:
    """lib.rs:11-16."""
    return PROTOCOL_VERSION


def _reject_constants(name: str):
    raise ValueError(f"invalid JSON number `{name}`")


def run_json(request_json: str, resume_json: str | None = None) -> str:
    """lib.rs:18-50: parse, dispatch on `mode`, serialise the output."""
    from . import research
    from ._lib import LPError

    if len(request_json) > MAX_JSON_BYTES or (resume_json is not None and len(resume_json) > MAX_JSON_BYTES):
        raise ValueError("native JSON input exceeds 256 MiB")
    try:
        request = json.loads(request_json, parse_constant=_reject_constants)
    except (json.JSONDecodeError, ValueError) as e:
        raise ValueError(f"invalid request JSON: {e}") from e
    resume = None
    if resume_json is not None:
        try:
            resume = json.loads(resume_json, parse_constant=_reject_constants)
        except (json.JSONDecodeError, ValueError) as e:
            raise ValueError(f"invalid checkpoint JSON: {e}") from e
    mode = request.get("mode") if isinstance(request, dict) else None
    if mode == "household":
        raise ValueError("household mode is not supported by this core (research mode only)")
    if mode != "research":
        raise ValueError("mode must be household or research")
    try:
        output = research.run(request, resume)
    except (research.SpecError, research.RunError, LPError, KeyError, TypeError) as e:
        raise ValueError(str(e)) from e
    return json.dumps(output, allow_nan=False)
