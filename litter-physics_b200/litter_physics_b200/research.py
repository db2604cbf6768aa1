"""Research wire request -> fixture specification.

Host-side restatement of `research::specification` (core/src/research.rs:171-305): the
envelope checks of `validate_envelope` (research.rs:137-168), the parameter checks of
`validate_parameters` (research.rs:235-270) and the shear-rheometer material mapping of
`material` (research.rs:274-305).  Error texts follow the reference so callers that match
on them keep working.
"""

from __future__ import annotations

import math
from typing import Any

from . import _abi

MAX_PARTICLES = 100_000  # research.rs:21
MAX_NODES = 1_000_000  # research.rs:22
MAX_FRAME_POINTS = 2_000_000.0  # research.rs:23

_PARAMETER_KEYS = {
    "fixture", "grid_spacing_m", "domain_m", "material", "density_kg_m3", "young_modulus_pa",
    "poisson_ratio", "yield_stress_pa", "consistency_pa_s_n", "flow_index", "initial_size_m",
    "initial_velocity_m_s",
}
_REQUEST_KEYS = {
    "schema_version", "mode", "seed", "duration_s", "dt_s", "record_interval_s", "max_wall_time_s",
    "boxes", "materials", "events", "research",
}
_MATERIAL_KEYS = {
    "friction", "restitution", "normal_stiffness_n_m", "water_capacity_ratio", "uptake_rate_s",
    "breakdown_rate_s", "evaporation_rate_s",
}
_BOX_KEYS = {
    "id", "size_m", "origin_m", "slot_width_m", "slot_length_m", "slot_pitch_m", "drawer_depth_m",
    "pellet_count", "pellet_radius_m", "pellet_length_m", "pellet_density_kg_m3",
}


class SpecError(ValueError):
    """Invalid research request (maps to the reference's `Err(String)`)."""


def _finite_positive(value: float) -> bool:
    return isinstance(value, (int, float)) and math.isfinite(value) and value > 0.0


def _check_keys(obj: dict, allowed: set, what: str) -> None:
    if not isinstance(obj, dict):
        raise SpecError(f"{what} must be an object")
    unknown = set(obj) - allowed
    if unknown:
        raise SpecError(f"unknown field `{sorted(unknown)[0]}` in {what}")
    missing = allowed - set(obj)
    if missing:
        raise SpecError(f"missing field `{sorted(missing)[0]}` in {what}")


def _validate_materials(m: dict) -> None:
    """household/request.rs:195-203."""
    if not (math.isfinite(m["friction"]) and m["friction"] >= 0.0):
        raise SpecError("materials.friction must be non-negative")
    if not (math.isfinite(m["restitution"]) and 0.0 <= m["restitution"] <= 1.0):
        raise SpecError("materials.restitution must lie in [0, 1]")
    for key in ("normal_stiffness_n_m", "water_capacity_ratio"):
        if not _finite_positive(m[key]):
            raise SpecError(f"materials.{key} must be positive")
    for key in ("uptake_rate_s", "breakdown_rate_s", "evaporation_rate_s"):
        if not (math.isfinite(m[key]) and m[key] >= 0.0):
            raise SpecError(f"materials.{key} must be non-negative")


def _validate_box(b: dict) -> None:
    """household/request.rs:223-260 (geometry checks used by research boxes)."""
    tag = f"boxes['{b['id']}']"
    if not b["id"]:
        raise SpecError("box `id` must not be empty")
    for v in b["size_m"]:
        if not _finite_positive(v):
            raise SpecError(f"{tag}.size_m must be positive")
    for key in ("slot_width_m", "slot_length_m", "slot_pitch_m", "drawer_depth_m", "pellet_radius_m",
                "pellet_length_m", "pellet_density_kg_m3"):
        if not _finite_positive(b[key]):
            raise SpecError(f"{tag}.{key} must be positive")
    if b["slot_width_m"] >= b["slot_pitch_m"]:
        raise SpecError(f"{tag}: `slot_width_m` must be smaller than `slot_pitch_m`")
    if b["slot_pitch_m"] > b["size_m"][1]:
        raise SpecError(f"{tag}: `slot_pitch_m` exceeds the box `size_m.y`")
    if b["slot_length_m"] + 2.0 * b["slot_width_m"] > b["size_m"][0]:
        raise SpecError(f"{tag}: one slot plus its bars does not fit `size_m.x`")
    bounding = max(b["pellet_length_m"], 2.0 * b["pellet_radius_m"])
    if bounding >= min(b["size_m"][0], b["size_m"][1]) or bounding >= b["size_m"][2]:
        raise SpecError(f"{tag}: a pellet does not fit inside the box")


def validate_envelope(req: dict) -> None:
    """research.rs:137-168."""
    _check_keys(req, _REQUEST_KEYS, "request")
    if req["schema_version"] != 1 or req["mode"] != "research" or req["events"]:
        raise SpecError("research requires schema_version=1, mode=research and no household events")
    for key in ("duration_s", "dt_s", "record_interval_s", "max_wall_time_s"):
        if not _finite_positive(req[key]):
            raise SpecError("research times and budgets must be finite and positive")
    if req["dt_s"] > req["duration_s"] or req["max_wall_time_s"] > 3600.0:
        raise SpecError("research dt exceeds duration or budget exceeds 3600 seconds")
    if req["duration_s"] / req["record_interval_s"] > 10_000.0 or req["duration_s"] / req["dt_s"] > 10_000_000.0:
        raise SpecError("research recording or nominal-step resource cap exceeded")
    if len(req["boxes"]) > 1:
        raise SpecError("research fixtures support at most one box supplying pellet geometry")
    for b in req["boxes"]:
        _check_keys(b, _BOX_KEYS, "box")
        _validate_box(b)
    _check_keys(req["materials"], _MATERIAL_KEYS, "materials")
    _validate_materials(req["materials"])


def validate_parameters(p: dict) -> None:
    """research.rs:235-270."""
    positive = [p["grid_spacing_m"], p["density_kg_m3"], p["young_modulus_pa"], p["flow_index"]]
    if (any(not _finite_positive(v) for v in positive)
            or any(not _finite_positive(v) for v in list(p["domain_m"]) + list(p["initial_size_m"]))
            or any(not math.isfinite(v) for v in p["initial_velocity_m_s"])):
        raise SpecError("research geometry, density, stiffness and flow index must be finite and positive")
    nu = p["poisson_ratio"]
    if (not math.isfinite(nu) or not (0.0 <= nu < 0.5) or not math.isfinite(p["yield_stress_pa"])
            or p["yield_stress_pa"] < 0.0 or not math.isfinite(p["consistency_pa_s_n"])
            or p["consistency_pa_s_n"] < 0.0):
        raise SpecError("invalid Poisson ratio, yield stress or consistency")
    for extent, domain in zip(p["initial_size_m"], p["domain_m"]):
        ratio = extent / (0.5 * p["grid_spacing_m"])
        if extent > domain or not math.isfinite(ratio) or abs(ratio - round(ratio)) > 1e-6:
            raise SpecError("initial block must fit domain and span whole particle subcells")


def material_paste(density, young, nu, ys, k, n) -> _abi.Material:
    """constitutive.rs:146-167."""
    m = _abi.Material()
    mu = young / (2.0 * (1.0 + nu))
    lam = young * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    m.kind, m.density, m.shear_modulus, m.lame_lambda = _abi.LP_PASTE, density, mu, lam
    m.bulk_modulus = lam + 2.0 * mu / 3.0
    m.yield_stress, m.consistency, m.flow_index, m.tait_gamma = ys, k, n, 1.0
    return m


def material_paste_shear(density, young, nu, tys, ks, n) -> _abi.Material:
    """constitutive.rs:180-197: shear-rheometer (tau_y, K_s) to von Mises (sigma_y, K)."""
    return material_paste(density, young, nu, math.sqrt(3.0) * tys, 3.0 ** ((1.0 + n) / 2.0) * ks, n)


def material_liquid(density, young, nu, viscosity, tait_gamma: float = 1.0) -> _abi.Material:
    """constitutive.rs:211-223 (+ Tait exponent extension, 1 = reference)."""
    m = _abi.Material()
    m.kind, m.density = _abi.LP_LIQUID, density
    m.bulk_modulus = young / (3.0 * (1.0 - 2.0 * nu))
    m.consistency, m.flow_index, m.tait_gamma = viscosity, 1.0, tait_gamma
    return m


def wave_speed(m: _abi.Material) -> float:
    modulus = m.lame_lambda + 2.0 * m.shear_modulus if m.kind == _abi.LP_PASTE else m.bulk_modulus
    return math.sqrt(modulus / m.density)


def _material(p: dict) -> _abi.Material:
    """research.rs:274-305."""
    name = p["material"]
    if name == "paste":
        m = material_paste_shear(p["density_kg_m3"], p["young_modulus_pa"], p["poisson_ratio"],
                                 p["yield_stress_pa"], p["consistency_pa_s_n"], p["flow_index"])
    elif name == "water" and p["yield_stress_pa"] == 0.0 and abs(p["flow_index"] - 1.0) < 1e-12:
        m = material_liquid(p["density_kg_m3"], p["young_modulus_pa"], p["poisson_ratio"],
                            p["consistency_pa_s_n"])
    elif name == "water":
        raise SpecError("water requires zero yield stress and flow_index=1")
    elif name == "fines":
        raise SpecError("porous Drucker-Prager fines are not implemented")
    else:
        raise SpecError(f"unsupported research material '{name}'")
    ws = wave_speed(m)
    if not math.isfinite(ws) or ws <= 0.0:
        raise SpecError("derived material properties are nonfinite")
    return m


def particle_count(spec: _abi.FixtureSpec) -> int:
    """fixtures.rs:120-133."""
    sub = spec.grid_spacing / 2.0
    n = 1
    for a in range(3):
        n *= max(int(round_half_away(spec.initial_size[a] / sub)), 1)
    return n


def round_half_away(x: float) -> float:
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def base_spec(**kw: Any) -> _abi.FixtureSpec:
    """A zero-initialised spec (reference behaviour for every extension) with fields set."""
    s = _abi.FixtureSpec()
    s.cfl = 0.3
    s.min_dt = 1e-12
    s.gravity[:] = [0.0, 0.0, -9.81]
    s.max_particles = MAX_PARTICLES
    s.max_nodes = MAX_NODES
    for key, value in kw.items():
        if key in ("domain", "initial_size", "initial_velocity", "gravity", "face_friction", "face_sticky"):
            getattr(s, key)[:] = list(value)
        else:
            setattr(s, key, value)
    return s


def spec_from_request(req: dict, *, max_particles: int = MAX_PARTICLES,
                      max_nodes: int = MAX_NODES) -> _abi.FixtureSpec:
    """research.rs:171-232: wire request -> fixture spec (gravity -9.81 z, CFL 0.3, min_dt 1e-12)."""
    validate_envelope(req)
    p = req["research"]
    if p is None:
        raise SpecError("research parameters are required")
    _check_keys(p, _PARAMETER_KEYS, "research parameters")
    validate_parameters(p)
    fixture = _abi.FIXTURES.get(p["fixture"])
    if fixture is None:
        raise SpecError(f"unsupported research fixture '{p['fixture']}'")
    if fixture != _abi.LP_COUPLED_PATCH and req["boxes"]:
        raise SpecError("only coupled_patch accepts a pellet geometry box")
    mat = _material(p)
    mats = req["materials"]
    s = base_spec(
        fixture=fixture,
        grid_spacing=float(p["grid_spacing_m"]),
        domain=p["domain_m"],
        initial_size=p["initial_size_m"],
        initial_velocity=p["initial_velocity_m_s"],
        seed=int(req["seed"]),
        wall_friction=float(mats["friction"]),
        max_dt=float(req["dt_s"]),
        contact_stiffness=float(mats["normal_stiffness_n_m"]),
        contact_restitution=float(mats["restitution"]),
        contact_friction=float(mats["friction"]),
        max_particles=max_particles,
        max_nodes=max_nodes,
    )
    s.material = mat
    if req["boxes"]:
        b = req["boxes"][0]
        s.has_pellet = 1
        s.pellet_radius = float(b["pellet_radius_m"])
        s.pellet_length = float(b["pellet_length_m"])
        s.pellet_density = float(b["pellet_density_kg_m3"])
    count = particle_count(s)
    frames = math.ceil(req["duration_s"] / req["record_interval_s"]) + 1.0
    if count > max_particles:
        raise SpecError(f"fixture would allocate '{count}' particles, exceeding the cap of '{max_particles}'")
    if frames * float(min(count + 64, 2**32 - 1)) > MAX_FRAME_POINTS:
        raise SpecError("research frame-point resource cap exceeded; reduce recording frequency")
    return s
