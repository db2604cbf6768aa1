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
        if key in ("domain", "initial_size", "initial_velocity", "gravity", "face_friction", "face_sticky", "bed_lo",
                   "bed_hi"):
            getattr(s, key)[:] = list(value)
        else:
            setattr(s, key, value)
    return s


def grid_layout(domain, spacing: float, max_nodes: int) -> list:
    """`GridLayout::new` (grid.rs:35-86): cells per axis; errors as the reference words them."""
    if not (math.isfinite(spacing) and spacing > 0.0):
        raise SpecError(f"`grid_spacing_m` must be positive and finite, got '{spacing}'")
    cap = float(min(max(max_nodes - 3, 0), 2**32 - 1))
    cells = []
    for axis in range(3):
        extent = float(domain[axis])
        if not (math.isfinite(extent) and extent > 0.0):
            raise SpecError(f"`domain_m[{axis}]` must be positive and finite, got '{extent}'")
        ratio = extent / spacing
        rounded = float(round_half_away(ratio)) if math.isfinite(ratio) else ratio
        if not math.isfinite(ratio) or rounded > cap:
            raise SpecError("grid axis exceeds the node allocation cap")
        if abs(ratio - rounded) > 1e-6 * max(rounded, 1.0):
            raise SpecError(f"`domain_m[{axis}]`='{extent}' is not an integer multiple of `grid_spacing_m`='{spacing}'")
        if rounded < 2.0:
            raise SpecError(f"`domain_m[{axis}]` must span at least two cells")
        cells.append(int(rounded))
    total = (cells[0] + 3) * (cells[1] + 3) * (cells[2] + 3)
    if total > max_nodes:
        raise SpecError(f"grid would allocate '{total}' nodes, exceeding the cap of '{max_nodes}'; coarsen "
                        "`grid_spacing_m` or shrink `domain_m`")
    return cells


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
    grid_layout(s.domain, s.grid_spacing, max_nodes)
    count = particle_count(s)
    frames = math.ceil(req["duration_s"] / req["record_interval_s"]) + 1.0
    if count > max_particles:
        raise SpecError(f"fixture would allocate '{count}' particles, exceeding the cap of '{max_particles}'")
    if frames * float(min(count + 64, 2**32 - 1)) > MAX_FRAME_POINTS:
        raise SpecError("research frame-point resource cap exceeded; reduce recording frequency")
    return s


# ====================================================================== research::run
# Host-side restatement of the research driver (core/src/research.rs:73-134, 308-488) over the
# GPU simulation: the record loop, the conservative recordings, the JSON checkpoint and the
# checked restore.  The checkpoint `state` keeps the reference's `Snapshot` layout
# (research.rs:43-56): `ParticleSet` arrays (particles.rs:11-32) with nalgebra's JSON forms
# (vectors as [x, y, z], 3x3 matrices as 9 numbers in column-major order, quaternions as
# [i, j, k, w]), the `Ledger` fields (solver.rs:65-124) and the integration history.

SCHEMA_VERSION = 1
_LEDGER_VECTORS = ("initial_momentum", "gravity_impulse", "wall_impulse", "pellet_wall_impulse", "coupling_impulse",
                   "coupling_angular_impulse", "outflow_momentum")
_LEDGER_SCALARS = ("initial_mass", "outflow_mass", "initial_mechanical_energy", "wall_normal_projection_energy",
                   "wall_friction_dissipation", "wall_normal_traction_energy", "pellet_wall_work",
                   "coupling_grid_energy", "coupling_pellet_energy", "plastic_dissipation")
_SNAPSHOT_KEYS = {"particles", "pellet", "ledger", "step_count", "limited_steps", "rejected_steps", "dt_scale",
                  "min_dt_used", "max_dt_used", "next_record_index"}
_PARTICLE_KEYS = ("id", "position", "velocity", "affine", "deformation", "volume_ratio", "kirchhoff",
                  "plastic_strain", "mass", "volume0")
_PELLET_KEYS = ("radius", "length", "mass", "inertia_body", "position", "orientation", "velocity",
                "angular_momentum", "sphere_offsets")
_DIAGNOSTICS = [
    "Unvalidated numerical fixture; no measured surrogate or household calibration",
    "Single-phase paste mass is booked as waste; no mobile/bound-water split",
    "No porous fines, wet fragmentation, absorption, adhesion or response-table generation",
    "Dense padded grid with active-node updates; no sparse-block storage",
    "Grid-level coupling conserves impulses but can create kinetic energy for light bodies; coupled energy "
    "stability, leakage and convergence remain unverified",
    "Wall lattice completion is an approximate contact treatment; its normal transfer is booked as a signed grid "
    "kinetic-energy diagnostic, not physical wall work; energy closure remains open",
]


class RunError(ValueError):
    """A research run failed (the reference's `Err(String)` from `research::run`)."""


def _ledger_to_json(led: _abi.Ledger) -> dict:
    d = led.as_dict()
    return {name: d[name] for name, _ in _abi.Ledger._fields_}


def _ledger_from_json(d: dict) -> _abi.Ledger:
    if not isinstance(d, dict):
        raise RunError("invalid type: ledger must be an object")
    names = [name for name, _ in _abi.Ledger._fields_]
    unknown = set(d) - set(names)
    if unknown:
        raise RunError(f"unknown field `{sorted(unknown)[0]}` in ledger")
    led = _abi.Ledger()
    for name in names:
        if name not in d:
            raise RunError(f"missing field `{name}`")
        value = d[name]
        if name in _LEDGER_VECTORS:
            if not (isinstance(value, list) and len(value) == 3 and all(_is_number(v) for v in value)):
                raise RunError(f"invalid type: ledger `{name}` must be a 3-vector")
            getattr(led, name)[:] = [float(v) for v in value]
        else:
            if not _is_number(value):
                raise RunError(f"invalid type: ledger `{name}` must be a number")
            setattr(led, name, float(value))
    return led


def _is_number(v) -> bool:
    return isinstance(v, (int, float)) and not isinstance(v, bool)


def _mat_to_json(m) -> list:
    """Row-major (n, 3, 3) -> nalgebra's column-major 9-number form per matrix."""
    import numpy as np

    return np.ascontiguousarray(np.transpose(m, (0, 2, 1))).reshape(len(m), 9).tolist()


def _mat_from_json(rows, n: int, name: str):
    import numpy as np

    a = _float_array(rows, (n, 9), name)
    return np.ascontiguousarray(a.reshape(n, 3, 3).transpose(0, 2, 1))


def _float_array(rows, shape, name: str):
    import numpy as np

    try:
        a = np.array(rows, dtype=np.float64)
    except (TypeError, ValueError) as e:
        raise RunError(f"invalid type: particle array `{name}`: {e}") from e
    if a.shape != tuple(shape):
        if a.ndim >= 1 and a.shape[0] != shape[0]:
            raise RunError(f"particle array `{name}` has length '{a.shape[0]}', expected '{shape[0]}'")
        raise RunError(f"invalid type: particle array `{name}` has shape {a.shape}")
    return a


def particles_to_json(p: dict) -> dict:
    """Exported FP64 particle arrays -> the `ParticleSet` JSON object."""
    return {
        "id": [int(v) for v in p["id"]],
        "position": p["position"].tolist(),
        "velocity": p["velocity"].tolist(),
        "affine": _mat_to_json(p["affine"]),
        "deformation": _mat_to_json(p["deformation"]),
        "volume_ratio": p["volume_ratio"].tolist(),
        "kirchhoff": _mat_to_json(p["kirchhoff"]),
        "plastic_strain": p["plastic_strain"].tolist(),
        "mass": p["mass"].tolist(),
        "volume0": p["volume0"].tolist(),
    }


def particles_from_json(d: dict) -> dict:
    """`ParticleSet` JSON -> FP64 arrays for the import; `ParticleSet::validate`
    (particles.rs:159-211) checks lengths, unique ids and per-particle invariants."""
    import numpy as np

    if not isinstance(d, dict):
        raise RunError("invalid type: particles must be an object")
    unknown = set(d) - set(_PARTICLE_KEYS)
    if unknown:
        raise RunError(f"unknown field `{sorted(unknown)[0]}` in particles")
    for key in _PARTICLE_KEYS:
        if key not in d or not isinstance(d[key], list):
            raise RunError(f"missing field `{key}`")
    ids = d["id"]
    if not all(isinstance(v, int) and not isinstance(v, bool) and 0 <= v < 2**32 for v in ids):
        raise RunError("invalid type: particle ids must be u32")
    n = len(ids)
    for key in _PARTICLE_KEYS[1:]:
        if len(d[key]) != n:
            raise RunError(f"particle array `{key}` has length '{len(d[key])}', expected '{n}'")
    out = {
        "id": np.array(ids, dtype=np.uint32),
        "position": _float_array(d["position"], (n, 3), "position"),
        "velocity": _float_array(d["velocity"], (n, 3), "velocity"),
        "affine": _mat_from_json(d["affine"], n, "affine"),
        "deformation": _mat_from_json(d["deformation"], n, "deformation"),
        "volume_ratio": _float_array(d["volume_ratio"], (n,), "volume_ratio"),
        "kirchhoff": _mat_from_json(d["kirchhoff"], n, "kirchhoff"),
        "plastic_strain": _float_array(d["plastic_strain"], (n,), "plastic_strain"),
        "mass": _float_array(d["mass"], (n,), "mass"),
        "volume0": _float_array(d["volume0"], (n,), "volume0"),
    }
    if len(np.unique(out["id"])) != n:
        raise RunError("particle ids are not unique")
    for i in range(n):
        finite = (np.isfinite(out["position"][i]).all() and np.isfinite(out["velocity"][i]).all()
                  and np.isfinite(out["affine"][i]).all() and np.isfinite(out["deformation"][i]).all()
                  and np.isfinite(out["kirchhoff"][i]).all() and np.isfinite(out["volume_ratio"][i])
                  and np.isfinite(out["plastic_strain"][i]) and np.isfinite(out["mass"][i])
                  and np.isfinite(out["volume0"][i]))
        if not finite:
            raise RunError(f"particle id '{ids[i]}' has non-finite state")
        if out["mass"][i] <= 0.0 or out["volume0"][i] <= 0.0:
            raise RunError(f"particle id '{ids[i]}' has non-positive mass or volume")
        if out["volume_ratio"][i] <= 0.0 or out["plastic_strain"][i] < 0.0:
            raise RunError(f"particle id '{ids[i]}' has invalid ratio/plastic state")
    return out


def pellet_to_json(p: _abi.Pellet | None):
    if p is None:
        return None
    return {
        "radius": p.radius, "length": p.length, "mass": p.mass,
        "inertia_body": list(p.inertia_body), "position": list(p.position),
        "orientation": list(p.orientation), "velocity": list(p.velocity),
        "angular_momentum": list(p.angular_momentum),
        "sphere_offsets": [p.sphere_offsets[i] for i in range(p.sphere_count)],
    }


def pellet_from_json(d) -> _abi.Pellet:
    if not isinstance(d, dict) or set(d) != set(_PELLET_KEYS):
        raise RunError("invalid type: pellet must carry exactly the `Pellet` fields")
    p = _abi.Pellet()
    try:
        p.radius, p.length, p.mass = float(d["radius"]), float(d["length"]), float(d["mass"])
        for key, size in (("inertia_body", 3), ("position", 3), ("orientation", 4), ("velocity", 3),
                          ("angular_momentum", 3)):
            if len(d[key]) != size:
                raise RunError(f"invalid type: pellet `{key}` must have {size} numbers")
            getattr(p, key)[:] = [float(v) for v in d[key]]
        offsets = [float(v) for v in d["sphere_offsets"]]
    except (TypeError, ValueError) as e:
        raise RunError(f"invalid type: pellet: {e}") from e
    if not 1 <= len(offsets) <= len(p.sphere_offsets):
        raise RunError("pellet proxy exceeds the sphere allocation cap")
    p.sphere_count = len(offsets)
    p.sphere_offsets[: len(offsets)] = offsets
    return p


def _pellet_is_finite(p: _abi.Pellet) -> bool:
    vals = list(p.position) + list(p.velocity) + list(p.angular_momentum) + list(p.orientation)
    return all(math.isfinite(v) for v in vals)


def _sphere_centers(p: _abi.Pellet) -> list:
    """`Pellet::sphere_centers` (rigid.rs:202-208): position + R(q) x_hat * offset."""
    i, j, k, w = p.orientation
    axis = (1.0 - 2.0 * (j * j + k * k), 2.0 * (i * j + w * k), 2.0 * (i * k - w * j))
    return [[p.position[a] + axis[a] * p.sphere_offsets[s] for a in range(3)] for s in range(p.sphere_count)]


def snapshot(sim, next_record_index: int) -> dict:
    """research.rs:308-322."""
    c = sim.counters
    return {
        "particles": particles_to_json(sim.particles()),
        "pellet": pellet_to_json(sim.pellet()),
        "ledger": _ledger_to_json(sim.ledger),
        "step_count": int(c.step_count),
        "limited_steps": int(c.limited_steps),
        "rejected_steps": int(c.rejected_steps),
        "dt_scale": c.dt_scale,
        "min_dt_used": c.min_dt_used if math.isfinite(c.min_dt_used) else None,
        "max_dt_used": c.max_dt_used,
        "next_record_index": int(next_record_index),
    }


def grid_nodes(spec: _abi.FixtureSpec) -> list:
    """Padded node counts per axis (grid.rs:35-86): cells = round(domain / dx), nodes = cells + 3."""
    return [int(round(spec.domain[a] / spec.grid_spacing)) + 3 for a in range(3)]


def validate_state(sim, spec: _abi.FixtureSpec, particles: dict | None = None) -> None:
    """`Simulation::validate` (solver.rs:1106-1139) and `Ledger::validate` (solver.rs:182-244)."""
    import numpy as np

    p = particles if particles is not None else sim.particles()
    led = sim.ledger
    for name in _LEDGER_SCALARS:
        v = getattr(led, name)
        if not math.isfinite(v):
            raise RunError(f"invalid solver state: ledger `{name}` is nonfinite: '{v}'")
    for name in _LEDGER_VECTORS:
        v = list(getattr(led, name))
        if not all(math.isfinite(x) for x in v):
            raise RunError(f"invalid solver state: ledger `{name}` is nonfinite: '{v}'")
    for name in ("initial_mass", "outflow_mass", "plastic_dissipation", "wall_friction_dissipation"):
        if getattr(led, name) < 0.0:
            raise RunError(f"invalid solver state: ledger `{name}` must be non-negative, got '{getattr(led, name)}'")
    if led.wall_normal_projection_energy > 0.0:
        raise RunError("invalid solver state: ledger `wall_normal_projection_energy` must be non-positive, got "
                       f"'{led.wall_normal_projection_energy}'")
    c = sim.counters
    if not math.isfinite(c.time) or c.time < 0.0:
        raise RunError(f"invalid solver state: time '{c.time}' invalid")
    if not (math.isfinite(c.dt_scale) and 0.0 < c.dt_scale <= 1.0):
        raise RunError(f"invalid solver state: dt_scale '{c.dt_scale}' invalid")
    pel = sim.pellet()
    if pel is not None and not _pellet_is_finite(pel):
        raise RunError("invalid solver state: pellet state non-finite")
    # grid.rs:151-170: the full stencil must lie inside the padded grid
    nodes = np.array(grid_nodes(spec), dtype=np.float64)
    base = np.floor(p["position"] / spec.grid_spacing - 0.5) + 1.0
    bad = ~np.isfinite(base).all(axis=1) | (base < 0.0).any(axis=1) | (base + 2.0 >= nodes).any(axis=1)
    if bad.any():
        i = int(np.argmax(bad))
        raise RunError(f"invalid solver state: particle id '{int(p['id'][i])}' lies outside the grid")


def check_closed_state(sim, spec: _abi.FixtureSpec, particles: dict | None = None) -> None:
    """research.rs:466-482."""
    validate_state(sim, spec, particles)
    led = sim.ledger
    if not math.isfinite(led.outflow_mass) or abs(led.outflow_mass) > 0.0:
        raise RunError(f"closed research fixture leaked '{led.outflow_mass}' kg beyond the padded grid")
    residual = sim.mass_residual()
    if not math.isfinite(residual) or abs(residual) > max(1e-6 * led.initial_mass, 1e-12):
        raise RunError(f"research mass conservation failed: '{residual}' kg")


def record(sim, spec: _abi.FixtureSpec, frames: list, metrics: list, particles: dict | None = None) -> None:
    """research.rs:484-518: material points plus pellet sphere proxies, and the two compartments."""
    p = particles if particles is not None else sim.particles()
    water = spec.material.kind == _abi.LP_LIQUID
    label = "water" if water else "waste"
    positions = p["position"].tolist()
    radii = [spec.grid_spacing / 4.0] * len(positions)
    materials = [label] * len(positions)
    pel = sim.pellet()
    if pel is not None:
        for point in _sphere_centers(pel):
            positions.append(point)
            radii.append(pel.radius)
            materials.append("wood")
    t = sim.time
    frames.append({"time_s": t, "positions_m": positions, "radii_m": radii, "materials": materials,
                   "box_ids": ["research"] * len(positions)})
    total = float(sum(float(m) for m in p["mass"]))
    for compartment, mass in (("domain", total), ("outflow", sim.ledger.outflow_mass)):
        metrics.append({
            "time_s": t, "compartment": compartment,
            "wood_kg": (pel.mass if pel is not None else 0.0) if compartment == "domain" else 0.0,
            "water_kg": mass if water else 0.0,
            "waste_kg": 0.0 if water else mass,
        })


def _contains_null(value) -> bool:
    if value is None:
        return True
    if isinstance(value, list):
        return any(_contains_null(v) for v in value)
    if isinstance(value, dict):
        return any(_contains_null(v) for v in value.values())
    return False


def _validate_snapshot(state: dict, parts: dict, time_s: float, req: dict, initial_ledger: _abi.Ledger,
                       initial_pellet: _abi.Pellet | None) -> None:
    """research.rs:380-447."""
    import numpy as np

    def num(key):
        v = state.get(key)
        if not _is_number(v):
            raise RunError(f"invalid type: checkpoint `{key}` must be a number")
        return v

    dt_scale, max_dt_used = num("dt_scale"), num("max_dt_used")
    step_count, limited, rejected, nri = (num("step_count"), num("limited_steps"), num("rejected_steps"),
                                          num("next_record_index"))
    for key, v in (("step_count", step_count), ("limited_steps", limited), ("rejected_steps", rejected)):
        if not isinstance(v, int) or v < 0 or v >= 2**64:
            raise RunError(f"invalid type: checkpoint `{key}` must be a u64")
    if not isinstance(nri, int) or nri < 0 or nri >= 2**32:
        raise RunError("invalid type: checkpoint `next_record_index` must be a u32")
    min_dt_used = state.get("min_dt_used")
    if min_dt_used is not None and not _is_number(min_dt_used):
        raise RunError("invalid type: checkpoint `min_dt_used` must be a number or null")
    if (not math.isfinite(dt_scale) or not (0.0 <= dt_scale <= 1.0) or dt_scale == 0.0
            or not math.isfinite(max_dt_used) or max_dt_used < 0.0
            or (min_dt_used is not None and (not math.isfinite(min_dt_used) or min_dt_used <= 0.0
                                             or min_dt_used > max_dt_used))
            or nri == 0 or nri > 10_002 or step_count > 1_000_000_000_000 or limited > step_count
            or rejected > 1_000_000_000_000):
        raise RunError("invalid research checkpoint integration history")
    next_time = float(nri) * req["record_interval_s"]
    previous = float(nri - 1) * req["record_interval_s"]
    if time_s < req["duration_s"] and (time_s < previous - 1e-12 or time_s >= next_time):
        raise RunError("research checkpoint recording schedule is inconsistent")
    det = np.linalg.det(parts["deformation"]) if len(parts["deformation"]) else np.zeros(0)
    if (~np.isfinite(det) | (det <= 0.0)).any():
        raise RunError("research checkpoint contains inverted deformation")
    ledger_json = state["ledger"]
    if _contains_null(ledger_json):
        raise RunError("research checkpoint initial inventory or ledger is inconsistent")
    led = _ledger_from_json(ledger_json)
    init_mom = list(initial_ledger.initial_momentum)
    mom = list(led.initial_momentum)
    if (led.outflow_mass < 0.0 or abs(led.initial_mass - initial_ledger.initial_mass) > 1e-12
            or _bits(led.initial_mechanical_energy) != _bits(initial_ledger.initial_mechanical_energy)
            or math.sqrt(sum((a - b) ** 2 for a, b in zip(mom, init_mom))) > 1e-12):
        raise RunError("research checkpoint initial inventory or ledger is inconsistent")
    pel = state.get("pellet")
    if pel is None and initial_pellet is None:
        return
    if pel is None or initial_pellet is None:
        raise RunError("research checkpoint pellet geometry is incompatible")
    p = pellet_from_json(pel)
    q = list(p.orientation)
    same_offsets = (p.sphere_count == initial_pellet.sphere_count
                    and all(p.sphere_offsets[i] == initial_pellet.sphere_offsets[i] for i in range(p.sphere_count)))
    if not (_pellet_is_finite(p) and _bits(p.mass) == _bits(initial_pellet.mass)
            and _bits(p.radius) == _bits(initial_pellet.radius) and _bits(p.length) == _bits(initial_pellet.length)
            and list(p.inertia_body) == list(initial_pellet.inertia_body) and same_offsets
            and abs(math.sqrt(sum(v * v for v in q)) - 1.0) < 1e-10):
        raise RunError("research checkpoint pellet geometry is incompatible")


def _bits(x: float) -> bytes:
    import struct

    return struct.pack("<d", float(x))


def restore(sim, spec: _abi.FixtureSpec, req: dict, value) -> int:
    """research.rs:325-377: checked restore of a checkpoint into the freshly built simulation."""
    if not isinstance(value, dict):
        raise RunError("invalid type: checkpoint must be an object")
    allowed = {"schema_version", "mode", "request", "time_s", "state"}
    unknown = set(value) - allowed
    if unknown:
        raise RunError(f"unknown field `{sorted(unknown)[0]}`")
    missing = allowed - set(value)
    if missing:
        raise RunError(f"missing field `{sorted(missing)[0]}`")
    time_s = value["time_s"]
    if (value["schema_version"] != 1 or value["mode"] != "research" or not _is_number(time_s)
            or not math.isfinite(time_s) or time_s < 0.0 or time_s > req["duration_s"]):
        raise RunError("invalid research checkpoint version, mode or time")
    original = value["request"]
    if not isinstance(original, dict):
        raise RunError("invalid type: checkpoint request must be an object")
    original = dict(original)
    original["max_wall_time_s"] = req["max_wall_time_s"]
    if original != req:
        raise RunError("research checkpoint request differs from resume request")
    state = value["state"]
    if not isinstance(state, dict):
        raise RunError("invalid type: checkpoint state must be an object")
    unknown = set(state) - _SNAPSHOT_KEYS
    if unknown:
        raise RunError(f"unknown field `{sorted(unknown)[0]}`")
    missing = _SNAPSHOT_KEYS - set(state) - {"pellet", "min_dt_used"}
    if missing:
        raise RunError(f"missing field `{sorted(missing)[0]}`")
    parts = particles_from_json(state["particles"])
    count = particle_count(spec)
    if len(parts["id"]) > count or (len(parts["id"]) and int(parts["id"].max()) >= count):
        raise RunError("research checkpoint particle identities are incompatible")
    _validate_snapshot(state, parts, float(time_s), req, sim.ledger, sim.pellet())
    sim.set_particles(parts)
    if state.get("pellet") is not None:
        sim.set_pellet(pellet_from_json(state["pellet"]))
    sim.set_ledger(_ledger_from_json(state["ledger"]))
    c = sim.counters
    c.time = float(time_s)
    c.step_count = int(state["step_count"])
    c.limited_steps = int(state["limited_steps"])
    c.rejected_steps = int(state["rejected_steps"])
    c.dt_scale = float(state["dt_scale"])
    c.min_dt_used = float(state["min_dt_used"]) if state.get("min_dt_used") is not None else math.inf
    c.max_dt_used = float(state["max_dt_used"])
    sim.set_counters(c)
    check_closed_state(sim, spec)
    return int(state["next_record_index"])


def run(req: dict, resume=None) -> dict:
    """`research::run` (research.rs:73-134) on the GPU simulation.

    Returns the output object; raises RunError (or SpecError) where the reference returns
    `Err(String)`.  Budget expiry returns status "budget_exhausted" with a resumable checkpoint."""
    import time as _time

    from ._lib import LPError
    from .sim import Simulation

    started = _time.monotonic()
    spec = spec_from_request(req)
    try:
        sim = Simulation(spec)
    except LPError as e:
        raise RunError(e.message) from e
    with sim:
        next_record = 1
        frames: list = []
        metrics: list = []
        if resume is not None:
            next_record = restore(sim, spec, req, resume)
        else:
            record(sim, spec, frames, metrics)
        duration = float(req["duration_s"])
        interval = float(req["record_interval_s"])
        budget = float(req["max_wall_time_s"])
        completed = sim.time >= duration
        while not completed:
            target = min(float(next_record) * interval, duration)
            try:
                reached = sim.advance_while(target, lambda: _time.monotonic() - started < budget)
            except LPError as e:
                raise RunError(e.message) from e
            if not reached:
                break
            parts = sim.particles()
            check_closed_state(sim, spec, parts)
            record(sim, spec, frames, metrics, parts)
            next_record += 1
            completed = sim.time >= duration
        check_closed_state(sim, spec)
        checkpoint = {"schema_version": SCHEMA_VERSION, "mode": "research", "request": req, "time_s": sim.time,
                      "state": snapshot(sim, next_record)}
        observables = sim.observables()
        if any(not math.isfinite(v) for v in observables.values()):
            raise RunError("research observables became nonfinite")
        output = {
            "schema_version": SCHEMA_VERSION, "mode": "research",
            "status": "completed" if completed else "budget_exhausted",
            "fidelity": "research_unvalidated", "time_s": sim.time,
            "frames": frames, "metrics": metrics, "observables": observables,
            "checkpoint": checkpoint, "diagnostics": list(_DIAGNOSTICS),
        }
        if _time.monotonic() - started >= budget:
            output["status"] = "budget_exhausted"
        return output


def run_batch(reqs: list, clock=None) -> list:
    """`research::run` for several requests in one batched launch (extension).

    The requests must share `duration_s`, `record_interval_s` and the fixture kind.  Entry k of
    the result is what `run(reqs[k])` returns for that request alone -- batched instances step
    exactly like single simulations -- or the RunError it would raise.  The wall budget is the
    smallest `max_wall_time_s` of the group.  Invalid requests raise SpecError before anything
    runs."""
    import time as _time

    from ._lib import LPError
    from .sim import Batch

    clock = clock or _time.monotonic
    started = clock()
    if not reqs:
        return []
    specs = [spec_from_request(r) for r in reqs]
    duration = float(reqs[0]["duration_s"])
    interval = float(reqs[0]["record_interval_s"])
    if any(float(r["duration_s"]) != duration or float(r["record_interval_s"]) != interval for r in reqs):
        raise SpecError("batched requests must share `duration_s` and `record_interval_s`")
    budget = min(float(r["max_wall_time_s"]) for r in reqs)
    try:
        batch = Batch(specs)
    except LPError as e:
        raise RunError(e.message) from e
    n = len(reqs)
    members = [batch.member(i) for i in range(n)]
    frames: list = [[] for _ in range(n)]
    metrics: list = [[] for _ in range(n)]
    errors: list = [None] * n

    def alive() -> list:
        return [i for i in range(n) if errors[i] is None]

    try:
        for i in range(n):
            record(members[i], specs[i], frames[i], metrics[i])
        next_record = 1
        completed = batch.counters(0).time >= duration
        while not completed and alive():
            target = min(float(next_record) * interval, duration)
            try:
                res = batch.advance_while(target, lambda: clock() - started < budget)
            except LPError as e:
                raise RunError(e.message) from e
            if res == "budget":
                break
            for i in alive():
                state, why = batch.state(i)
                if state in ("min_step", "outflow"):
                    errors[i] = RunError(why)
                    continue
                try:
                    parts = members[i].particles()
                    check_closed_state(members[i], specs[i], parts)
                    record(members[i], specs[i], frames[i], metrics[i], parts)
                except RunError as e:
                    errors[i] = e
            next_record += 1
            live = alive()
            completed = bool(live) and members[live[0]].time >= duration
        out: list = []
        for i in range(n):
            if errors[i] is not None:
                out.append(errors[i])
                continue
            m = members[i]
            try:
                check_closed_state(m, specs[i])
                checkpoint = {"schema_version": SCHEMA_VERSION, "mode": "research", "request": reqs[i],
                              "time_s": m.time, "state": snapshot(m, next_record)}
                observables = m.observables()
                if any(not math.isfinite(v) for v in observables.values()):
                    raise RunError("research observables became nonfinite")
            except RunError as e:
                out.append(e)
                continue
            done = m.time >= duration
            output = {
                "schema_version": SCHEMA_VERSION, "mode": "research",
                "status": "completed" if done else "budget_exhausted",
                "fidelity": "research_unvalidated", "time_s": m.time,
                "frames": frames[i], "metrics": metrics[i], "observables": observables,
                "checkpoint": checkpoint, "diagnostics": list(_DIAGNOSTICS),
            }
            if clock() - started >= budget:
                output["status"] = "budget_exhausted"
            out.append(output)
        return out
    finally:
        batch.close()
