"""ctypes mirrors of the POD structs declared in include/lp_mpm.h.

The layouts must match the C header field for field; `tests/test_abi.py` checks the sizes
against the compiled library.
"""

from __future__ import annotations

import ctypes as C

LP_OK, LP_INVALID, LP_MIN_STEP, LP_BUDGET, LP_DEVICE, LP_UNSUPPORTED = range(6)
STATUS_NAMES = {
    LP_OK: "ok",
    LP_INVALID: "invalid input",
    LP_MIN_STEP: "minimum step reached",
    LP_BUDGET: "budget stop",
    LP_DEVICE: "device error",
    LP_UNSUPPORTED: "unsupported",
}
LP_SLUMP, LP_HYDROSTATIC, LP_DAM_BREAK, LP_COUPLED_PATCH = range(4)
LP_BED_HERTZ_MINDLIN, LP_BED_LINEAR = range(2)
# warm-start logit table: node j at la8 = MLP_TAB_LO + j * MLP_TAB_H (LP_MLP_TAB_* of lp_mpm.h)
MLP_TAB_N, MLP_TAB_LO, MLP_TAB_H = 2049, -10.75, 11.0 / 1024.0
LP_PASTE, LP_LIQUID = range(2)
FIXTURES = {"slump": LP_SLUMP, "hydrostatic": LP_HYDROSTATIC, "dam_break": LP_DAM_BREAK,
            "coupled_patch": LP_COUPLED_PATCH}


class Material(C.Structure):
    """Mirror of `Material` (core/src/mpm/constitutive.rs:111-131) plus the Tait exponent."""

    _fields_ = [
        ("kind", C.c_int32),
        ("_pad", C.c_int32),
        ("density", C.c_double),
        ("shear_modulus", C.c_double),
        ("lame_lambda", C.c_double),
        ("bulk_modulus", C.c_double),
        ("yield_stress", C.c_double),
        ("consistency", C.c_double),
        ("flow_index", C.c_double),
        ("tait_gamma", C.c_double),
    ]


class FixtureSpec(C.Structure):
    """Mirror of `FixtureSpec` + `SolverConfig` (fixtures.rs:94-115, solver.rs:48-62)."""

    _fields_ = [
        ("fixture", C.c_int32),
        ("has_pellet", C.c_int32),
        ("material", Material),
        ("grid_spacing", C.c_double),
        ("domain", C.c_double * 3),
        ("initial_size", C.c_double * 3),
        ("initial_velocity", C.c_double * 3),
        ("seed", C.c_uint64),
        ("pellet_radius", C.c_double),
        ("pellet_length", C.c_double),
        ("pellet_density", C.c_double),
        ("gravity", C.c_double * 3),
        ("wall_friction", C.c_double),
        ("cfl", C.c_double),
        ("max_dt", C.c_double),
        ("min_dt", C.c_double),
        ("contact_stiffness", C.c_double),
        ("contact_restitution", C.c_double),
        ("contact_friction", C.c_double),
        ("max_particles", C.c_uint64),
        ("max_nodes", C.c_uint64),
        ("face_mode_enabled", C.c_int32),
        ("face_sticky", C.c_int32 * 6),
        ("face_friction", C.c_double * 6),
        ("newton_tolerance", C.c_double),
        ("yield_random", C.c_int32),
        ("_pad2", C.c_int32),
        ("yield_min", C.c_double),
        ("yield_max", C.c_double),
        ("bed_count", C.c_int32),
        ("_pad3", C.c_int32),
        ("bed_seed", C.c_uint64),
        ("bed_lo", C.c_double * 3),
        ("bed_hi", C.c_double * 3),
        ("hm_young", C.c_double),
        ("hm_poisson", C.c_double),
        ("hm_friction", C.c_double),
        ("hm_restitution", C.c_double),
        ("bed_law", C.c_int32),
        ("_pad4", C.c_int32),
        ("dem_stiffness", C.c_double),
        ("dem_rolling", C.c_double),
    ]


class Ledger(C.Structure):
    """Mirror of `Ledger` (core/src/mpm/solver.rs:65-124)."""

    _fields_ = [
        ("initial_mass", C.c_double),
        ("outflow_mass", C.c_double),
        ("initial_momentum", C.c_double * 3),
        ("initial_mechanical_energy", C.c_double),
        ("gravity_impulse", C.c_double * 3),
        ("wall_impulse", C.c_double * 3),
        ("pellet_wall_impulse", C.c_double * 3),
        ("coupling_impulse", C.c_double * 3),
        ("coupling_angular_impulse", C.c_double * 3),
        ("wall_normal_projection_energy", C.c_double),
        ("wall_friction_dissipation", C.c_double),
        ("wall_normal_traction_energy", C.c_double),
        ("pellet_wall_work", C.c_double),
        ("coupling_grid_energy", C.c_double),
        ("coupling_pellet_energy", C.c_double),
        ("plastic_dissipation", C.c_double),
        ("outflow_momentum", C.c_double * 3),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            value = getattr(self, name)
            out[name] = list(value) if hasattr(value, "__len__") else float(value)
        return out


class Counters(C.Structure):
    """Simulation counters (solver.rs:332-352)."""

    _fields_ = [
        ("time", C.c_double),
        ("step_count", C.c_uint64),
        ("limited_steps", C.c_uint64),
        ("rejected_steps", C.c_uint64),
        ("dt_scale", C.c_double),
        ("min_dt_used", C.c_double),
        ("max_dt_used", C.c_double),
        ("particle_count", C.c_uint64),
        ("newton_iterations", C.c_uint64),
        ("yielded_particles", C.c_uint64),
    ]


class Particles(C.Structure):
    """Host view of `ParticleSet` (core/src/mpm/particles.rs:11-32)."""

    _fields_ = [
        ("count", C.c_uint64),
        ("id", C.POINTER(C.c_uint32)),
        ("position", C.POINTER(C.c_double)),
        ("velocity", C.POINTER(C.c_double)),
        ("affine", C.POINTER(C.c_double)),
        ("deformation", C.POINTER(C.c_double)),
        ("volume_ratio", C.POINTER(C.c_double)),
        ("kirchhoff", C.POINTER(C.c_double)),
        ("plastic_strain", C.POINTER(C.c_double)),
        ("mass", C.POINTER(C.c_double)),
        ("volume0", C.POINTER(C.c_double)),
        ("yield_stress", C.POINTER(C.c_double)),
    ]


class EnergyAudit(C.Structure):
    """Mirror of `lp_energy_audit` (audit.rs:254-271 EnergyAudit)."""

    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("before", C.c_double * 5),
        ("after", C.c_double * 5),
        ("stages", C.c_double * 8),
        ("increments", C.c_double * 7),
        ("terms", C.c_double * 12),
        ("coupled", C.c_int32),
        ("_pad", C.c_int32),
    ]

    STATE = ("translation", "affine", "elastic", "potential", "pellet")
    STAGES = ("grid_transport", "grid_after_stress", "grid_after_traction", "grid_after_gravity",
              "grid_after_walls", "grid_after_coupling", "pellet_after_coupling", "plastic_dissipation")
    INCREMENTS = ("plastic_dissipation", "wall_friction_dissipation", "wall_normal_projection_energy",
                  "wall_normal_traction_energy", "coupling_grid_energy", "coupling_pellet_energy", "pellet_wall_work")
    TERMS = ("p2g_transfer_loss", "g2p_transfer_loss", "stress_storage_plastic_mismatch",
             "uncoupled_gravity_potential_mismatch", "coupled_grid_gravity_total_potential_change",
             "pellet_integrator_combined_change", "traction_change", "walls_change", "coupling_change",
             "augmented_energy_change", "telescoping_sum", "telescoping_error")

    def as_dict(self) -> dict:
        """The reference's `EnergyAudit` JSON shape; the optional gravity term of the other
        scope is None, like the reference's `Option`."""
        terms = {}
        for k, name in enumerate(self.TERMS):
            v = float(self.terms[k])
            optional = (k == 3 and self.coupled) or (k == 4 and not self.coupled)
            terms[name] = None if optional else v
        return {
            "time": self.time, "dt": self.dt,
            "before": dict(zip(self.STATE, map(float, self.before))),
            "after": dict(zip(self.STATE, map(float, self.after))),
            "stages": dict(zip(self.STAGES, map(float, self.stages))),
            "increments": dict(zip(self.INCREMENTS, map(float, self.increments))),
            "terms": terms,
        }


class Pellet(C.Structure):
    """Mirror of `Pellet` (core/src/mpm/rigid.rs:30-49)."""

    _fields_ = [
        ("radius", C.c_double),
        ("length", C.c_double),
        ("mass", C.c_double),
        ("inertia_body", C.c_double * 3),
        ("position", C.c_double * 3),
        ("orientation", C.c_double * 4),
        ("velocity", C.c_double * 3),
        ("angular_momentum", C.c_double * 3),
        ("sphere_count", C.c_int32),
        ("_pad", C.c_int32),
        ("sphere_offsets", C.c_double * 64),
    ]


class LaunchShape(C.Structure):
    """Mirror of `lp_launch_shape`: launch shape of the persistent tile kernels (no reference
    counterpart)."""

    _fields_ = [
        ("g2p_variant", C.c_int32),
        ("g2p_per_sm", C.c_int32),
        ("p2g_variant", C.c_int32),
        ("p2g_per_sm", C.c_int32),
        ("dynamic_tiles", C.c_int32),
        ("graph_attempts", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


KEEP_GOING_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)

PARTICLE_FIELDS = {
    # name: (ctype, components)
    "id": (C.c_uint32, 1),
    "position": (C.c_double, 3),
    "velocity": (C.c_double, 3),
    "affine": (C.c_double, 9),
    "deformation": (C.c_double, 9),
    "volume_ratio": (C.c_double, 1),
    "kirchhoff": (C.c_double, 9),
    "plastic_strain": (C.c_double, 1),
    "mass": (C.c_double, 1),
    "volume0": (C.c_double, 1),
    "yield_stress": (C.c_double, 1),
}


def particle_buffers(count: int):
    """Allocate numpy arrays for `count` particles and a `Particles` view over them."""
    import numpy as np

    arrays = {}
    view = Particles()
    view.count = count
    for name, (ctype, comps) in PARTICLE_FIELDS.items():
        dtype = np.uint32 if ctype is C.c_uint32 else np.float64
        shape = (count,) if comps == 1 else (count, 3) if comps == 3 else (count, 3, 3)
        arr = np.zeros(shape, dtype=dtype)
        arrays[name] = arr
        setattr(view, name, arr.ctypes.data_as(C.POINTER(ctype)))
    return arrays, view


def particle_out_view(arrays: dict, count: int) -> Particles:
    """A `Particles` view over caller-owned output arrays for an export of `count` particles.

    Every field must be present, C-contiguous, writable and of the dtype and shape that
    `particle_buffers` allocates; a resident host particle set can then be refreshed in place,
    without allocating (and first touching) new pages."""
    import numpy as np

    view = Particles()
    view.count = count
    for name, (ctype, comps) in PARTICLE_FIELDS.items():
        arr = arrays.get(name)
        dtype = np.uint32 if ctype is C.c_uint32 else np.float64
        shape = (count,) if comps == 1 else (count, 3) if comps == 3 else (count, 3, 3)
        if (arr is None or not isinstance(arr, np.ndarray) or arr.dtype != dtype or arr.shape != shape
                or not arr.flags.c_contiguous or not arr.flags.writeable):
            raise ValueError(f"output field {name!r} must be a writable C-contiguous {np.dtype(dtype).name} "
                             f"array of shape {shape}")
        setattr(view, name, arr.ctypes.data_as(C.POINTER(ctype)))
    return view


def particle_view(arrays: dict) -> Particles:
    """A `Particles` view over caller arrays (must be C-contiguous, dtype as above)."""
    view = Particles()
    view.count = len(arrays["id"])
    for name, (ctype, _) in PARTICLE_FIELDS.items():
        arr = arrays.get(name)
        if arr is None:
            setattr(view, name, None)
            continue
        setattr(view, name, arr.ctypes.data_as(C.POINTER(ctype)))
    return view
