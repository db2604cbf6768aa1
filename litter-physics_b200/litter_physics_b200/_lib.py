"""ctypes binding of the device library (liblp_mpm.so, C ABI in include/lp_mpm.h).

This is the Python side of the drop-in boundary: the same entry points a Rust host binds with
`extern "C"`.  The library is built in-tree (`make -C litter-physics_b200`); importing a module
that needs it fails loudly when the shared object is missing, and every compute entry point
returns LP_DEVICE without a CUDA device: there is no host fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
from pathlib import Path

from . import _abi

PKG_ROOT = Path(__file__).resolve().parents[1]  # litter-physics_b200/
LIB_PATH = PKG_ROOT / "_build" / "liblp_mpm.so"
HEADER = PKG_ROOT.parent / "include" / "lp_mpm.h"

_lib = None


class LibraryMissing(RuntimeError):
    """The CUDA library has not been built."""


class LPError(RuntimeError):
    """An lp_* call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def build(quiet: bool = True) -> Path:
    """Compile the library for sm_100a with its Makefile (nvcc; no GPU needed)."""
    cmd = ["make", "-C", str(PKG_ROOT)]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return LIB_PATH


def declared_functions() -> list[str]:
    """Names of every function the C header declares."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(lp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_fn")))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise LibraryMissing(f"{LIB_PATH} is missing; build it with `make -C {PKG_ROOT}`")
    L = C.CDLL(str(LIB_PATH), mode=os.RTLD_GLOBAL)
    P, D, I32, I64, U64 = C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.c_int64, C.c_uint64
    F = C.POINTER(C.c_float)
    sig = {
        "lp_abi_version": ([], I32),
        "lp_last_error": ([], C.c_char_p),
        "lp_kernel_launches": ([], U64),
        "lp_abi_struct_sizes": ([C.POINTER(C.c_uint64)], None),
        "lp_material_paste": ([C.c_double] * 6, _abi.Material),
        "lp_material_paste_from_shear_rheology": ([C.c_double] * 6, _abi.Material),
        "lp_material_liquid": ([C.c_double] * 4, _abi.Material),
        "lp_material_wave_speed": ([C.POINTER(_abi.Material)], C.c_double),
        "lp_material_diffusivity": ([C.POINTER(_abi.Material)], C.c_double),
        "lp_sim_create": ([C.POINTER(_abi.FixtureSpec), C.POINTER(P)], I32),
        "lp_sim_destroy": ([P], None),
        "lp_sim_set_stream": ([P, P], I32),
        "lp_sim_advance": ([P, C.c_double, _abi.KEEP_GOING_FN, P, C.POINTER(I32)], I32),
        "lp_sim_try_step": ([P, C.c_double, C.POINTER(I32), C.c_char_p, C.c_size_t], I32),
        "lp_sim_run_substeps": ([P, I32], I32),
        "lp_sim_sync": ([P], I32),
        "lp_sim_stability_limit": ([P, D], I32),
        "lp_sim_audit_step": ([P, C.c_double, C.POINTER(_abi.EnergyAudit)], I32),
        "lp_sim_get_ledger": ([P, C.POINTER(_abi.Ledger)], I32),
        "lp_sim_set_ledger": ([P, C.POINTER(_abi.Ledger)], I32),
        "lp_sim_get_counters": ([P, C.POINTER(_abi.Counters)], I32),
        "lp_sim_set_counters": ([P, C.POINTER(_abi.Counters)], I32),
        "lp_sim_particle_count": ([P, C.POINTER(U64)], I32),
        "lp_sim_export_particles": ([P, C.POINTER(_abi.Particles)], I32),
        "lp_sim_import_particles": ([P, C.POINTER(_abi.Particles)], I32),
        "lp_host_pin": ([P, U64], I32),
        "lp_host_unpin": ([P], I32),
        "lp_sim_get_pellet": ([P, C.POINTER(_abi.Pellet), C.POINTER(I32)], I32),
        "lp_sim_set_pellet": ([P, C.POINTER(_abi.Pellet)], I32),
        "lp_sim_get_pellets": ([P, C.POINTER(_abi.Pellet), I32, C.POINTER(I32)], I32),
        "lp_sim_set_pellets": ([P, C.POINTER(_abi.Pellet), I32], I32),
        "lp_sim_observables": ([P, C.c_char_p, D, I32, C.POINTER(I32)], I32),
        "lp_sim_energies": ([P, D], I32),
        "lp_sim_set_warm_start": ([P, F, I32, I32], I32),
        "lp_sim_warm_table": ([P, F, I32, D], I32),
        "lp_sim_use_graph": ([P, I32], I32),
        "lp_sim_prepare": ([P], I32),
        "lp_sim_grid_totals": ([P, C.c_double, D], I32),
        "lp_sim_grid_dump": ([P, C.c_double, D, D, D, I64], I32),
        "lp_sim_kernel_times": ([P, I32, D, C.c_char_p, I32, C.POINTER(I32)], I32),
        "lp_sim_enable_newton_log": ([P, I64], I32),
        "lp_sim_read_newton_log": ([P, F, F, I64, C.POINTER(I64)], I32),
        "lp_batch_create": ([C.POINTER(_abi.FixtureSpec), I32, C.POINTER(P)], I32),
        "lp_batch_destroy": ([P], None),
        "lp_batch_set_stream": ([P, P], I32),
        "lp_batch_advance": ([P, C.c_double, _abi.KEEP_GOING_FN, P, C.POINTER(I32)], I32),
        "lp_batch_run_substeps": ([P, I32], I32),
        "lp_batch_sync": ([P], I32),
        "lp_batch_get_counters": ([P, I32, C.POINTER(_abi.Counters)], I32),
        "lp_batch_get_ledger": ([P, I32, C.POINTER(_abi.Ledger)], I32),
        "lp_batch_export_particles": ([P, I32, C.POINTER(_abi.Particles)], I32),
        "lp_batch_total_particles": ([P, C.POINTER(U64)], I32),
        "lp_batch_set_warm_start": ([P, F, I32, I32], I32),
        "lp_batch_warm_table": ([P, I32, F, I32, D], I32),
        "lp_batch_use_graph": ([P, I32], I32),
        "lp_batch_prepare": ([P], I32),
        "lp_batch_autotune": ([P, I32, C.c_char_p, C.c_size_t], I32),
        "lp_sim_autotune": ([P, I32, C.c_char_p, C.c_size_t], I32),
        "lp_sim_g2p_return_share": ([P, I32, D], I32),
        "lp_sim_set_launch_shape": ([P, C.POINTER(_abi.LaunchShape)], I32),
        "lp_sim_get_launch_shape": ([P, C.POINTER(_abi.LaunchShape)], I32),
        "lp_batch_set_launch_shape": ([P, C.POINTER(_abi.LaunchShape)], I32),
        "lp_batch_get_launch_shape": ([P, C.POINTER(_abi.LaunchShape)], I32),
        "lp_batch_kernel_times": ([P, I32, D, C.c_char_p, I32, C.POINTER(I32)], I32),
        "lp_batch_get_pellet": ([P, I32, C.POINTER(_abi.Pellet), C.POINTER(I32)], I32),
        "lp_batch_observables": ([P, I32, C.c_char_p, D, I32, C.POINTER(I32)], I32),
        "lp_batch_energies": ([P, I32, D], I32),
        "lp_batch_instance_state": ([P, I32, C.POINTER(I32), C.c_char_p, C.c_size_t], I32),
        "lp_hb_return_batch": ([I64, D, D, D, D, D, D, C.c_double, F, I32, D, C.POINTER(I32)], I32),
        "lp_update_paste_batch": ([I64, D, C.POINTER(_abi.Material), C.c_double, D, D, D, D, D, C.POINTER(I32)], I32),
        "lp_update_liquid_batch": ([I64, D, D, C.POINTER(_abi.Material), C.c_double, D, D, D, C.POINTER(I32)], I32),
        "lp_mlp_weight_count": ([], I32),
        "lp_mlp_init": ([F, I32, U64], I32),
        "lp_mlp_train": ([F, I32, F, F, I64, I32, I32, C.c_float, F], I32),
        "lp_mlp_forward": ([F, I32, F, I64, F], I32),
        "lp_mlp_forward_mma": ([F, I32, F, I64, F], I32),
        "lp_mlp_loss_grad": ([F, I32, F, F, I64, F, F], I32),
        "lp_mlp_loss_grad_noalloc": ([P, P, P, I64, P, P, P], I32),
        "lp_hb_features": ([C.c_double] * 6 + [F], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != 0:
        raise LPError(status, lib().lp_last_error().decode(errors="replace"))


def struct_sizes() -> dict:
    out = (C.c_uint64 * 6)()
    lib().lp_abi_struct_sizes(out)
    return dict(zip(["material", "fixture_spec", "ledger", "counters", "particles", "pellet"], list(out)))


def kernel_launches() -> int:
    return int(lib().lp_kernel_launches())
