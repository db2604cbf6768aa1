"""Python loader of the FP64 CPU oracle (oracle/_build/liblp_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline to check and time the reference algorithm.  The product package never imports
this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "litter-physics_b200"))
from litter_physics_b200 import _abi  # noqa: E402

LIB_PATH = HERE / "_build" / "liblp_oracle.so"
_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (seconds)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        L.ora_sim_create.argtypes = [C.POINTER(_abi.FixtureSpec), C.POINTER(P), C.c_char_p, C.c_int32]
        L.ora_sim_create.restype = C.c_int32
        L.ora_sim_destroy.argtypes = [P]
        L.ora_sim_advance.argtypes = [P, C.c_double, C.c_int64, C.POINTER(C.c_int32), C.c_char_p, C.c_int32]
        L.ora_sim_advance.restype = C.c_int32
        L.ora_sim_try_step.argtypes = [P, C.c_double, C.POINTER(C.c_int32), C.c_char_p, C.c_int32]
        L.ora_sim_try_step.restype = C.c_int32
        L.ora_sim_stability_limit.argtypes = [P]
        L.ora_sim_stability_limit.restype = C.c_double
        L.ora_sim_counters.argtypes = [P, C.POINTER(_abi.Counters)]
        L.ora_sim_ledger.argtypes = [P, C.POINTER(_abi.Ledger)]
        L.ora_sim_set_ledger.argtypes = [P, C.POINTER(_abi.Ledger)]
        L.ora_sim_particle_count.argtypes = [P]
        L.ora_sim_particle_count.restype = C.c_uint64
        L.ora_sim_export_particles.argtypes = [P, C.POINTER(_abi.Particles)]
        L.ora_sim_import_particles.argtypes = [P, C.POINTER(_abi.Particles)]
        L.ora_sim_import_particles.restype = C.c_int32
        L.ora_sim_get_pellet.argtypes = [P, C.POINTER(_abi.Pellet)]
        L.ora_sim_get_pellet.restype = C.c_int32
        L.ora_sim_set_pellet.argtypes = [P, C.POINTER(_abi.Pellet)]
        L.ora_sim_audit_step.argtypes = [P, C.c_double, C.POINTER(_abi.EnergyAudit), C.c_char_p, C.c_int32]
        L.ora_sim_audit_step.restype = C.c_int32
        L.ora_sim_set_counters.argtypes = [P, C.POINTER(_abi.Counters)]
        L.ora_sim_set_counters.restype = C.c_int32
        L.ora_sim_get_pellets.argtypes = [P, C.POINTER(_abi.Pellet), C.c_int32]
        L.ora_sim_get_pellets.restype = C.c_int32
        L.ora_sim_set_pellets.argtypes = [P, C.POINTER(_abi.Pellet), C.c_int32]
        L.ora_sim_set_pellets.restype = C.c_int32
        L.ora_sim_observables.argtypes = [P, C.c_char_p, C.POINTER(C.c_double), C.c_int32]
        L.ora_sim_observables.restype = C.c_int32
        L.ora_sim_energies.argtypes = [P, C.POINTER(C.c_double)]
        L.ora_set_threads.argtypes = [C.c_int32]
        D = C.POINTER(C.c_double)
        L.ora_sim_probe_p2g.argtypes = [P, C.c_double, D, D, D, D]
        L.ora_sim_probe_p2g.restype = C.c_int64
        L.ora_sim_probe_grid.argtypes = [P, C.c_double, D, D, D]
        L.ora_sim_probe_grid.restype = C.c_int64
        L.ora_hb_return.argtypes = [C.c_double] * 7 + [D]
        L.ora_hb_return.restype = C.c_int32
        L.ora_update_paste.argtypes = [D, C.POINTER(_abi.Material), C.c_double, C.c_double, C.c_double, D, D, D]
        L.ora_update_paste.restype = C.c_int32
        L.ora_update_liquid.argtypes = [C.c_double, D, C.POINTER(_abi.Material), C.c_double, D, D, D]
        L.ora_update_liquid.restype = C.c_int32
        L.ora_eigen3.argtypes = [D, D, D]
        L.ora_eigen3.restype = C.c_int32
        L.ora_stencil.argtypes = [C.c_double, C.POINTER(C.c_int32), D, C.POINTER(C.c_int32), D, D]
        L.ora_stencil.restype = C.c_int32
        L.ora_splitmix_next_unit.argtypes = [C.POINTER(C.c_uint64)]
        L.ora_splitmix_next_unit.restype = C.c_double
        L.ora_splitmix_next_u64.argtypes = [C.POINTER(C.c_uint64)]
        L.ora_splitmix_next_u64.restype = C.c_uint64
        for name in ("ora_material_paste", "ora_material_paste_shear"):
            getattr(L, name).argtypes = [C.c_double] * 6
            getattr(L, name).restype = _abi.Material
        L.ora_material_liquid.argtypes = [C.c_double] * 4
        L.ora_material_liquid.restype = _abi.Material
        L.ora_grid_update_node.argtypes = [C.POINTER(_abi.FixtureSpec), C.POINTER(C.c_int32), C.c_double, D, D,
                                           C.c_double, D]
        L.ora_grid_update_node.restype = C.c_int32
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleError(RuntimeError):
    pass


class OracleSim:
    """FP64 restatement of `Simulation` built by `FixtureSpec::build` (fixtures.rs:238)."""

    def __init__(self, spec: _abi.FixtureSpec, threads: int = 0):
        L = lib()
        if threads:
            L.ora_set_threads(threads)
        self._h = C.c_void_p()
        err = C.create_string_buffer(512)
        st = L.ora_sim_create(C.byref(spec), C.byref(self._h), err, 512)
        if st != 0:
            raise OracleError(err.value.decode())
        self.spec = spec

    def close(self):
        if self._h:
            lib().ora_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance_to(self, target: float, max_accepted: int = 0) -> bool:
        reached = C.c_int32()
        err = C.create_string_buffer(512)
        st = lib().ora_sim_advance(self._h, target, max_accepted, C.byref(reached), err, 512)
        if st not in (0, _abi.LP_BUDGET):
            raise OracleError(err.value.decode())
        return bool(reached.value)

    def try_step(self, dt: float) -> tuple[bool, str]:
        acc = C.c_int32()
        reason = C.create_string_buffer(256)
        lib().ora_sim_try_step(self._h, dt, C.byref(acc), reason, 256)
        return bool(acc.value), reason.value.decode()

    def stability_limit(self) -> float:
        return lib().ora_sim_stability_limit(self._h)

    def counters(self) -> _abi.Counters:
        c = _abi.Counters()
        lib().ora_sim_counters(self._h, C.byref(c))
        return c

    def set_counters(self, c: _abi.Counters) -> None:
        if lib().ora_sim_set_counters(self._h, C.byref(c)) != 0:
            raise ValueError("invalid counters")

    def ledger(self) -> _abi.Ledger:
        led = _abi.Ledger()
        lib().ora_sim_ledger(self._h, C.byref(led))
        return led

    def set_ledger(self, led: _abi.Ledger) -> None:
        lib().ora_sim_set_ledger(self._h, C.byref(led))

    def particles(self) -> dict:
        n = int(lib().ora_sim_particle_count(self._h))
        arrays, view = _abi.particle_buffers(n)
        lib().ora_sim_export_particles(self._h, C.byref(view))
        return arrays

    def set_particles(self, arrays: dict) -> None:
        view = _abi.particle_view(arrays)
        lib().ora_sim_import_particles(self._h, C.byref(view))

    def pellet(self):
        p = _abi.Pellet()
        return p if lib().ora_sim_get_pellet(self._h, C.byref(p)) else None

    def set_pellet(self, p: _abi.Pellet) -> None:
        lib().ora_sim_set_pellet(self._h, C.byref(p))

    def audit_step(self, dt: float) -> dict:
        """audit.rs:284-353: energy audit of one trial step on a copy; raises ValueError."""
        out = _abi.EnergyAudit()
        err = C.create_string_buffer(512)
        if lib().ora_sim_audit_step(self._h, float(dt), C.byref(out), err, 512) != 0:
            raise ValueError(err.value.decode())
        return out.as_dict()

    def pellets(self) -> list:
        """Pellet bed (extension): committed pellets in index order."""
        n = lib().ora_sim_get_pellets(self._h, None, 0)
        arr = (_abi.Pellet * max(n, 1))()
        lib().ora_sim_get_pellets(self._h, arr, n)
        return list(arr)[:n]

    def set_pellets(self, pellets: list) -> None:
        arr = (_abi.Pellet * len(pellets))(*pellets)
        if lib().ora_sim_set_pellets(self._h, arr, len(pellets)) != 0:
            raise ValueError("pellet count differs from the bed's")

    def observables(self) -> dict:
        cap = 128
        names = C.create_string_buffer(64 * cap)
        values = (C.c_double * cap)()
        n = lib().ora_sim_observables(self._h, names, values, cap)
        raw = names.raw
        return {raw[64 * i:64 * i + 64].split(b"\0", 1)[0].decode(): values[i] for i in range(n)}

    def energies(self) -> dict:
        out = (C.c_double * 9)()
        lib().ora_sim_energies(self._h, out)
        keys = ["kinetic", "potential", "elastic", "mechanical", "mass_residual", "momentum_residual_x",
                "momentum_residual_y", "momentum_residual_z", "energy_residual"]
        return dict(zip(keys, list(out)))

    def probe_p2g(self, dt: float, node_count: int):
        mass = np.zeros(node_count)
        mom = np.zeros((node_count, 3))
        e = C.c_double()
        imp = np.zeros(3)
        active = lib().ora_sim_probe_p2g(self._h, dt, _dptr(mass), _dptr(mom), C.byref(e), _dptr(imp))
        return mass, mom, e.value, imp, active


    def probe_grid(self, dt: float, node_count: int):
        """One step's P2G deposit and wall traction on a copy: (node mass, node momentum before
        the reactions, signed reaction impulse per node), dense padded node order."""
        mass = np.zeros(node_count)
        mom = np.zeros((node_count, 3))
        reaction = np.zeros((node_count, 3))
        lib().ora_sim_probe_grid(self._h, dt, _dptr(mass), _dptr(mom), _dptr(reaction))
        return mass, mom, reaction


def hb_return(trial, yield_stress, consistency, flow_index, mu, dt, tol=1e-12):
    out = np.zeros(3)
    st = lib().ora_hb_return(trial, yield_stress, consistency, flow_index, mu, dt, tol, _dptr(out))
    return st, out[0], out[1], int(out[2])


def update_paste(f_trial, material: _abi.Material, dt, yield_override=-1.0, tol=1e-12):
    f = np.ascontiguousarray(np.asarray(f_trial, dtype=np.float64).reshape(9))
    fn = np.zeros(9)
    tau = np.zeros(9)
    out = np.zeros(3)
    st = lib().ora_update_paste(_dptr(f), C.byref(material), yield_override, dt, tol, _dptr(fn), _dptr(tau),
                                _dptr(out))
    return st, fn.reshape(3, 3), tau.reshape(3, 3), out[0], out[1], out[2]


def update_liquid(j, grad, material: _abi.Material, dt):
    g = np.ascontiguousarray(np.asarray(grad, dtype=np.float64).reshape(9))
    jn = C.c_double()
    tau = np.zeros(9)
    p = C.c_double()
    st = lib().ora_update_liquid(j, _dptr(g), C.byref(material), dt, C.byref(jn), _dptr(tau), C.byref(p))
    return st, jn.value, tau.reshape(3, 3), p.value


def eigen3(m):
    a = np.ascontiguousarray(np.asarray(m, dtype=np.float64).reshape(9))
    vals = np.zeros(3)
    vecs = np.zeros(9)
    st = lib().ora_eigen3(_dptr(a), _dptr(vals), _dptr(vecs))
    return st, vals, vecs.reshape(3, 3)


def stencil(spacing, nodes, x):
    n = (C.c_int32 * 3)(*nodes)
    xx = np.asarray(x, dtype=np.float64)
    base = (C.c_int32 * 3)()
    w = np.zeros(9)
    off = np.zeros(9)
    st = lib().ora_stencil(spacing, n, _dptr(xx), base, _dptr(w), _dptr(off))
    return st, list(base), w.reshape(3, 3), off.reshape(3, 3)


def material_paste(*args):
    return lib().ora_material_paste(*[float(a) for a in args])


def material_paste_shear(*args):
    return lib().ora_material_paste_shear(*[float(a) for a in args])


def material_liquid(*args):
    return lib().ora_material_liquid(*[float(a) for a in args])


def grid_update_node(spec, coords, mass, momentum, traction, dt):
    out = np.zeros(8)
    mom = np.asarray(momentum, dtype=np.float64)
    tr = np.asarray(traction, dtype=np.float64)
    st = lib().ora_grid_update_node(C.byref(spec), (C.c_int32 * 3)(*coords), mass, _dptr(mom), _dptr(tr), dt,
                                    _dptr(out))
    if st:
        raise OracleError("grid update probe failed")
    return out[:3], out[3:6], out[6], out[7]


def threads_available() -> int:
    return len(os.sched_getaffinity(0))
