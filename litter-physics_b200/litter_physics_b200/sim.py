"""Python mirror of the reference's `Simulation` / `FixtureSpec` API over the device library.

`Simulation(spec)` corresponds to `FixtureSpec::build` (core/src/mpm/fixtures.rs:238-268) and
exposes the calls the reference's tests and research driver make on a `Simulation`
(core/src/mpm/solver.rs): `advance_to`, `advance_while`, `try_step`, `stability_limit`,
`ledger`, the residual and energy accessors, `observables` (fixtures.rs:369-461), and
checkpoint-style state export / import.  All arithmetic happens on the GPU; this module only
marshals plain buffers across the C ABI.
"""

from __future__ import annotations

import ctypes as C
from typing import Callable

import numpy as np

from . import _abi
from ._lib import LPError, check, lib


def _shape_with(read, fields: dict) -> _abi.LaunchShape:
    """The current launch shape (read(s) fills s with the CTAs per SM in use) with `fields`
    replaced.  A changed G2P block shape or P2G variant without its own CTAs-per-SM field gets 0
    (as many as fit that instantiation) instead of the count that fitted the previous one."""
    s = _abi.LaunchShape()
    read(s)
    if "g2p_variant" in fields and "g2p_per_sm" not in fields and int(fields["g2p_variant"]) != s.g2p_variant:
        s.g2p_per_sm = 0
    if "p2g_variant" in fields and "p2g_per_sm" not in fields and int(fields["p2g_variant"]) != s.p2g_variant:
        s.p2g_per_sm = 0
    for k, v in fields.items():
        setattr(s, k, int(v))
    return s


class Simulation:
    """One MLS-MPM simulation resident on the GPU."""

    def __init__(self, spec: _abi.FixtureSpec):
        self.spec = spec
        self._h = C.c_void_p()
        check(lib().lp_sim_create(C.byref(spec), C.byref(self._h)))

    # ------------------------------------------------------------------ lifetime
    def close(self) -> None:
        if self._h:
            lib().lp_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ stepping
    def advance_while(self, target_time: float, should_continue: Callable[[], bool] | None = None) -> bool:
        """solver.rs:413-472: returns False at a resumable budget stop."""
        reached = C.c_int32()
        cb = _abi.KEEP_GOING_FN(lambda _ctx: 1 if should_continue() else 0) if should_continue else \
            _abi.KEEP_GOING_FN(0)
        st = lib().lp_sim_advance(self._h, float(target_time), cb, None, C.byref(reached))
        if st == _abi.LP_BUDGET:
            return False
        check(st)
        return bool(reached.value)

    def advance_to(self, target_time: float) -> None:
        """solver.rs:402-404."""
        self.advance_while(target_time)

    def try_step(self, dt: float) -> tuple[bool, str]:
        """One trial step of exactly dt (solver.rs:535-611); committed only on success."""
        acc = C.c_int32()
        reason = C.create_string_buffer(256)
        check(lib().lp_sim_try_step(self._h, float(dt), C.byref(acc), reason, 256))
        return bool(acc.value), reason.value.decode()

    def run_substeps(self, steps: int) -> None:
        """Queue `steps` controlled attempts on the stream without synchronising."""
        check(lib().lp_sim_run_substeps(self._h, int(steps)))

    def sync(self) -> None:
        check(lib().lp_sim_sync(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib().lp_sim_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def use_graph(self, steps: int) -> None:
        check(lib().lp_sim_use_graph(self._h, int(steps)))

    def prepare(self) -> None:
        """Build the launch shape's CUDA graph now (no launch), so run_substeps pays no capture."""
        check(lib().lp_sim_prepare(self._h))

    def autotune(self, trial_steps: int = 16) -> str:
        """Pick the launch shape on the live simulation (advances it); returns the report."""
        buf = C.create_string_buffer(8192)
        check(lib().lp_sim_autotune(self._h, int(trial_steps), buf, 8192))
        return buf.value.decode()

    def launch_shape(self) -> dict:
        s = _abi.LaunchShape()
        check(lib().lp_sim_get_launch_shape(self._h, C.byref(s)))
        return s.as_dict()

    def g2p_return_share(self, steps: int) -> float:
        """Share of G2P warp time in the FP64 Herschel-Bulkley return over `steps` real attempts
        (clock-instrumented G2P): what any Newton start could save in G2P at most."""
        out = C.c_double()
        check(lib().lp_sim_g2p_return_share(self._h, int(steps), C.byref(out)))
        return out.value

    def set_launch_shape(self, **fields) -> None:
        """Set fields of `lp_launch_shape` (g2p_variant, g2p_per_sm, p2g_variant, p2g_per_sm,
        dynamic_tiles, graph_attempts); the others keep their values, except that a new G2P
        block shape or P2G variant given without its CTAs per SM gets as many as fit."""
        check(lib().lp_sim_set_launch_shape(self._h, C.byref(_shape_with(
            lambda s: check(lib().lp_sim_get_launch_shape(self._h, C.byref(s))), fields))))

    def stability_limit(self) -> float:
        out = C.c_double()
        check(lib().lp_sim_stability_limit(self._h, C.byref(out)))
        return out.value

    def audit_step(self, dt: float) -> dict:
        """Energy audit of one trial step of exactly `dt` (audit.rs:284-353): endpoint energies,
        stage grid energies, ledger increments and the stage telescope terms.  The committed
        state is unchanged.  A refused `dt` or a rejected trial raises ValueError."""
        out = _abi.EnergyAudit()
        status = lib().lp_sim_audit_step(self._h, float(dt), C.byref(out))
        if status == _abi.LP_INVALID:
            raise ValueError(lib().lp_last_error().decode(errors="replace"))
        check(status)
        return out.as_dict()

    # ------------------------------------------------------------------ state
    @property
    def ledger(self) -> _abi.Ledger:
        led = _abi.Ledger()
        check(lib().lp_sim_get_ledger(self._h, C.byref(led)))
        return led

    def set_ledger(self, led: _abi.Ledger) -> None:
        check(lib().lp_sim_set_ledger(self._h, C.byref(led)))

    @property
    def counters(self) -> _abi.Counters:
        c = _abi.Counters()
        check(lib().lp_sim_get_counters(self._h, C.byref(c)))
        return c

    def set_counters(self, c: _abi.Counters) -> None:
        check(lib().lp_sim_set_counters(self._h, C.byref(c)))

    @property
    def time(self) -> float:
        return self.counters.time

    def particle_count(self) -> int:
        n = C.c_uint64()
        check(lib().lp_sim_particle_count(self._h, C.byref(n)))
        return int(n.value)

    def particles(self, out: dict | None = None) -> dict:
        """Export the committed particle set (FP64 arrays in the reference layout, slot order).

        `out`: arrays of a resident host particle set (as returned by an earlier export) to
        overwrite in place instead of allocating new ones."""
        n = self.particle_count()
        if out is None:
            arrays, view = _abi.particle_buffers(n)
        else:
            arrays, view = out, _abi.particle_out_view(out, n)
        check(lib().lp_sim_export_particles(self._h, C.byref(view)))
        return arrays

    def set_particles(self, arrays: dict) -> None:
        view = _abi.particle_view(arrays)
        check(lib().lp_sim_import_particles(self._h, C.byref(view)))

    def pellet(self) -> _abi.Pellet | None:
        p = _abi.Pellet()
        has = C.c_int32()
        check(lib().lp_sim_get_pellet(self._h, C.byref(p), C.byref(has)))
        return p if has.value else None

    def set_pellet(self, p: _abi.Pellet) -> None:
        check(lib().lp_sim_set_pellet(self._h, C.byref(p)))

    def pellets(self) -> list:
        """Pellet bed (extension): committed state of every pellet, in index order."""
        n = C.c_int32()
        check(lib().lp_sim_get_pellets(self._h, None, 0, C.byref(n)))
        arr = (_abi.Pellet * max(n.value, 1))()
        check(lib().lp_sim_get_pellets(self._h, arr, n.value, C.byref(n)))
        return list(arr)[: n.value]

    def set_pellets(self, pellets: list) -> None:
        """Pellet bed: replace every pellet's pose and momenta (contact histories restart)."""
        arr = (_abi.Pellet * len(pellets))(*pellets)
        check(lib().lp_sim_set_pellets(self._h, arr, len(pellets)))

    def observables(self) -> dict:
        cap = 128
        names = C.create_string_buffer(64 * cap)
        values = (C.c_double * cap)()
        n = C.c_int32()
        check(lib().lp_sim_observables(self._h, names, values, cap, C.byref(n)))
        raw = names.raw
        return {raw[64 * i:64 * i + 64].split(b"\0", 1)[0].decode(): values[i] for i in range(n.value)}

    def energies(self) -> dict:
        out = (C.c_double * 9)()
        check(lib().lp_sim_energies(self._h, out))
        keys = ["kinetic", "potential", "elastic", "mechanical", "mass_residual", "momentum_residual_x",
                "momentum_residual_y", "momentum_residual_z", "energy_residual"]
        return dict(zip(keys, list(out)))

    def momentum_residual(self) -> np.ndarray:
        e = self.energies()
        return np.array([e["momentum_residual_x"], e["momentum_residual_y"], e["momentum_residual_z"]])

    def mass_residual(self) -> float:
        return self.energies()["mass_residual"]

    def energy_residual(self) -> float:
        return self.energies()["energy_residual"]

    def grid_totals(self, dt: float) -> dict:
        """Scatter the committed state (P2G only) and compare grid and particle totals."""
        out = (C.c_double * 8)()
        check(lib().lp_sim_grid_totals(self._h, float(dt), out))
        return {"grid_mass": out[0], "grid_momentum": np.array(out[1:4]), "particle_mass": out[4],
                "particle_momentum": np.array(out[5:8])}

    def grid_dump(self, dt: float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """P2G and wall traction of the committed state with step `dt`: (node mass, node
        momentum before the wall reactions, signed wall reaction impulse), dense padded node
        order ((n+3)^3 nodes, grid.rs:71-109).  The simulation state is unchanged."""
        nodes = [int(round(d / self.spec.grid_spacing)) + 3 for d in self.spec.domain]
        nn = nodes[0] * nodes[1] * nodes[2]
        mass = np.zeros(nn)
        mom = np.zeros((nn, 3))
        reaction = np.zeros((nn, 3))
        D = C.POINTER(C.c_double)
        check(lib().lp_sim_grid_dump(self._h, float(dt), mass.ctypes.data_as(D), mom.ctypes.data_as(D),
                                     reaction.ctypes.data_as(D), nn))
        return mass, mom, reaction

    def kernel_times(self, steps: int) -> dict:
        """Mean per-kernel duration (ms) over `steps` attempts, CUDA events on the stream."""
        cap = 24
        ms = (C.c_double * cap)()
        names = C.create_string_buffer(32 * cap)
        n = C.c_int32()
        check(lib().lp_sim_kernel_times(self._h, int(steps), ms, names, cap, C.byref(n)))
        raw = names.raw
        return {raw[32 * i:32 * i + 32].split(b"\0", 1)[0].decode(): ms[i] for i in range(n.value)}

    # ------------------------------------------------------------------ learned warm start
    def set_warm_start(self, weights: np.ndarray | None) -> None:
        if weights is None:
            check(lib().lp_sim_set_warm_start(self._h, None, 0, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32)
        check(lib().lp_sim_set_warm_start(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size, 1))

    def warm_table(self) -> tuple[np.ndarray | None, float]:
        """The warm start's logit table (network logits at the la8 nodes of `_abi.MLP_TAB_*`)
        and the dt it was built for; (None, nan) before the first warm-started attempt."""
        out = np.zeros(_abi.MLP_TAB_N, dtype=np.float32)
        dt = C.c_double()
        check(lib().lp_sim_warm_table(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size, C.byref(dt)))
        return (out if np.isfinite(dt.value) else None), dt.value

    def enable_newton_log(self, capacity: int) -> None:
        check(lib().lp_sim_enable_newton_log(self._h, int(capacity)))

    def read_newton_log(self, capacity: int) -> tuple[np.ndarray, np.ndarray]:
        x = np.zeros((capacity, 6), dtype=np.float32)
        y = np.zeros(capacity, dtype=np.float32)
        n = C.c_int64()
        check(lib().lp_sim_read_newton_log(self._h, x.ctypes.data_as(C.POINTER(C.c_float)),
                                           y.ctypes.data_as(C.POINTER(C.c_float)), capacity, C.byref(n)))
        return x[: n.value], y[: n.value]


class PinnedParticles:
    """Page-locks the arrays of a resident host particle set (lp_host_pin) until close().

    Export and import then move them by DMA straight between host and device, without the
    library's staging copy.  Pin a set once and reuse it: page-locking is itself costly."""

    def __init__(self, arrays: dict):
        self.arrays = arrays
        self._pinned = []
        try:
            for a in arrays.values():
                if a is None or a.nbytes == 0:
                    continue
                if not a.flags["C_CONTIGUOUS"]:
                    raise ValueError("pinned particle arrays must be C-contiguous")
                check(lib().lp_host_pin(a.ctypes.data, a.nbytes))
                self._pinned.append(a)
        except Exception:
            self.close()
            raise

    def close(self) -> None:
        while self._pinned:
            a = self._pinned.pop()
            check(lib().lp_host_unpin(a.ctypes.data))

    def __enter__(self):
        return self.arrays

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Many independent simulations advanced by one device launch sequence (extension)."""

    def __init__(self, specs: list[_abi.FixtureSpec]):
        arr = (_abi.FixtureSpec * len(specs))(*specs)
        self.specs = specs
        self._h = C.c_void_p()
        check(lib().lp_batch_create(arr, len(specs), C.byref(self._h)))

    def close(self) -> None:
        if self._h:
            lib().lp_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance_to(self, target_time: float) -> bool:
        reached = C.c_int32()
        check(lib().lp_batch_advance(self._h, float(target_time), _abi.KEEP_GOING_FN(0), None, C.byref(reached)))
        return bool(reached.value)

    def advance_while(self, target_time: float, should_continue: Callable[[], bool] | None = None) -> str:
        """Advance every running instance toward `target_time`.  Returns "budget" at a resumable
        budget stop, else "done"; instances that stop on their own (min step, outflow) stay
        stopped and are reported by `state(i)`, not raised."""
        reached = C.c_int32()
        cb = _abi.KEEP_GOING_FN(lambda _ctx: 1 if should_continue() else 0) if should_continue else \
            _abi.KEEP_GOING_FN(0)
        st = lib().lp_batch_advance(self._h, float(target_time), cb, None, C.byref(reached))
        if st == _abi.LP_BUDGET:
            return "budget"
        if st in (_abi.LP_OK, _abi.LP_MIN_STEP) or (st == _abi.LP_INVALID and "outflow" in
                                                   lib().lp_last_error().decode(errors="replace")):
            return "done"
        check(st)
        return "done"

    def state(self, i: int) -> tuple[str, str]:
        """("running" | "reached" | "min_step" | "outflow", reason) of instance i."""
        st = C.c_int32()
        msg = C.create_string_buffer(256)
        check(lib().lp_batch_instance_state(self._h, i, C.byref(st), msg, 256))
        return ("running", "reached", "min_step", "outflow")[st.value], msg.value.decode()

    def pellet(self, i: int) -> _abi.Pellet | None:
        p = _abi.Pellet()
        has = C.c_int32()
        check(lib().lp_batch_get_pellet(self._h, i, C.byref(p), C.byref(has)))
        return p if has.value else None

    def observables(self, i: int) -> dict:
        cap = 128
        names = C.create_string_buffer(64 * cap)
        values = (C.c_double * cap)()
        n = C.c_int32()
        check(lib().lp_batch_observables(self._h, i, names, values, cap, C.byref(n)))
        raw = names.raw
        return {raw[64 * k:64 * k + 64].split(b"\0", 1)[0].decode(): values[k] for k in range(n.value)}

    def energies(self, i: int) -> dict:
        out = (C.c_double * 9)()
        check(lib().lp_batch_energies(self._h, i, out))
        keys = ["kinetic", "potential", "elastic", "mechanical", "mass_residual", "momentum_residual_x",
                "momentum_residual_y", "momentum_residual_z", "energy_residual"]
        return dict(zip(keys, list(out)))

    def member(self, i: int) -> "BatchMember":
        return BatchMember(self, i)

    def run_substeps(self, steps: int) -> None:
        check(lib().lp_batch_run_substeps(self._h, int(steps)))

    def sync(self) -> None:
        check(lib().lp_batch_sync(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib().lp_batch_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def use_graph(self, steps: int) -> None:
        check(lib().lp_batch_use_graph(self._h, int(steps)))

    def prepare(self) -> None:
        """`Simulation.prepare` for the whole batch."""
        check(lib().lp_batch_prepare(self._h))

    def autotune(self, trial_steps: int = 16) -> str:
        """Pick the launch shape on the live batch (advances it); returns the tuner's report."""
        buf = C.create_string_buffer(8192)
        check(lib().lp_batch_autotune(self._h, int(trial_steps), buf, 8192))
        return buf.value.decode()

    def launch_shape(self) -> dict:
        s = _abi.LaunchShape()
        check(lib().lp_batch_get_launch_shape(self._h, C.byref(s)))
        return s.as_dict()

    def set_launch_shape(self, **fields) -> None:
        """`Simulation.set_launch_shape` for the whole batch."""
        check(lib().lp_batch_set_launch_shape(self._h, C.byref(_shape_with(
            lambda s: check(lib().lp_batch_get_launch_shape(self._h, C.byref(s))), fields))))

    def kernel_times(self, steps: int) -> dict:
        """Mean per-kernel duration (ms) over `steps` attempts of the whole batch."""
        cap = 24
        ms = (C.c_double * cap)()
        names = C.create_string_buffer(32 * cap)
        n = C.c_int32()
        check(lib().lp_batch_kernel_times(self._h, int(steps), ms, names, cap, C.byref(n)))
        raw = names.raw
        return {raw[32 * i:32 * i + 32].split(b"\0", 1)[0].decode(): ms[i] for i in range(n.value)}

    def counters(self, i: int) -> _abi.Counters:
        c = _abi.Counters()
        check(lib().lp_batch_get_counters(self._h, i, C.byref(c)))
        return c

    def ledger(self, i: int) -> _abi.Ledger:
        led = _abi.Ledger()
        check(lib().lp_batch_get_ledger(self._h, i, C.byref(led)))
        return led

    def particles(self, i: int, out: dict | None = None) -> dict:
        """Export instance i's committed particle set (`out`: arrays to overwrite in place)."""
        n = int(self.counters(i).particle_count)
        if out is None:
            arrays, view = _abi.particle_buffers(n)
        else:
            arrays, view = out, _abi.particle_out_view(out, n)
        check(lib().lp_batch_export_particles(self._h, i, C.byref(view)))
        return arrays

    def total_particles(self) -> int:
        n = C.c_uint64()
        check(lib().lp_batch_total_particles(self._h, C.byref(n)))
        return int(n.value)

    def set_warm_start(self, weights: np.ndarray | None) -> None:
        if weights is None:
            check(lib().lp_batch_set_warm_start(self._h, None, 0, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32)
        check(lib().lp_batch_set_warm_start(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size, 1))

    def warm_table(self, i: int) -> tuple[np.ndarray | None, float]:
        """`Simulation.warm_table` of member i."""
        out = np.zeros(_abi.MLP_TAB_N, dtype=np.float32)
        dt = C.c_double()
        check(lib().lp_batch_warm_table(self._h, int(i), out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                        C.byref(dt)))
        return (out if np.isfinite(dt.value) else None), dt.value


class BatchMember:
    """Read-only view of one batch instance with the `Simulation` accessors the research driver
    uses (particles, ledger, counters, time, pellet, observables, residuals)."""

    def __init__(self, batch: Batch, index: int):
        self.batch, self.index = batch, index

    def particles(self) -> dict:
        return self.batch.particles(self.index)

    @property
    def ledger(self) -> _abi.Ledger:
        return self.batch.ledger(self.index)

    @property
    def counters(self) -> _abi.Counters:
        return self.batch.counters(self.index)

    @property
    def time(self) -> float:
        return self.counters.time

    def pellet(self) -> _abi.Pellet | None:
        return self.batch.pellet(self.index)

    def observables(self) -> dict:
        return self.batch.observables(self.index)

    def energies(self) -> dict:
        return self.batch.energies(self.index)

    def mass_residual(self) -> float:
        return self.energies()["mass_residual"]


__all__ = ["Simulation", "Batch", "BatchMember", "LPError"]
