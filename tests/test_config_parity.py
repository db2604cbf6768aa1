"""Parity at the benchmark configurations' own sizes, against the FP64 oracle, through the C ABI.

Every case runs 100 substeps on the GPU and in the oracle from the same seeded fixture, matches
particles by id and checks the north-star bars:
  * positions: max_p |x_gpu - x_ref| / L_domain <= 1e-5;
  * velocities: ||v_gpu - v_ref||_2 / ||v_ref||_2 <= 1e-5 (every case here is in motion: a
    slumping column or a breaking dam, so ||v_ref|| is the physical velocity, not noise);
  * the same accepted and rejected step counts;
  * ledgers: gravity and wall impulses to 1e-5, the energy channels (wall projection, wall
    friction, wall traction, plastic work) to 1e-4 relative (FP32 particle arithmetic against
    FP64; measured at most 5e-7 and 1e-5).

Cases (sizes as the benchmark configurations state them):
  * the plain HB slump: 64^3 grid, 16x16x32-cell column, 65,536 particles, seed 0;
  * the Tait dam break: 128^3 grid, 64x32x64-cell block, 1,048,576 particles, seed 1, gamma 7,
    dt capped at 5e-5 s;
  * the large slump's resolution and material on a 32^3-cell column (256^3 grid, 262,144
    particles, seed 2, yield stress U(20, 100) Pa per particle), plain and warm-started;
  * the first eight members of the 256-instance calibration sweep, advanced together in one
    batch, each against its own oracle run.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
VEL_TOL = 1e-5
STEPS = 100


@pytest.fixture(scope="module")
def lib_built():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


def by_id(p: dict) -> dict:
    order = np.argsort(p["id"])
    return {k: v[order] for k, v in p.items()}


def particle_errors(gpu: dict, ref: dict, length: float) -> dict:
    g, r = by_id(gpu), by_id(ref)
    assert np.array_equal(g["id"], r["id"])
    x_err = float(np.max(np.abs(g["position"] - r["position"]))) / length
    v_ref = float(np.linalg.norm(r["velocity"]))
    dv = float(np.linalg.norm(g["velocity"] - r["velocity"]))
    return {"x": x_err, "v": dv / v_ref, "v_norm": v_ref, "n": len(g["id"])}


def ledger_errors(lg, lr) -> dict:
    out = {}
    for f in ("gravity_impulse", "wall_impulse"):
        a, b = np.array(getattr(lg, f)), np.array(getattr(lr, f))
        out[f] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    for f in ("wall_normal_projection_energy", "wall_friction_dissipation", "wall_normal_traction_energy",
              "plastic_dissipation"):
        a, b = getattr(lg, f), getattr(lr, f)
        out[f] = abs(a - b) / max(abs(b), 1e-300) if b != 0.0 else abs(a)
    return out


def check_ledgers(err: dict, lr) -> None:
    for f in ("gravity_impulse", "wall_impulse"):
        assert err[f] <= 1e-5, (f, err[f])
    for f in ("wall_normal_projection_energy", "wall_friction_dissipation", "wall_normal_traction_energy",
              "plastic_dissipation"):
        if getattr(lr, f) != 0.0:
            assert err[f] <= 1e-4, (f, err[f])


def oracle_run(spec, steps: int):
    import oracle

    ref = oracle.OracleSim(spec, threads=oracle.threads_available())
    ref.advance_to(steps * spec.max_dt)
    return ref


def gpu_run(spec, steps: int, weights=None):
    from litter_physics_b200.sim import Simulation

    sim = Simulation(spec)
    sim.set_warm_start(weights)
    sim.advance_to(steps * spec.max_dt)
    return sim


def check_pair(sim, ref, spec, label: str) -> dict:
    d = particle_errors(sim.particles(), ref.particles(), max(spec.domain))
    gc, rc = sim.counters, ref.counters()
    led = ledger_errors(sim.ledger, ref.ledger())
    print(label, d, led, "steps", gc.step_count, "rejected", gc.rejected_steps,
          "newton", gc.newton_iterations, "yielded", gc.yielded_particles)
    assert gc.step_count == rc.step_count and gc.rejected_steps == rc.rejected_steps
    assert d["x"] <= POS_TOL, (label, d)
    assert d["v"] <= VEL_TOL, (label, d)
    check_ledgers(led, ref.ledger())
    return d


def test_plain_slump_full_size_matches_oracle(lib_built):
    """64^3 grid, 65,536 particles (the plain HB slump configuration)."""
    from litter_physics_b200 import configs

    spec = configs.config0()
    ref = oracle_run(spec, STEPS)
    sim = gpu_run(spec, STEPS)
    assert sim.particle_count() == 65_536
    check_pair(sim, ref, spec, "slump 64^3")


def test_dam_break_full_size_matches_oracle(lib_built):
    """128^3 grid, 1,048,576 particles, Tait gamma 7 (the liquid dam-break configuration)."""
    from litter_physics_b200 import configs

    spec = configs.config1()
    ref = oracle_run(spec, STEPS)
    sim = gpu_run(spec, STEPS)
    assert sim.particle_count() == 1_048_576
    check_pair(sim, ref, spec, "dam break 128^3")


@pytest.fixture(scope="module")
def trained_weights(lib_built):
    """Network trained by the device kernels on Newton pairs a small slump logs."""
    from litter_physics_b200 import configs, warmstart
    from litter_physics_b200.sim import Simulation

    sim = Simulation(configs.slump(32, (8, 8, 16), seed=3, yield_range=(20.0, 100.0)))
    raw, sigma = warmstart.collect(sim, 150, capacity=1_000_000)
    sim.close()
    x, y = warmstart.dataset(raw, sigma)
    w, loss = warmstart.train(x, y, epochs=20, batch=1024, lr=2e-3)
    assert loss < 0.05
    return w


def test_large_slump_sample_plain_and_warm_match_oracle(lib_built, trained_weights):
    """256^3 grid spacing, per-particle yield stress U(20, 100) Pa, 262,144 particles: the plain
    Newton and the learned warm start both meet the bars against one oracle run, and the warm
    start takes fewer Newton iterations."""
    from litter_physics_b200 import configs

    spec = configs.slump(256, (32, 32, 32), seed=2, yield_range=(20.0, 100.0))
    ref = oracle_run(spec, STEPS)
    it = {}
    for name, w in (("plain", None), ("warm", trained_weights)):
        sim = gpu_run(spec, STEPS, w)
        assert sim.particle_count() == 262_144
        check_pair(sim, ref, spec, f"large-slump sample {name}")
        it[name] = sim.counters.newton_iterations
        assert sim.counters.yielded_particles > 0
        sim.close()
    assert it["warm"] < it["plain"]


def test_sweep_members_in_one_batch_match_oracle(lib_built):
    """The first eight calibration-sweep instances (35k-110k particles, own grids and materials)
    advanced together in one batch; each member against its own oracle run."""
    from litter_physics_b200 import configs
    from litter_physics_b200.sim import Batch

    specs = configs.config3()[:8]
    batch = Batch(specs)
    batch.advance_to(STEPS * 1e-4)
    for i, spec in enumerate(specs):
        ref = oracle_run(spec, STEPS)
        d = particle_errors(batch.particles(i), ref.particles(), max(spec.domain))
        bc, rc = batch.counters(i), ref.counters()
        led = ledger_errors(batch.ledger(i), ref.ledger())
        print(f"sweep member {i}", d, led, "steps", bc.step_count, "yielded", bc.yielded_particles)
        assert bc.step_count == rc.step_count and bc.rejected_steps == rc.rejected_steps
        assert d["x"] <= POS_TOL, (i, d)
        assert d["v"] <= VEL_TOL, (i, d)
        check_ledgers(led, ref.ledger())
        ref.close()
    batch.close()
