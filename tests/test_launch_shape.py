"""Launch shapes and the autotuner: every shape of the persistent tile kernels gives the same
particle state bit for bit (a tile's results do not depend on the CTA that takes it, on the
order, on the G2P block size or on the P2G chunk size), and the autotuner leaves the state
as it found it.  The ledgers are identical too, except that the G2P block size changes which
thread sums which particles' FP64 plastic work, so with 128-thread CTAs that one ledger entry
agrees to rounding."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [
    {},  # default: 256-thread G2P, 1024-particle P2G chunks, as many CTAs as fit, dynamic tiles
    {"dynamic_tiles": 0},
    {"g2p_variant": 1},
    {"g2p_variant": 1, "g2p_per_sm": 3},
    {"g2p_variant": 2},
    {"g2p_variant": 3},
    {"p2g_variant": 1},
    {"p2g_variant": 2},
    {"p2g_variant": 2, "dynamic_tiles": 0},
    {"p2g_per_sm": 1, "g2p_per_sm": 1, "dynamic_tiles": 0},
    {"graph_attempts": 4},
]


def by_id(p: dict) -> dict:
    order = np.argsort(p["id"])
    return {k: v[order] for k, v in p.items()}


def run(specs_fn, shape: dict, steps: int):
    from litter_physics_b200.sim import Batch

    b = Batch(specs_fn())
    if shape:
        b.set_launch_shape(**shape)
    b.run_substeps(steps)
    b.sync()
    out = []
    for i in range(len(b.specs)):
        p = by_id(b.particles(i))
        led = b.ledger(i)
        plastic = led.plastic_dissipation
        led.plastic_dissipation = 0.0
        out.append(((p["position"].tobytes(), p["velocity"].tobytes(), p["deformation"].tobytes(), bytes(led),
                     b.counters(i).step_count), plastic))
    b.close()
    return out


def uneven_batch():
    from litter_physics_b200 import configs

    # one fixture kind per batch: three slumps of uneven size, one with per-particle yield stress
    return [configs.slump(16, (4, 4, 8), seed=21), configs.slump(32, (8, 8, 16), seed=22, yield_range=(20.0, 100.0)),
            configs.slump(24, (6, 6, 12), seed=23)]


def liquid_batch():
    from litter_physics_b200 import configs

    return [configs.dam_break(32, (16, 8, 16), seed=23), configs.dam_break(24, (12, 6, 12), seed=24)]


def test_every_launch_shape_gives_identical_results():
    from litter_physics_b200 import _lib

    _lib.build()
    for batch in (uneven_batch, liquid_batch):
        ref = run(batch, SHAPES[0], 24)
        for shape in SHAPES[1:]:
            got = run(batch, shape, 24)
            for (state, plastic), (ref_state, ref_plastic) in zip(got, ref, strict=True):
                assert state == ref_state, shape
                if shape.get("g2p_variant"):
                    assert abs(plastic - ref_plastic) <= 1e-13 * abs(ref_plastic), shape
                else:
                    assert plastic == ref_plastic, shape


def test_launch_shape_round_trip_and_refusal():
    from litter_physics_b200 import _lib, configs
    from litter_physics_b200.sim import Simulation

    _lib.build()
    sim = Simulation(configs.slump(16, (4, 4, 8), seed=1))
    sim.set_launch_shape(g2p_variant=1, p2g_variant=1, dynamic_tiles=0, graph_attempts=4)
    s = sim.launch_shape()
    assert (s["g2p_variant"], s["p2g_variant"], s["dynamic_tiles"], s["graph_attempts"]) == (1, 1, 0, 4)
    assert s["g2p_per_sm"] >= 1 and s["p2g_per_sm"] >= 1
    # a new block shape without its CTAs per SM takes as many as fit it (4 of 128 threads on a B200)
    wide = Simulation(configs.slump(16, (4, 4, 8), seed=1))
    base = wide.launch_shape()["g2p_per_sm"]
    wide.set_launch_shape(g2p_variant=1)
    assert wide.launch_shape()["g2p_per_sm"] >= 2 * base
    wide.close()
    with pytest.raises(_lib.LPError):
        sim.set_launch_shape(g2p_variant=4)
    sim.close()


def test_return_share_measurement_steps_like_the_solver():
    """The clock-instrumented G2P used to measure the return's share of G2P time takes the same
    steps as the solver's G2P, and the share is a fraction."""
    from litter_physics_b200 import _lib, configs
    from litter_physics_b200.sim import Simulation

    _lib.build()
    spec = configs.slump(32, (8, 8, 16), seed=4, yield_range=(20.0, 100.0))
    a, b = Simulation(spec), Simulation(spec)
    a.run_substeps(30)
    b.run_substeps(20)
    share = b.g2p_return_share(10)
    a.sync()
    b.sync()
    assert 0.0 < share < 1.0
    pa, pb = by_id(a.particles()), by_id(b.particles())
    assert np.array_equal(pa["position"], pb["position"]) and np.array_equal(pa["deformation"], pb["deformation"])
    liquid = Simulation(configs.dam_break(32, (16, 8, 16), seed=1))
    assert liquid.g2p_return_share(3) == 0.0


def test_autotuner_picks_a_shape_on_the_live_batch():
    """The autotuner times every candidate from the same state (a device copy put back before
    each candidate) and leaves the batch where it found it: the same particles, ledgers and
    counters, and a continuation that matches an untuned run."""
    from litter_physics_b200 import _lib
    from litter_physics_b200.sim import Batch

    _lib.build()
    b = Batch(uneven_batch())
    b.run_substeps(6)
    b.sync()
    before = [(by_id(b.particles(i)), bytes(b.ledger(i)), b.counters(i).step_count, b.counters(i).time)
              for i in range(3)]
    report = b.autotune(4)
    lines = report.strip().splitlines()
    assert lines[-1].startswith("chosen: ") and len(lines) >= 8
    chosen = b.launch_shape()
    assert chosen["g2p_per_sm"] >= 1 and chosen["graph_attempts"] >= 1
    b.sync()
    for i, (p, led, steps, t) in enumerate(before):
        q = by_id(b.particles(i))
        for k in ("position", "velocity", "deformation", "kirchhoff"):
            assert np.array_equal(p[k], q[k]), (i, k)
        assert bytes(b.ledger(i)) == led
        assert b.counters(i).step_count == steps and b.counters(i).time == t
    ref = Batch(uneven_batch())
    ref.run_substeps(14)
    b.run_substeps(8)
    for i in range(3):
        assert np.array_equal(by_id(b.particles(i))["position"], by_id(ref.particles(i))["position"])
    ref.close()
    b.close()


def test_mixed_material_batch_matches_single_kind_runs():
    """A batch that mixes a paste and a liquid instance runs the mixed-kind G2P; each member
    matches the same instance run alone (which runs the paste-only or liquid-only G2P) bit for
    bit."""
    from litter_physics_b200 import _lib, configs
    from litter_physics_b200.sim import Batch, Simulation

    _lib.build()
    paste = configs.slump(16, (4, 4, 8), seed=31)
    liquid = configs.slump(16, (4, 4, 8), seed=32)
    liquid.material = configs.dam_break(16, (4, 4, 8)).material
    specs = [paste, liquid]
    b = Batch(specs)
    b.run_substeps(20)
    b.sync()
    for i, spec in enumerate(specs):
        one = Simulation(spec)
        one.run_substeps(20)
        one.sync()
        pb, ps = by_id(b.particles(i)), by_id(one.particles())
        assert b.counters(i).step_count == one.counters.step_count
        for k in ("position", "velocity", "deformation", "volume_ratio"):
            assert np.array_equal(pb[k], ps[k]), (i, k)
        one.close()
    b.close()


def test_prepared_graph_runs_like_the_graph_captured_on_first_use():
    """lp_batch_prepare builds the attempt graph without launching anything: the state, ledgers
    and counters after a prepared run equal those of a run whose graph is captured on first use,
    and both count the same kernel launches."""
    from litter_physics_b200 import _lib
    from litter_physics_b200.sim import Batch

    results, launches = [], []
    for prepare in (False, True):
        b = Batch(uneven_batch())
        b.set_launch_shape(graph_attempts=4)
        if prepare:
            b.prepare()
            b.sync()
            assert b.counters(0).step_count == 0  # nothing ran
            b.prepare()  # already built: a no-op
        l0 = _lib.kernel_launches()
        b.run_substeps(10)
        b.sync()
        launches.append(_lib.kernel_launches() - l0)
        results.append([(by_id(b.particles(i))["position"].tobytes(), bytes(b.ledger(i)), b.counters(i).step_count)
                        for i in range(len(b.specs))])
        b.close()
    assert results[0] == results[1]
    assert launches[0] == launches[1] > 0
