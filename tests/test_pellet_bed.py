"""Pellet bed (config 4 extension): many multisphere pellets coupled to the grid, with
Hertz-Mindlin sphere contact between pellets.

CPU tests check the oracle's model on its own: placement invariants, and a head-on collision
in free space (restitution close to the requested coefficient, momentum conserved, the
contact work equal to the kinetic energy lost).  GPU tests check the device path against the
oracle: identical placement, the same collision, and a small bed falling onto a paste layer."""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest


def small_bed(pellets: int = 24, gravity: float = -9.81, region=None, law: str = "hertz_mindlin"):
    """Config-4 geometry at 7.8 mm cells on a 32^3 grid (0.25 m), a 2-cell paste layer."""
    from litter_physics_b200 import configs

    dx = 0.25 / 32
    top = 2 * dx
    if region is None:
        region = ([0.095, 0.095, top + 0.004], [0.155, 0.155, top + 0.03])
    return configs.pellet_bed(cells=32, layer_cells=2, pellets=pellets, domain_m=0.25, region=region,
                              gravity=gravity, law=law)


def sphere_centres(p) -> np.ndarray:
    i, j, k, w = p.orientation
    ax = np.array([1 - 2 * (j * j + k * k), 2 * (i * j + w * k), 2 * (i * k - w * j)])
    return np.array([np.array(p.position[:]) + ax * p.sphere_offsets[s] for s in range(p.sphere_count)])


def collision_pair(pellets: list, speed: float = 0.1) -> list:
    """Two pellets along x, end to end 1 mm apart, approaching at +-speed; the others far away."""
    out = []
    for n, p in enumerate(pellets):
        q = type(p)()
        C.memmove(C.byref(q), C.byref(p), C.sizeof(p))
        q.orientation[:] = [0.0, 0.0, 0.0, 1.0]
        q.angular_momentum[:] = [0.0, 0.0, 0.0]
        if n == 0:
            q.position[:] = [0.100, 0.050, 0.150]
            q.velocity[:] = [speed, 0.0, 0.0]
        elif n == 1:
            q.position[:] = [0.100 + 0.021, 0.050, 0.150]
            q.velocity[:] = [-speed, 0.0, 0.0]
        else:
            q.position[:] = [0.03 + 0.025 * (n % 8), 0.20, 0.05 + 0.03 * (n // 8)]
            q.velocity[:] = [0.0, 0.0, 0.0]
        out.append(q)
    return out


def momentum(pellets) -> np.ndarray:
    return sum(np.array(p.velocity[:]) * p.mass for p in pellets)


# ---------------------------------------------------------------------------- CPU (oracle)
def test_placement_is_deterministic_inside_and_non_overlapping():
    import oracle

    spec = small_bed(pellets=64, region=([0.02, 0.02, 0.03], [0.23, 0.23, 0.2]))
    a = oracle.OracleSim(spec).pellets()
    b = oracle.OracleSim(spec).pellets()
    assert len(a) == 64
    r = a[0].radius
    allc = []
    for pa, pb in zip(a, b):
        assert list(pa.position) == list(pb.position) and list(pa.orientation) == list(pb.orientation)
        assert abs(math.sqrt(sum(v * v for v in pa.orientation)) - 1.0) < 1e-14
        c = sphere_centres(pa)
        assert (c >= r - 1e-12).all() and (c <= 0.25 - r + 1e-12).all()
        allc.append(c)
    assert a[0].sphere_count == 6  # rigid.rs:147-160 for r = 3 mm, L = 20 mm
    for i in range(len(allc)):
        for j in range(i):
            d = np.linalg.norm(allc[i][:, None, :] - allc[j][None, :, :], axis=2)
            assert d.min() >= 2.02 * r - 1e-12


LAWS = ["hertz_mindlin", "linear"]


@pytest.mark.parametrize("law", LAWS)
def test_head_on_collision_restitution_momentum_and_work(law):
    """Both contact laws: restitution within the household DEM's bounds for a clamped dashpot
    (dem.rs:981-1021: e - 0.02 to e + 0.15; Hertz-Mindlin lands at 0.301)."""
    import oracle

    spec = small_bed(pellets=4, gravity=0.0, law=law)
    sim = oracle.OracleSim(spec)
    start = collision_pair(sim.pellets())
    sim.set_pellets(start)
    ke0 = sum(0.5 * p.mass * sum(v * v for v in p.velocity) for p in start)
    sim.advance_to(0.015)
    end = sim.pellets()
    vrel0 = start[1].velocity[0] - start[0].velocity[0]
    vrel1 = end[1].velocity[0] - end[0].velocity[0]
    e = -vrel1 / vrel0
    print("restitution", e)
    assert 0.3 - 0.02 <= e <= 0.3 + (0.05 if law == "hertz_mindlin" else 0.15)
    p0, p1 = momentum(start), momentum(end)
    assert np.linalg.norm(p1 - p0) <= 1e-15 * max(np.linalg.norm([s.mass * 0.1 for s in start]), 1e-30)
    ke1 = sum(0.5 * p.mass * sum(v * v for v in p.velocity) for p in end)
    obs = sim.observables()
    # the contact work (force times the step's mean velocity) is the kinetic energy the
    # collision removed: exact for the explicit update up to rounding
    assert obs["pellet_contacts"] == 0.0
    assert abs((ke1 - ke0) - obs["pellet_contact_work_j"]) <= 1e-9 * ke0


def _rot(q):
    i, j, k, w = q
    return np.array([[w * w + i * i - j * j - k * k, 2 * (i * j - w * k), 2 * (w * j + i * k)],
                     [2 * (w * k + i * j), w * w - i * i + j * j - k * k, 2 * (j * k - w * i)],
                     [2 * (i * k - w * j), 2 * (w * i + j * k), w * w - i * i - j * j + k * k]])


def _omega(p):
    R = _rot(p.orientation)
    return R @ ((R.T @ np.array(p.angular_momentum[:])) / np.array(p.inertia_body[:]))


def linear_contact_reference(pa, pb, params, dt):
    """`World::contact_force` and `pellet_pair_force` (dem.rs:651-704, 789-834) written out
    for every sphere pair of pellet a (first body) against pellet b, with empty tangential
    history: the force and torque on a.  params = (k_n, friction, restitution, rolling)."""
    kn, mu, e, mur = params
    lnE = math.log(e)
    zeta = min(-lnE / math.sqrt(math.pi**2 + lnE * lnE), 1.0)
    xa, xb = np.array(pa.position[:]), np.array(pb.position[:])
    ax_a, ax_b = _rot(pa.orientation)[:, 0], _rot(pb.orientation)[:, 0]
    wa, wb = _omega(pa), _omega(pb)
    va, vb = np.array(pa.velocity[:]), np.array(pb.velocity[:])
    mstar = pa.mass * pb.mass / (pa.mass + pb.mass)
    force, torque = np.zeros(3), np.zeros(3)
    for i in range(pa.sphere_count):
        ca = xa + ax_a * pa.sphere_offsets[i]
        for j in range(pb.sphere_count):
            cb = xb + ax_b * pb.sphere_offsets[j]
            offset = ca - cb
            dist = np.linalg.norm(offset)
            overlap = pa.radius + pb.radius - dist
            if overlap <= 0.0:
                continue
            n = offset / dist
            point = ca - n * (pa.radius - 0.5 * overlap)
            rel = (va + np.cross(wa, point - xa)) - (vb + np.cross(wb, point - xb))
            radius = pa.radius * pb.radius / (pa.radius + pb.radius)
            vn = rel @ n
            cn = 2.0 * zeta * math.sqrt(kn * mstar)
            fn = max(kn * overlap - cn * vn, 0.0)
            vt = rel - n * vn
            xi = vt * dt
            ft = -(xi * (2.0 / 7.0) * kn) - vt * math.sqrt(2.0 / 7.0) * cn
            if np.linalg.norm(ft) > mu * fn:
                ft = ft * (mu * fn / np.linalg.norm(ft))
            wrel = wa - wb
            roll = -wrel / np.linalg.norm(wrel) * (mur * radius * fn)
            f = n * fn + ft
            force += f
            torque += np.cross(point - xa, f) + roll
    return force, torque


def test_linear_law_force_and_torque_match_the_household_dem_formulas():
    """One step of two spinning, sliding, overlapping pellets away from walls and paste: the
    oracle's velocity and angular-momentum changes are the household DEM's contact force and
    torque (normal dashpot, tangential spring and damper, Coulomb cap, rolling resistance)
    times dt, to 1e-12."""
    import oracle

    spec = small_bed(pellets=4, gravity=0.0, law="linear")
    sim = oracle.OracleSim(spec)
    start = collision_pair(sim.pellets(), speed=0.02)
    start[1].position[:] = [0.100 + 0.0195, 0.0502, 0.1501]  # end spheres overlap about 0.5 mm, offset
    start[0].angular_momentum[:] = [1e-9, -2e-9, 3e-9]
    start[1].angular_momentum[:] = [-2e-9, 1e-9, 0.5e-9]
    start[0].velocity[:] = [0.02, 0.01, -0.005]
    sim.set_pellets(start)
    dt = 2e-5
    ok, why = sim.try_step(dt)
    assert ok, why
    end = sim.pellets()
    params = (spec.dem_stiffness, spec.hm_friction, spec.hm_restitution, spec.dem_rolling)
    for a, b in ((0, 1), (1, 0)):
        f, t = linear_contact_reference(start[a], start[b], params, dt)
        dv = (np.array(end[a].velocity[:]) - np.array(start[a].velocity[:])) * start[a].mass / dt
        dl = (np.array(end[a].angular_momentum[:]) - np.array(start[a].angular_momentum[:])) / dt
        print(a, f, dv, t, dl)
        assert np.abs(f).max() > 0.0 and np.abs(t).max() > 0.0
        assert np.linalg.norm(dv - f) <= 1e-9 * np.linalg.norm(f)
        assert np.linalg.norm(dl - t) <= 1e-9 * np.linalg.norm(t)


# ---------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def built():
    from litter_physics_b200 import _lib

    _lib.build()
    return _lib


def pellet_arrays(ps) -> dict:
    return {k: np.array([list(getattr(p, k)) for p in ps]) for k in ("position", "velocity", "angular_momentum",
                                                                       "orientation")}


@pytest.mark.gpu
def test_gpu_placement_matches_oracle(built):
    import oracle

    from litter_physics_b200.sim import Simulation

    spec = small_bed(pellets=64, region=([0.02, 0.02, 0.03], [0.23, 0.23, 0.2]))
    g = pellet_arrays(Simulation(spec).pellets())
    r = pellet_arrays(oracle.OracleSim(spec).pellets())
    assert np.array_equal(g["position"], r["position"])
    assert np.array_equal(g["orientation"], r["orientation"])


@pytest.mark.gpu
@pytest.mark.parametrize("law", LAWS)
def test_gpu_collision_matches_oracle(built, law):
    """The same head-on collision on the device: pellet states agree with the FP64 oracle to
    1e-12 relative (pellet arithmetic is FP64 on both sides), the contact work to 1e-9."""
    import oracle

    from litter_physics_b200.sim import Simulation

    spec = small_bed(pellets=4, gravity=0.0, law=law)
    ref = oracle.OracleSim(spec)
    gpu = Simulation(spec)
    start = collision_pair(ref.pellets())
    ref.set_pellets(start)
    gpu.set_pellets(start)
    ref.advance_to(0.015)
    gpu.advance_to(0.015)
    g, r = pellet_arrays(gpu.pellets()), pellet_arrays(ref.pellets())
    for k in g:
        scale = max(np.abs(r[k]).max(), 1e-30)
        print(k, np.abs(g[k] - r[k]).max() / scale)
        assert np.abs(g[k] - r[k]).max() <= 1e-12 * scale, k
    go, ro = gpu.observables(), ref.observables()
    assert abs(go["pellet_contact_work_j"] - ro["pellet_contact_work_j"]) <= 1e-9 * abs(ro["pellet_contact_work_j"])
    assert go["step_count"] == ro["step_count"]


@pytest.mark.gpu
@pytest.mark.parametrize("law", LAWS)
def test_gpu_bed_falling_on_paste_matches_oracle(built, law):
    """24 pellets dropped onto a 2-cell paste layer for 0.04 s (800 substeps): pellet and paste
    positions within 1e-5 of the domain, the coupling and contact energies within 1e-3 of the
    pellets' kinetic-energy scale (FP32 paste state on the device against FP64), and momentum
    closed to 1e-6 of the gravity impulse."""
    import oracle

    from litter_physics_b200.sim import Simulation

    spec = small_bed(law=law)
    ref = oracle.OracleSim(spec)
    gpu = Simulation(spec)
    t = 0.04
    ref.advance_to(t)
    gpu.advance_to(t)
    g, r = pellet_arrays(gpu.pellets()), pellet_arrays(ref.pellets())
    L = max(spec.domain)
    dxp = np.abs(g["position"] - r["position"]).max() / L
    print("pellet position error / L", dxp)
    pg, pr = gpu.particles(), ref.particles()
    og, orr = np.argsort(pg["id"]), np.argsort(pr["id"])
    dxq = np.abs(pg["position"][og] - pr["position"][orr]).max() / L
    print("paste position error / L", dxq)
    go, ro = gpu.observables(), ref.observables()
    scale = max(ro["pellet_kinetic_energy_j"], 1e-12)
    bad = []
    for k in ("pellet_contact_work_j", "coupling_grid_energy_j", "coupling_pellet_energy_j", "pellet_kinetic_energy_j"):
        print(k, go[k], ro[k])
        if not abs(go[k] - ro[k]) <= 1e-3 * scale:
            bad.append(k)
    assert dxp <= 1e-5
    assert dxq <= 1e-5
    assert not bad, bad
    assert ro["pellet_contact_work_j"] < 0.0  # contacts happened
    assert go["step_count"] == ro["step_count"] and go["rejected_steps"] == ro["rejected_steps"]
    # momentum closes to FP32 rounding of the particle velocities (1e-6 of the gravity impulse)
    impulse = (sum(p.mass for p in gpu.pellets()) + float(pg["mass"].sum())) * 9.81 * t
    assert abs(go["momentum_residual_kg_m_s"]) <= 1e-6 * impulse
