"""Benchmark workloads as fixture specs.

Material parameters follow the reference's wire convention (research.rs:274-305): yield
stress and consistency are shear-rheometer values converted to the von Mises form by
`Material::paste_from_shear_rheology` (constitutive.rs:180-197).  Young's modulus and
Poisson's ratio are derived from the stated shear and bulk moduli.  Extensions used here
(labelled in the spec): per-face wall friction with a sticky floor, per-particle yield stress,
the Tait EOS exponent, and the Newton tolerance.
"""

from __future__ import annotations

import math

from . import _abi
from .research import base_spec, material_liquid, material_paste_shear


def young_poisson(shear: float, bulk: float) -> tuple[float, float]:
    e = 9.0 * bulk * shear / (3.0 * bulk + shear)
    nu = (3.0 * bulk - 2.0 * shear) / (2.0 * (3.0 * bulk + shear))
    return e, nu


def _sticky_floor_slip_walls(s: _abi.FixtureSpec) -> None:
    s.face_mode_enabled = 1
    for f in range(6):
        s.face_friction[f] = 0.0
        s.face_sticky[f] = 0
    s.face_sticky[4] = 1  # floor: axis 2, low face


def slump(cells: int = 64, column=(16, 16, 32), seed: int = 0, yield_range=None, newton_tol: float = 1e-10,
          dt: float = 1e-4, domain_m: float = 1.0) -> _abi.FixtureSpec:
    """HB paste slump: rho 1200, G 2e4, K 1e5, tau_y 50, K_s 5, n 0.5, sticky floor, slip walls."""
    dx = domain_m / cells
    e, nu = young_poisson(2e4, 1e5)
    s = base_spec(fixture=_abi.LP_SLUMP, grid_spacing=dx, domain=[domain_m] * 3,
                  initial_size=[c * dx for c in column], initial_velocity=[0, 0, 0], seed=seed,
                  wall_friction=0.0, max_dt=dt, min_dt=1e-12, contact_stiffness=1000.0,
                  contact_restitution=0.2, contact_friction=0.4, max_particles=2**31 - 1, max_nodes=2**40)
    s.material = material_paste_shear(1200.0, e, nu, 50.0, 5.0, 0.5)
    _sticky_floor_slip_walls(s)
    s.newton_tolerance = newton_tol
    if yield_range is not None:
        s.yield_random = 1
        s.yield_min = math.sqrt(3.0) * yield_range[0]
        s.yield_max = math.sqrt(3.0) * yield_range[1]
    return s


def config0() -> _abi.FixtureSpec:
    """64^3 grid, 16x16x32-cell column, 65,536 particles, seed 0, dt 1e-4, 500 substeps."""
    return slump(64, (16, 16, 32), seed=0)


def config2() -> _abi.FixtureSpec:
    """256^3 grid, 128^3-cell column, ~16.8M particles, seed 2, yield U(20, 100) per particle."""
    return slump(256, (128, 128, 128), seed=2, yield_range=(20.0, 100.0))


def dam_break(cells: int = 128, block=(64, 32, 64), seed: int = 1, gamma: float = 7.0,
              dt: float = 5e-5) -> _abi.FixtureSpec:
    """Weakly compressible water dam break: rho 1000, K 2e5, Tait gamma, eta 1e-3, slip walls."""
    dx = 1.0 / cells
    bulk = 2e5
    nu = 0.2
    e = 3.0 * bulk * (1.0 - 2.0 * nu)
    s = base_spec(fixture=_abi.LP_DAM_BREAK, grid_spacing=dx, domain=[1.0] * 3,
                  initial_size=[b * dx for b in block], initial_velocity=[0, 0, 0], seed=seed,
                  wall_friction=0.0, max_dt=dt, min_dt=1e-12, contact_stiffness=1000.0,
                  contact_restitution=0.2, contact_friction=0.4, max_particles=2**31 - 1, max_nodes=2**40)
    s.material = material_liquid(1000.0, e, nu, 1e-3, tait_gamma=gamma)
    return s


def config1() -> _abi.FixtureSpec:
    """128^3 grid, 64x32x64-cell water block, ~1.05M particles, seed 1, dt <= 5e-5, 2000 substeps."""
    return dam_break()


def sweep_instance(k: int, rng) -> _abi.FixtureSpec:
    """One member of the batched calibration sweep (seed 100 + k).

    Particle count log-uniform in 8k-260k: a column of a x a x 2a cells at 8 particles per cell
    (16 a^3 particles) in a cubic domain 1.5 times the column height (3a cells), dx = 1 cm.
    Yield U(10, 200) Pa, consistency U(1, 20) Pa s^n, flow index U(0.3, 1.0), shear modulus
    U(5e3, 5e4) Pa (bulk modulus 1e5 Pa), rho 1200, sticky floor and slip walls, dt 1e-4.
    """
    n_target = math.exp(rng.uniform(math.log(8_000), math.log(260_000)))
    a = max(2, round((n_target / 16.0) ** (1.0 / 3.0)))
    cells = 3 * a
    dx = 0.01
    shear = rng.uniform(5e3, 5e4)
    e, nu = young_poisson(shear, 1e5)
    s = base_spec(fixture=_abi.LP_SLUMP, grid_spacing=dx, domain=[cells * dx] * 3,
                  initial_size=[a * dx, a * dx, 2 * a * dx], initial_velocity=[0, 0, 0], seed=100 + k,
                  wall_friction=0.0, max_dt=1e-4, min_dt=1e-12, contact_stiffness=1000.0,
                  contact_restitution=0.2, contact_friction=0.4, max_particles=2**31 - 1, max_nodes=2**40)
    s.material = material_paste_shear(1200.0, e, nu, rng.uniform(10.0, 200.0), rng.uniform(1.0, 20.0),
                                      rng.uniform(0.3, 1.0))
    _sticky_floor_slip_walls(s)
    s.newton_tolerance = 1e-10
    return s


def config3(count: int = 256, seed: int = 2024) -> list[_abi.FixtureSpec]:
    """256 independent HB slumps of uneven size (seeds 100-355), 300 substeps each."""
    import random

    rng = random.Random(seed)
    return [sweep_instance(k, rng) for k in range(count)]


def pellet_bed(cells: int = 128, layer_cells: int = 8, pellets: int = 512, seed: int = 7, dt: float = 5e-5,
               domain_m: float = 1.0, young: float = 5e6, region=None, gravity: float = -9.81,
               law: str = "hertz_mindlin", dem_stiffness: float = 1000.0, dem_rolling: float = 0.05) -> _abi.FixtureSpec:
    """Config 4 (extension): an HB paste layer with config-0 material under a bed of rigid pine pellets.

    Paste: a full-width layer `layer_cells` cells thick at 8 particles per cell (128 x 128 x 8
    cells = 1,048,576 particles at the defaults), sticky floor and slip walls.  Pellets: radius
    3 mm, length 20 mm, density 650 kg/m^3 -- 6 spheres by the reference's count rule
    (rigid.rs:147-160), where the config text says 5 -- with random orientations and
    non-overlapping centres drawn from `seed` in the slab 1-6 cm above the layer.  Pellet-pellet
    contact is Hertz-Mindlin with friction 0.5, restitution 0.3, Poisson 0.3 and a softened
    Young's modulus (5 MPa: the contact time stays above ten steps of 5e-5 s); pellet-wall
    contact is the reference's spring-dashpot.  The config's 3 mm radius is below the
    reference's 1.5 dx resolution rule for the coupled patch (dx = 7.8 mm), which the bed does
    not apply.

    `law="linear"` replaces Hertz-Mindlin by the household DEM's contact law (dem.rs:789-834):
    a linear spring-dashpot of `dem_stiffness` N/m (1000 N/m keeps the reference's stable step
    0.1 sqrt(m/k) above 5e-5 s), a tangential spring of 2/7 of it with Coulomb sliding, and
    rolling resistance `dem_rolling`, with the same friction and restitution.
    """
    dx = domain_m / cells
    e, nu = young_poisson(2e4, 1e5)
    top = layer_cells * dx
    s = base_spec(fixture=_abi.LP_SLUMP, grid_spacing=dx, domain=[domain_m] * 3,
                  initial_size=[domain_m, domain_m, top], initial_velocity=[0, 0, 0], seed=seed,
                  wall_friction=0.0, max_dt=dt, min_dt=1e-12, contact_stiffness=1000.0,
                  contact_restitution=0.2, contact_friction=0.4, max_particles=2**31 - 1, max_nodes=2**40)
    s.gravity[:] = [0.0, 0.0, gravity]
    s.material = material_paste_shear(1200.0, e, nu, 50.0, 5.0, 0.5)
    _sticky_floor_slip_walls(s)
    s.newton_tolerance = 1e-10
    s.has_pellet = 1
    s.pellet_radius, s.pellet_length, s.pellet_density = 0.003, 0.020, 650.0
    s.bed_count = pellets
    s.bed_seed = seed
    lo, hi = region if region is not None else ([0.02, 0.02, top + 0.01], [domain_m - 0.02, domain_m - 0.02,
                                                                              top + 0.06])
    s.bed_lo[:] = list(lo)
    s.bed_hi[:] = list(hi)
    s.hm_young, s.hm_poisson, s.hm_friction, s.hm_restitution = young, 0.3, 0.5, 0.3
    if law == "linear":
        s.bed_law, s.dem_stiffness, s.dem_rolling = _abi.LP_BED_LINEAR, dem_stiffness, dem_rolling
    elif law != "hertz_mindlin":
        raise ValueError(f"unknown contact law '{law}'")
    return s


def config4() -> _abi.FixtureSpec:
    """Coupled pellet bed: 128^3 grid, ~1M paste particles, 512 pellets, seed 7, dt 5e-5 s."""
    return pellet_bed()

