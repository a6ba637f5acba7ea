"""Synthetic seeded scenes for the plain-path workloads.

The reference samples its scenes from SDF/OBJ assets that are not shipped
(LoadSample.cpp:109-176); these scenes stand in for them with the sizes and
parameters of the benchmark configurations:

* ``notched_bar``  — 16x16x64 cells at dx=1/128, 8 particles per cell
  (131,072 before the notch), pulled apart at +/-0.5 m/s at both ends.
* ``plates``       — 4 stacked plates of 256x256x16 cells at dx=1/256, 8 ppc
  (33,554,432 particles), sphere impactor r=0.1 at 5 m/s, gravity -9.8.
* ``plates_8m``    — the same scene at 8,388,608 particles: 4 plates of
  128x128x16 cells at dx=1/128 with 8 ppc.
* ``notched_bar_batch`` — independent notched bars for batched stepping:
  particle counts log-uniform in [10k, 500k], material parameters uniform
  within +/-50% of the notched bar's, pull speed uniform in [0.2, 1.0] m/s,
  FP32 with the FP64 SVD fallback.

Material parameters follow the configurations: rho=1000, E=1e5 (per plate
log-uniform in [5e4, 5e5] for the plate scenes), nu=0.3, yield 200 Pa with
linear hardening H=0.1E, phase-field length scale L0=2dx, softening onset at
equivalent plastic strain 0.05 (the reference compares alpha/2 with ps, so
ps=0.025), and the reference's remaining fracture constants.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import gmpm as G


@dataclasses.dataclass
class SceneSpec:
    name: str
    desc: G.SceneDesc
    positions: np.ndarray
    masses: np.ndarray
    velocities: np.ndarray
    material_ids: np.ndarray
    substeps: int

    @property
    def n(self) -> int:
        return len(self.positions)

    def build(self, ctx: G.Context) -> G.Scene:
        return G.Scene(ctx, self.desc, self.positions, self.masses, self.velocities, self.material_ids)


def config_material(m: G.Material, dx: float, E: float = 1e5) -> None:
    m.youngs_modulus = E
    m.poisson_ratio = 0.3
    m.density = 1000.0
    m.yield_stress = 200.0
    m.hardening_law = G.HARDENING_LINEAR
    m.hardening = 0.1 * E
    m.length_scale = 2.0 * dx
    m.softening_onset = 0.05 / 2.0


def notched_bar(seed: int = 0, precision: int = G.PRECISION_FP32, cells=(16, 16, 64), ppc: int = 8,
                dx: float = 1.0 / 128, pull: float = 0.5, notch=(1, 4), res: int = 128,
                substeps: int = 500, setup=G) -> SceneSpec:
    """Notched bar along z, gripped over 2 cells at each end and pulled apart.
    setup: as for the plate scenes."""
    nx, ny, nz = cells
    origin = ((res - nx) // 2 * dx, (res - ny) // 2 * dx, (res - nz) // 2 * dx)
    geom = G.Geometry(kind=0, cells=(nx, ny, nz), ppc=ppc, n_plates=1, gap_cells=0, notch_width=notch[0],
                      notch_depth=notch[1], dx=dx, origin=origin, seed=seed)
    pos, mat = setup.generate_particles(geom)
    d = setup.reference_defaults(dx, (res, res, res))
    d.dt = 1e-4
    d.gravity[0] = d.gravity[1] = d.gravity[2] = 0.0
    d.particle_volume = dx ** 3 / ppc
    config_material(d.materials[0], dx)
    z0, z1 = origin[2], origin[2] + nz * dx
    d.n_slab_bcs = 2
    d.slabs[0].axis = 2
    d.slabs[0].lo, d.slabs[0].hi = 0.0, z0 + 2 * dx
    d.slabs[0].velocity[2] = -pull
    d.slabs[1].axis = 2
    d.slabs[1].lo, d.slabs[1].hi = z1 - 2 * dx, res * dx
    d.slabs[1].velocity[2] = pull
    d.precision = precision
    mass = np.full(len(pos), 1000.0 * d.particle_volume)
    vel = np.zeros_like(pos)
    return SceneSpec("notched_bar", d, pos, mass, vel, mat, substeps)


def notched_bar_sized(n_target: int, seed: int = 0, precision: int = G.PRECISION_FP32_FP64SVD, E: float = 1e5,
                      yield_stress: float = 200.0, density: float = 1000.0, pull: float = 0.5,
                      dx: float = 1.0 / 128, ppc: int = 8, substeps: int = 1000) -> SceneSpec:
    """Notched bar of a x a x 4a cells with about n_target particles; the grid
    is sized to the bar (cubic, 8-cell margins)."""
    a = max(4, int(round((n_target / (4.0 * ppc)) ** (1.0 / 3.0))))
    res = max(32, -(-(4 * a + 16) // 4) * 4)
    sp = notched_bar(seed=seed, precision=precision, cells=(a, a, 4 * a), ppc=ppc, dx=dx, pull=pull,
                     notch=(1, max(1, a // 4)), res=res, substeps=substeps)
    m = sp.desc.materials[0]
    config_material(m, dx, E)
    m.yield_stress = yield_stress
    m.density = density
    sp.masses = np.full(sp.n, density * sp.desc.particle_volume)
    sp.name = f"notched_bar_{sp.n}"
    return sp


def notched_bar_batch(n_scenes: int = 64, seed: int = 0, lo: int = 10_000, hi: int = 500_000,
                      precision: int = G.PRECISION_FP32_FP64SVD, substeps: int = 1000) -> list[SceneSpec]:
    """Independent notched bars of uneven size and parameters (batched workload)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_scenes))
    out = []
    for k in range(n_scenes):
        f = rng.uniform(0.5, 1.5, 3)
        out.append(notched_bar_sized(int(sizes[k]), seed=seed * 1000 + k, precision=precision, E=1e5 * f[0],
                                     yield_stress=200.0 * f[1], density=1000.0 * f[2],
                                     pull=float(rng.uniform(0.2, 1.0)), substeps=substeps))
    return out


def _plate_scene(name: str, cells_xy: int, dx: float, ppc: int, margin: int, gap: int, res_y: int, seed: int,
                 precision: int, substeps: int, sphere_gap: float = 2.0, setup=G) -> SceneSpec:
    """setup: provides generate_particles(geometry) and reference_defaults(dx,
    res); this module's library binding unless a caller that must not load the
    library passes another implementation of the same two functions."""
    n_plates = 4
    thick = 16
    res_xz = cells_xy + 2 * margin
    origin = (margin * dx, margin * dx, margin * dx)
    geom = G.Geometry(kind=1, cells=(cells_xy, thick, cells_xy), ppc=ppc, n_plates=n_plates, gap_cells=gap,
                      notch_width=0, notch_depth=0, dx=dx, origin=origin, seed=seed)
    pos, mat = setup.generate_particles(geom)
    d = setup.reference_defaults(dx, (res_xz, res_y, res_xz))
    d.dt = 5e-5
    d.gravity[0], d.gravity[1], d.gravity[2] = 0.0, -9.8, 0.0
    d.particle_volume = dx ** 3 / ppc
    rng = np.random.default_rng(seed)
    Es = np.exp(rng.uniform(np.log(5e4), np.log(5e5), n_plates))
    d.n_materials = n_plates
    for k in range(1, n_plates):
        d.materials[k] = d.materials[0]  # reference constants for every plate
    for k in range(n_plates):
        config_material(d.materials[k], dx, float(Es[k]))
    top = origin[1] + (n_plates * thick + (n_plates - 1) * gap) * dx
    r = 0.1
    d.n_sphere_bcs = 1
    sp = d.spheres[0]
    sp.center[0] = sp.center[2] = res_xz * dx / 2
    sp.center[1] = top + r + sphere_gap * dx
    sp.radius = r
    sp.velocity[1] = -5.0
    d.precision = precision
    mass = np.full(len(pos), 1000.0 * d.particle_volume)
    vel = np.zeros_like(pos)
    return SceneSpec(name, d, pos, mass, vel, mat, substeps)


def plates(seed: int = 0, precision: int = G.PRECISION_FP32, substeps: int = 2000, setup=G) -> SceneSpec:
    """4 plates of 256x256x16 cells at dx=1/256, 8 ppc: 33,554,432 particles."""
    return _plate_scene("plates_33m", 256, 1.0 / 256, 8, 8, 8, 160, seed, precision, substeps, setup=setup)


def plates_8m(seed: int = 0, precision: int = G.PRECISION_FP32, substeps: int = 100, setup=G) -> SceneSpec:
    """4 plates of 128x128x16 cells at dx=1/128, 8 ppc: 8,388,608 particles."""
    return _plate_scene("plates_8m", 128, 1.0 / 128, 8, 8, 4, 96, seed, precision, substeps, setup=setup)


def plates_small(cells_xy: int = 32, seed: int = 0, precision: int = G.PRECISION_FP32,
                 substeps: int = 50, sphere_gap: float = 2.0) -> SceneSpec:
    """Scaled-down plate-impact scene with the same parameters (test size).
    sphere_gap: height of the sphere's lowest point above the top plate, in
    cells (0.5 puts the top layer of nodes with mass inside the sphere at once)."""
    dx = 1.0 / 128
    return _plate_scene(f"plates_{cells_xy}", cells_xy, dx, 8, 8, 4, 96, seed, precision, substeps, sphere_gap)


def wall_slide(corner: str = "low", n_side: int = 8, ppc: int = 8, seed: int = 11, precision: int = G.PRECISION_FP32,
               dx: float = 1.0 / 64, res: int = 48, speed: float = 2.0) -> SceneSpec:
    """A box moving diagonally into a corner of the domain with the sticky
    walls on (collideWithGround, TimeIntegrator.cu:117-165).  "low": the box's
    lowest cells start at node 5 on every axis and it moves towards -x, -y, -z;
    "high": its highest cells end at node res - 4 and it moves towards +x, +y,
    +z.  Either way the stencils reach the wall layers (nodes i <= 4 and
    i > res - 4) at once.  No gravity; elastic material."""
    lo = 5 if corner == "low" else res - 4 - n_side
    origin = (lo * dx,) * 3
    geom = G.Geometry(kind=2, cells=(n_side, n_side, n_side), ppc=ppc, n_plates=1, gap_cells=0, notch_width=0,
                      notch_depth=0, dx=dx, origin=origin, seed=seed)
    pos, mat = G.generate_particles(geom)
    d = G.reference_defaults(dx, (res, res, res))
    d.dt = 1e-4
    d.gravity[0] = d.gravity[1] = d.gravity[2] = 0.0
    d.wall_bc = 1
    d.wall_layers = 4
    d.particle_volume = dx ** 3 / ppc
    config_material(d.materials[0], dx)
    d.materials[0].yield_stress = 1e9  # elastic
    d.precision = precision
    sign = -1.0 if corner == "low" else 1.0
    vel = np.tile(sign * speed * np.array([1.0, 0.7, 0.4]), (len(pos), 1))
    mass = np.full(len(pos), 1000.0 * d.particle_volume)
    return SceneSpec(f"wall_slide_{corner}", d, pos, mass, vel, mat, 20)


def plates_sized(n_target: int, seed: int = 0, precision: int = G.PRECISION_FP32_FP64SVD, e_scale: float = 1.0,
                 substeps: int = 1000) -> SceneSpec:
    """Plate-impact scene (4 plates of c x c x 16 cells at dx=1/128, 8 ppc) with
    about n_target particles; the sphere radius is capped at 0.4 plate widths."""
    dx = 1.0 / 128
    c = max(4, int(round((n_target / (4 * 16 * 8)) ** 0.5)))
    sp = _plate_scene(f"plates_{c}", c, dx, 8, 8, 4, 96, seed, precision, substeps)
    sp.desc.spheres[0].radius = min(0.1, 0.4 * c * dx)
    top = 8 * dx + (4 * 16 + 3 * 4) * dx
    sp.desc.spheres[0].center[1] = top + sp.desc.spheres[0].radius + 2 * dx
    for k in range(sp.desc.n_materials):
        config_material(sp.desc.materials[k], dx, sp.desc.materials[k].youngs_modulus * e_scale)
    return sp


def served_request_params(rng: np.random.Generator, lo: int = 20_000, hi: int = 2_000_000) -> dict:
    """The random draws of one request of the served workload (cheap; the
    particles are generated by served_request_build): a notched bar or a plate
    impact (50/50), size log-uniform in [lo, hi], horizon uniform in
    [200, 2000] substeps, parameters within +/-50% of the notched bar's."""
    n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    horizon = int(rng.integers(200, 2001))
    f = rng.uniform(0.5, 1.5, 3)
    bar = bool(rng.random() < 0.5)
    pull = float(rng.uniform(0.2, 1.0)) if bar else None
    return dict(n=n, horizon=horizon, f=f, bar=bar, pull=pull)


def served_request_build(params: dict, k: int) -> tuple[SceneSpec, int]:
    p = params
    f = p["f"]
    if p["bar"]:
        sp = notched_bar_sized(p["n"], seed=k, E=1e5 * f[0], yield_stress=200.0 * f[1], density=1000.0 * f[2],
                               pull=p["pull"], substeps=p["horizon"])
    else:
        sp = plates_sized(p["n"], seed=k, e_scale=float(f[0]), substeps=p["horizon"])
    return sp, p["horizon"]


def served_request(rng: np.random.Generator, k: int, lo: int = 20_000, hi: int = 2_000_000) -> tuple[SceneSpec, int]:
    """One request of the served workload (served_request_params, then its particles)."""
    return served_request_build(served_request_params(rng, lo, hi), k)


def blob(n_side: int = 12, ppc: int = 8, seed: int = 3, precision: int = G.PRECISION_FP32, dx: float = 1.0 / 64,
         res: int = 64, velocity=(0.3, -0.2, 0.1), spin: float = 2.0) -> SceneSpec:
    """Free-flying box with translation + rotation, no gravity, no walls or
    velocity conditions: mass and momentum must be conserved exactly."""
    origin = ((res - n_side) // 2 * dx,) * 3
    geom = G.Geometry(kind=2, cells=(n_side, n_side, n_side), ppc=ppc, n_plates=1, gap_cells=0, notch_width=0,
                      notch_depth=0, dx=dx, origin=origin, seed=seed)
    pos, mat = G.generate_particles(geom)
    d = G.reference_defaults(dx, (res, res, res))
    d.dt = 1e-4
    d.gravity[0] = d.gravity[1] = d.gravity[2] = 0.0
    d.wall_bc = 0
    d.particle_volume = dx ** 3 / ppc
    config_material(d.materials[0], dx)
    d.materials[0].yield_stress = 1e9  # elastic
    d.precision = precision
    c = pos.mean(axis=0)
    vel = np.tile(np.asarray(velocity, dtype=np.float64), (len(pos), 1))
    r = pos - c
    vel[:, 0] += -spin * r[:, 1]
    vel[:, 1] += spin * r[:, 0]
    mass = np.full(len(pos), 1000.0 * d.particle_volume)
    return SceneSpec("blob", d, pos, mass, vel, mat, 20)
