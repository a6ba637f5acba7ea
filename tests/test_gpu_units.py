"""Parity with the FP64 oracle on scenes shaped to hit the edges of the
kernels' work splitting: G2P units of 256 sorted slots that run across page
boundaries (at most three pages per unit, each CTA an equal share of the
slots), and P2G page chunks.

* one particle: a single unit with a single page, most CTAs idle;
* sparse pages: one particle per page, so every unit is cut at its third
  page and a CTA's share spans many pages;
* a crowded page: 700 particles in one page (more than a P2G chunk and more
  than a G2P unit) next to a few lone particles;
* a share boundary: 3,000 particles on a lattice, so CTA shares end inside
  pages.
"""
from __future__ import annotations

import numpy as np
import pytest

from parity import errors, format_errors

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "F", "damage", "B", "volume")
TOL = dict(position=1e-9, velocity=1e-9, F=1e-9, damage=1e-9, B=1e-8, volume=1e-9)


def _spec(pkg, name, pos, vel, steps=10, dx=1.0 / 64, res=64):
    G, S = pkg.gmpm, pkg.scenes
    d = G.reference_defaults(dx, (res, res, res))
    d.dt = 1e-4
    d.gravity[0] = d.gravity[1] = d.gravity[2] = 0.0
    d.wall_bc = 0
    d.particle_volume = dx ** 3 / 8
    S.config_material(d.materials[0], dx)
    d.precision = G.PRECISION_FP64
    n = len(pos)
    mass = np.full(n, 1000.0 * d.particle_volume)
    return S.SceneSpec(name, d, np.ascontiguousarray(pos, dtype=np.float64),
                       mass, np.ascontiguousarray(vel, dtype=np.float64), np.zeros(n, dtype=np.int32), steps)


def _scenes(pkg):
    rng = np.random.default_rng(11)
    dx = 1.0 / 64
    out = []
    # one particle
    out.append(_spec(pkg, "one_particle", np.array([[0.5, 0.5, 0.5]]), np.array([[0.3, -0.2, 0.1]])))
    # one particle per page: a lattice with a spacing of 8 cells (two pages)
    g = np.arange(2, 7) * 8 + 2.3
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * dx
    out.append(_spec(pkg, "sparse_pages", lat, rng.uniform(-0.2, 0.2, lat.shape)))
    # a crowded page (base nodes 28..31 on every axis) and lone particles
    crowd = (28.5 + rng.uniform(0.0, 4.0, (700, 3))) * dx
    lone = (np.array([[10.7, 12.2, 40.1], [50.3, 20.8, 9.9], [33.3, 50.5, 45.2]])) * dx
    pos = np.concatenate([crowd, lone])
    out.append(_spec(pkg, "crowded_page", pos, rng.uniform(-0.05, 0.05, pos.shape)))
    # 3,000 particles on a jittered lattice: CTA shares end inside pages
    side = np.arange(20, 35) + 0.5
    lat2 = np.stack(np.meshgrid(side, side, np.arange(20, 34) + 0.5, indexing="ij"), -1).reshape(-1, 3)
    lat2 = (lat2 + rng.uniform(-0.3, 0.3, lat2.shape)) * dx
    out.append(_spec(pkg, "share_boundary", lat2, rng.uniform(-0.1, 0.1, lat2.shape)))
    return out


@pytest.mark.parametrize("idx", range(4), ids=["one_particle", "sparse_pages", "crowded_page", "share_boundary"])
def test_work_split_edges_match_oracle(pkg, ctx, oracle, idx):
    G = pkg.gmpm
    sp = _scenes(pkg)[idx]
    gpu = sp.build(ctx)
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    gpu.substep(sp.substeps)
    orc.substep(sp.substeps)
    assert gpu.sync() == G.OK
    # A lone particle's APIC matrix is v sum_i w_i (x_i - x_p)^T, zero in exact
    # arithmetic (the B-spline weights reproduce linear functions), so in the
    # scenes of lone particles B is rounding noise on both sides.
    fields = tuple(f for f in FIELDS if not (f == "B" and sp.name in ("one_particle", "sparse_pages")))
    e = errors(G, gpu, orc, sp.positions, fields=fields, dx=sp.desc.dx)
    print(f"\n[{sp.name} n={sp.n}] {format_errors(e)}")
    for k in fields:
        assert e[k] <= TOL[k], (sp.name, k, e[k])


def test_crowded_page_is_deterministic(pkg, ctx):
    """The crowded page in FP32 (two P2G chunks, several G2P units) runs
    bitwise the same twice."""
    G = pkg.gmpm
    sp = _scenes(pkg)[2]
    sp.desc.precision = G.PRECISION_FP32
    a, b = sp.build(ctx), sp.build(ctx)
    a.substep(10)
    b.substep(10)
    for f in ("position", "velocity", "F", "damage"):
        assert np.array_equal(a.read(f), b.read(f)), f
