"""Conservation, determinism and error reporting of the CUDA library."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1], ids=["fp32", "fp64"])
def test_mass_and_momentum_conserved(pkg, ctx, prec):
    """Free-flying elastic blob (no gravity, walls or velocity conditions):
    total mass and momentum are conserved to 1e-6 relative (FP32) through P2G,
    the grid update and G2P."""
    G = pkg.gmpm
    sp = pkg.scenes.blob(precision=prec)
    gpu = sp.build(ctx)
    p0 = (sp.masses[:, None] * sp.velocities).sum(axis=0)
    m0 = sp.masses.sum()
    gpu.substep(20)
    d = gpu.diagnostics()
    tol = 1e-6 if prec == 0 else 1e-12
    assert abs(d["particle_mass"] - m0) <= tol * m0
    assert abs(d["grid_mass"] - m0) <= tol * m0
    for key in ("particle_momentum", "grid_momentum"):
        assert np.abs(np.array(d[key]) - p0).max() <= tol * np.abs(p0).max(), (key, d[key], p0)
    assert d["flags"] == 0 and d["substeps"] == 20
    assert abs(d["time"] - 20 * sp.desc.dt) < 1e-12


def test_deterministic_mode_is_bitwise_reproducible(pkg, ctx):
    G = pkg.gmpm
    sp = pkg.scenes.plates_small(32)
    a, b = sp.build(ctx), sp.build(ctx)
    a.substep(40)
    b.substep(40)
    for f in ("position", "velocity", "F", "B", "damage", "alpha", "psi_max", "stress", "id"):
        assert np.array_equal(a.read(f, order=G.ORDER_INTERNAL), b.read(f, order=G.ORDER_INTERNAL)), f


def test_readback_orders_agree(pkg, ctx):
    G = pkg.gmpm
    sp = pkg.scenes.notched_bar()
    g = sp.build(ctx)
    g.substep(5)
    ids = g.read("id", order=G.ORDER_INTERNAL).astype(np.int64)
    assert np.array_equal(np.sort(ids), np.arange(sp.n))
    for f in ("position", "F", "damage", "mass"):
        internal = g.read(f, order=G.ORDER_INTERNAL)
        original = g.read(f, order=G.ORDER_ORIGINAL)
        assert np.array_equal(original[ids], internal), f
    x32 = g.read("position", order=G.ORDER_ORIGINAL, dtype=G.DTYPE_F32)
    assert np.array_equal(x32.astype(np.float64), g.read("position"))
    assert np.array_equal(g.read("mass"), sp.masses)


def test_out_of_domain_is_flagged(pkg, ctx):
    """A particle whose stencil leaves the grid raises OUT_OF_DOMAIN (the
    reference would form a negative base node, Particle_kernal.cu:162-164)."""
    G = pkg.gmpm
    dx = 1.0 / 32
    d = G.reference_defaults(dx, (32, 32, 32))
    pos = np.array([[0.5, 0.5, 0.5], [0.2 * dx, 0.5, 0.5], [0.5, 0.5, 31.9 * dx]])
    g = G.Scene(ctx, d, pos, np.full(3, 1e-6))
    g.substep(1)
    assert g.sync() == G.OUT_OF_DOMAIN
    assert g.diagnostics()["flags"] & G.FLAG_OUT_OF_DOMAIN


def test_invalid_scene_arguments(pkg, ctx):
    G = pkg.gmpm
    dx = 1.0 / 32
    pos = np.full((4, 3), 0.5)
    m = np.full(4, 1e-6)
    bad = []
    d = G.reference_defaults(dx, (32, 32, 32)); d.dt = 0.0; bad.append(d)
    d = G.reference_defaults(dx, (32, 32, 4)); bad.append(d)
    d = G.reference_defaults(dx, (32, 32, 32)); d.n_materials = 0; bad.append(d)
    d = G.reference_defaults(dx, (32, 32, 32)); d.materials[0].poisson_ratio = 0.5; bad.append(d)
    d = G.reference_defaults(dx, (32, 32, 32)); d.precision = 7; bad.append(d)
    d = G.reference_defaults(dx, (32, 32, 32)); d.n_slab_bcs = 1; d.slabs[0].axis = 3; bad.append(d)
    for d in bad:
        with pytest.raises(G.GmpmError) as e:
            G.Scene(ctx, d, pos, m)
        assert e.value.status == G.INVALID_ARG
    d = G.reference_defaults(dx, (32, 32, 32))
    with pytest.raises(G.GmpmError):
        G.Scene(ctx, d, pos, m, material_ids=np.array([0, 0, 1, 0]))


def test_table_capacity_overflow(pkg, ctx):
    """A page capacity below the scene's page count is refused at creation."""
    G = pkg.gmpm
    sp = pkg.scenes.notched_bar()
    sp.desc.block_capacity = 16
    with pytest.raises(G.GmpmError) as e:
        sp.build(ctx)
    assert e.value.status == G.TABLE_OVERFLOW


def test_overlapped_reads_match_blocking_reads(pkg, ctx):
    """gmpm_read_particles_async: reads queued behind later substeps (more than
    the two staging buffers in flight) land as the blocking reads of the same
    substeps."""
    import torch

    G = pkg.gmpm
    sp = pkg.scenes.notched_bar()
    a, b = sp.build(ctx), sp.build(ctx)
    want, got = [], []
    for _ in range(4):
        a.substep(1)
        want.append((a.read("position", order=G.ORDER_INTERNAL, dtype=G.DTYPE_F32),
                     a.read("damage", order=G.ORDER_INTERNAL, dtype=G.DTYPE_F32)))
        pos = torch.empty(sp.n * 3, dtype=torch.float32, pin_memory=True)
        dmg = np.empty(sp.n, dtype=np.float32)  # pageable destinations are allowed too
        b.substep(1)
        b.read_into_async("position", pos.data_ptr(), pos.numel() * 4)
        b.read_into_async("damage", dmg.ctypes.data, dmg.nbytes)
        got.append((pos, dmg))
    b.read_wait()
    for (wp, wd), (gp, gd) in zip(want, got):
        assert np.array_equal(wp.reshape(-1), gp.numpy()), "position"
        assert np.array_equal(wd.reshape(-1), gd), "damage"
    with pytest.raises(G.GmpmError):
        b.read_into_async("position", 0, sp.n * 12)
