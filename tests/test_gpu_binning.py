"""Binning on the GPU is bit-exact with the oracle's canonical binning: the
permutation (d_indexTrans), sorted keys, active pages, per-page and per-cell
particle ranges, grid pages and the page adjacency."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ARRAYS = [("perm", 1), ("keys", 2), ("block_keys", 3), ("block_start", 4), ("cell_start", 5), ("grid_keys", 6),
          ("adj", 7)]


def assert_same_binning(gpu, orc):
    for name, aid in ARRAYS:
        a = gpu.binning(name).astype(np.int64)
        b = orc.binning(aid).astype(np.int64)
        assert a.shape == b.shape, name
        assert np.array_equal(a, b), f"{name}: {np.count_nonzero(a != b)} entries differ"


SCENES = {
    "blob": lambda S: S.blob(),
    "notched_bar": lambda S: S.notched_bar(),
    "plates32": lambda S: S.plates_small(32),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_initial_binning_bit_exact(pkg, ctx, oracle, name):
    sp = SCENES[name](pkg.scenes)
    gpu = sp.build(ctx)
    gpu.rebin()
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    assert_same_binning(gpu, orc)


@pytest.mark.parametrize("name", ["notched_bar", "plates32"])
def test_binning_after_motion_bit_exact(pkg, ctx, oracle, name):
    """After 25 FP32 substeps, bin the GPU's own (moved, reordered) particles on
    both sides: the GPU permutation must equal the oracle's stable sort."""
    G = pkg.gmpm
    sp = SCENES[name](pkg.scenes)
    gpu = sp.build(ctx)
    gpu.substep(25)
    pos = gpu.read("position", order=G.ORDER_INTERNAL)
    mass = gpu.read("mass", order=G.ORDER_INTERNAL)
    ids = gpu.read("id", order=G.ORDER_INTERNAL).astype(np.int64)
    gpu.rebin()
    orc = oracle.OracleScene(sp.desc, pos, mass, None, sp.material_ids[ids])
    assert_same_binning(gpu, orc)
    assert gpu.sync() == G.OK


def test_duplicate_and_boundary_positions(pkg, ctx, oracle):
    """Many particles on identical positions and on cell faces still bin exactly."""
    G = pkg.gmpm
    dx = 1.0 / 64
    rng = np.random.default_rng(5)
    cells = rng.integers(8, 56, size=(4000, 3))
    pos = (cells + rng.integers(0, 2, size=(4000, 3)) * 0.5) * dx  # exact cell faces and centres
    pos = np.concatenate([pos, np.repeat(pos[:100], 7, axis=0)])  # duplicates
    pos = pos.astype(np.float32).astype(np.float64)
    d = G.reference_defaults(dx, (64, 64, 64))
    mass = np.full(len(pos), 1e-6)
    gpu = G.Scene(ctx, d, pos, mass)
    gpu.rebin()
    orc = oracle.OracleScene(d, pos, mass)
    assert_same_binning(gpu, orc)


@pytest.mark.parametrize("name", ["notched_bar", "plates32"])
def test_binning_from_g2p_keys_bit_exact(pkg, ctx, oracle, name):
    """A substep's binning starts from the cell keys its previous G2P formed
    for the positions it wrote (no key pass): the binning the 25th substep
    ran equals the oracle's binning of the positions the 24th wrote."""
    G = pkg.gmpm
    sp = SCENES[name](pkg.scenes)
    gpu = sp.build(ctx)
    gpu.substep(24)
    pos = gpu.read("position", order=G.ORDER_INTERNAL)
    mass = gpu.read("mass", order=G.ORDER_INTERNAL)
    ids = gpu.read("id", order=G.ORDER_INTERNAL).astype(np.int64)
    gpu.substep(1)
    assert gpu.sync() == G.OK
    orc = oracle.OracleScene(sp.desc, pos, mass, None, sp.material_ids[ids])
    assert_same_binning(gpu, orc)


def test_crowded_page_and_cell(pkg, ctx, oracle):
    """Canonical order where the warp's buffer does not hold the page: a page of
    1,280 particles (20 in each of its 64 cells, ranked in windows of whole
    cells) and one cell of 1,000 particles (ranked from global memory), all
    in shuffled order, bin exactly like the oracle's stable sort."""
    G = pkg.gmpm
    dx = 1.0 / 64
    rng = np.random.default_rng(11)
    # base node b for x = (b + 1 + u) dx, u in [-0.5, 0.5)
    page = np.stack(np.meshgrid(np.arange(8, 12), np.arange(8, 12), np.arange(8, 12), indexing="ij"), -1).reshape(-1, 3)
    crowded = np.repeat(page, 20, axis=0)
    cell = np.repeat(np.array([[20, 20, 20]]), 1000, axis=0)
    other = rng.integers(4, 56, size=(3000, 3))
    base = np.concatenate([crowded, cell, other])
    pos = (base + 1 + rng.random(base.shape) - 0.5) * dx
    pos = pos[rng.permutation(len(pos))].astype(np.float32).astype(np.float64)
    d = G.reference_defaults(dx, (64, 64, 64))
    mass = np.full(len(pos), 1e-6)
    gpu = G.Scene(ctx, d, pos, mass)
    gpu.rebin()
    assert gpu.sync() == G.OK
    orc = oracle.OracleScene(d, pos, mass)
    assert_same_binning(gpu, orc)
    counts = np.diff(gpu.binning("cell_start"))
    assert counts.max() >= 1000 and (counts >= 20).sum() >= 64
