"""Binning without device allocation.

gmpm_bin_positions_noalloc serves callers that cannot allocate device memory
on the call path (a host framework that owns all device memory and passes
this library only views of its own buffers, or a latency-critical loop that
may not pay for cudaMalloc).  Its scratch is a fixed file-scope device array
shared by all calls.  Here its output, called through the C-ABI on
caller-owned device buffers, must equal the scene binning (gmpm_rebin) of the
same positions bit for bit, on consecutive calls with different inputs, so
nothing left in the shared scratch by one call leaks into the next; also at
the top of its key space (128 nodes per axis, page coordinate 31) with
positions outside the domain, which are clamped and reported; and a cell
holding more particles than the in-cell ordering handles is reported too.

This file is collected last (test_zz_*) and also passes on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scene_binning(G, ctx, desc, positions, masses):
    scene = G.Scene(ctx, desc, positions, masses)
    scene.rebin()
    out = scene.binning("perm"), scene.binning("keys")
    scene.close()
    return out


def noalloc_binning(G, torch, positions, desc):
    n = len(positions)
    pos = torch.tensor(np.asarray(positions, dtype=np.float32), device="cuda").contiguous()
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    keys = torch.zeros((n,), dtype=torch.int32, device="cuda")
    flags = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    res = desc.grid_res
    st = G.lib().gmpm_bin_positions_noalloc(C.c_void_p(pos.data_ptr()), n, desc.dx, res[0], res[1], res[2],
                                            C.c_void_p(perm.data_ptr()), C.c_void_p(keys.data_ptr()),
                                            C.c_void_p(flags.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == G.OK, G.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    return perm.cpu().numpy(), keys.cpu().numpy().view(np.uint32), int(flags.cpu().numpy().view(np.uint32)[0])


def test_noalloc_binning_matches_scene_binning(pkg, ctx):
    torch = pytest.importorskip("torch")
    G, S = pkg.gmpm, pkg.scenes
    # consecutive calls with different sizes, then the first input again
    cases = [S.notched_bar(), S.blob(), S.notched_bar()]
    for spec in cases:
        ref_perm, ref_keys = scene_binning(G, ctx, spec.desc, spec.positions, spec.masses)
        perm, keys, flags = noalloc_binning(G, torch, spec.positions, spec.desc)
        assert flags == 0
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(perm, ref_perm)


def test_noalloc_at_the_top_of_its_key_space(pkg, ctx):
    """128 nodes per axis (page coordinates up to 31, the top of the 5-bit
    key), particles crowding the upper faces, and a few outside the domain on
    either side, which both paths clamp the same way."""
    torch = pytest.importorskip("torch")
    G = pkg.gmpm
    res, dx = 128, 1.0 / 128
    rng = np.random.default_rng(3)
    inside = rng.uniform(100 * dx, 126 * dx, (60_000, 3))
    outside = np.array([[1.2, 0.5, 0.5], [0.5, -0.1, 0.5], [0.5, 0.5, 1.01], [-0.3, 1.3, 0.2], [0.999, 0.999, 0.999]])
    pos = np.concatenate([inside, outside]).astype(np.float32).astype(np.float64)
    pos = pos[rng.permutation(len(pos))]
    desc = G.reference_defaults(dx, (res, res, res))
    masses = np.full(len(pos), 1e-6)
    ref_perm, ref_keys = scene_binning(G, ctx, desc, pos, masses)
    for _ in range(2):
        perm, keys, flags = noalloc_binning(G, torch, pos, desc)
        assert flags == G.FLAG_OUT_OF_DOMAIN
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(perm, ref_perm)
    assert (keys >> 6).max() >= (1 << 15) - 64  # pages at the top of the key space are in use


def test_noalloc_reports_an_overfull_cell(pkg, ctx):
    """7,000 positions below the domain all clamp into one cell, more than the
    6,144 the in-cell ordering ranks: the call reports it, the keys are still
    sorted and equal the scene binning's, every other cell is in canonical
    order, and the overfull cell holds exactly the clamped particles."""
    torch = pytest.importorskip("torch")
    G = pkg.gmpm
    res, dx = 64, 1.0 / 64
    rng = np.random.default_rng(5)
    normal = rng.uniform(16 * dx, 40 * dx, (20_000, 3))
    clamped = rng.uniform(-0.2, -0.01, (7_000, 3))
    pos = np.concatenate([normal, clamped]).astype(np.float32).astype(np.float64)
    order = rng.permutation(len(pos))
    pos = pos[order]
    is_clamped = order >= len(normal)
    desc = G.reference_defaults(dx, (res, res, res))
    ref_perm, ref_keys = scene_binning(G, ctx, desc, pos, np.full(len(pos), 1e-6))
    perm, keys, flags = noalloc_binning(G, torch, pos, desc)
    assert flags == G.FLAG_OUT_OF_DOMAIN | G.FLAG_TABLE_OVERFLOW
    assert np.array_equal(keys, ref_keys)
    assert (np.diff(keys.astype(np.int64)) >= 0).all()
    assert np.array_equal(np.sort(perm), np.arange(len(pos)))
    big = keys == keys[0]  # the clamped cell: page 0, cell 0, first in key order
    assert big.sum() == 7_000 and np.array_equal(np.sort(perm[big]), np.nonzero(is_clamped)[0])
    assert np.array_equal(perm[~big], ref_perm[~big])
    # the canonical order elsewhere: ascending input index within each cell
    k, p = keys[~big], perm[~big]
    same = k[1:] == k[:-1]
    assert (p[1:][same] > p[:-1][same]).all()


def test_noalloc_rejects_inputs_beyond_its_limits(pkg, ctx):
    torch = pytest.importorskip("torch")
    G = pkg.gmpm
    L = G.lib()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert L.gmpm_bin_positions_noalloc(p, G.NOALLOC_MAX_PARTICLES + 1, 0.01, 64, 64, 64, p, p, None, None) == \
        G.INVALID_ARG
    assert L.gmpm_bin_positions_noalloc(p, 4, 0.01, 64, G.NOALLOC_MAX_RES + 1, 64, p, p, None, None) == \
        G.INVALID_ARG
    assert L.gmpm_bin_positions_noalloc(None, 4, 0.01, 64, 64, 64, p, p, None, None) == G.INVALID_ARG
