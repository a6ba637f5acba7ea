"""Binning without device allocation.

gmpm_bin_positions_noalloc serves callers that cannot allocate device memory
on the call path (a host framework that owns all device memory and passes
this library only views of its own buffers, or a latency-critical loop that
may not pay for cudaMalloc).  Its scratch is a fixed file-scope device array
shared by all calls.  Here its output, called through the C-ABI on
caller-owned device buffers, must equal the scene binning (gmpm_rebin) of the
same positions bit for bit, on consecutive calls with different inputs, so
nothing left in the shared scratch by one call leaks into the next.

This file is collected last (test_zz_*) and also passes on its own.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scene_binning(ctx, spec):
    scene = spec.build(ctx)
    scene.rebin()
    return scene.binning("perm"), scene.binning("keys")


def noalloc_binning(G, spec, torch):
    n = spec.n
    pos = torch.tensor(spec.positions.astype(np.float32), device="cuda").contiguous()
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    keys = torch.zeros((n,), dtype=torch.int32, device="cuda")
    res = spec.desc.grid_res
    st = G.lib().gmpm_bin_positions_noalloc(C.c_void_p(pos.data_ptr()), n, spec.desc.dx, res[0], res[1], res[2],
                                            C.c_void_p(perm.data_ptr()), C.c_void_p(keys.data_ptr()),
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == G.OK, G.STATUS_NAMES.get(st, st)
    torch.cuda.synchronize()
    return perm.cpu().numpy(), keys.cpu().numpy().view(np.uint32)


def test_noalloc_binning_matches_scene_binning(pkg, ctx):
    torch = pytest.importorskip("torch")
    G, S = pkg.gmpm, pkg.scenes
    # consecutive calls with different sizes, then the first input again
    cases = [S.notched_bar(), S.blob(), S.notched_bar()]
    for spec in cases:
        ref_perm, ref_keys = scene_binning(ctx, spec)
        perm, keys = noalloc_binning(G, spec, torch)
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(perm, ref_perm)


def test_noalloc_rejects_inputs_beyond_its_limits(pkg, ctx):
    torch = pytest.importorskip("torch")
    G = pkg.gmpm
    L = G.lib()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert L.gmpm_bin_positions_noalloc(p, G.NOALLOC_MAX_PARTICLES + 1, 0.01, 64, 64, 64, p, p, None) == \
        G.INVALID_ARG
    assert L.gmpm_bin_positions_noalloc(p, 4, 0.01, 64, G.NOALLOC_MAX_RES + 1, 64, p, p, None) == G.INVALID_ARG
    assert L.gmpm_bin_positions_noalloc(None, 4, 0.01, 64, 64, 64, p, p, None) == G.INVALID_ARG
