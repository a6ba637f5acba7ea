"""Implicit phase-field mode: the reference's Jacobi-PCG solve
(ExplicitTimeIntegrator.cu:909-972) on the GPU against the oracle's
restatement, with and without the reference's max-combine dot-product quirk;
reproducibility and batched capture of the solve."""
from __future__ import annotations

import numpy as np
import pytest

from parity import errors, format_errors

pytestmark = pytest.mark.gpu

CORE = ("position", "velocity", "F", "damage")


def _bar(pkg, prec, quirk=0):
    G = pkg.gmpm
    sp = pkg.scenes.notched_bar(cells=(6, 6, 24), res=48, precision=prec, pull=1.0)
    sp.desc.phase_field = G.PHASE_FIELD_IMPLICIT
    sp.desc.pcg_max_combine = quirk
    return sp


@pytest.mark.parametrize("quirk", [0, 1], ids=["sum", "max_combine"])
def test_implicit_fp64_matches_oracle(pkg, ctx, oracle, quirk):
    G = pkg.gmpm
    sp = _bar(pkg, G.PRECISION_FP64, quirk)
    gpu = sp.build(ctx)
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    for step in range(8):
        gpu.substep(1)
        orc.substep(1)
        assert gpu.diagnostics()["pcg_iterations"] == orc.diagnostics(G.Diag)["pcg_iterations"], step
    assert gpu.sync() == G.OK
    e = errors(G, gpu, orc, sp.positions, dx=sp.desc.dx, fields=CORE)
    print(f"\n[implicit FP64 quirk={quirk} 8 substeps] its={gpu.diagnostics()['pcg_iterations']} {format_errors(e)}")
    for k in CORE:
        assert e[k] <= 1e-9, (k, e[k])


def test_implicit_fp32_reproducible_and_batched(pkg, ctx):
    G = pkg.gmpm
    sp = _bar(pkg, G.PRECISION_FP32)
    a, b, c = sp.build(ctx), sp.build(ctx), sp.build(ctx)
    a.substep(10)
    b.substep(10)
    batch = G.Batch(ctx, [c], autotune=False)
    batch.substep(10)
    for f in CORE:
        assert np.array_equal(a.read(f), b.read(f)), f
        assert np.array_equal(a.read(f), c.read(f)), f
    assert a.sync() == G.OK and a.diagnostics()["pcg_iterations"] >= 1
    batch.close()
