"""Substep parity of the CUDA library with the FP64 oracle, per particle
(matched by original index), as relative L2 errors.

Two horizons:
* short (10-20 substeps), where differences are rounding-level: FP64 on the
  GPU must agree with the oracle to 1e-9 and FP32 to the FP32 tolerances;
* the first 100 substeps of the notched bar: the reference's return map
  (dlambda = y / (2/3 g tr tau) capped at 100, ExplicitTimeIntegrator.cu:211-220)
  amplifies rounding exponentially once plastic flow starts, so the stated
  100-substep tolerances are also checked against the oracle's own spread
  under a rounding-size perturbation of its input.
"""
from __future__ import annotations

import numpy as np
import pytest

from parity import errors, format_errors

pytestmark = pytest.mark.gpu

CORE = ("position", "velocity", "F", "damage")

# short horizon, FP64 GPU vs FP64 oracle
TOL_FP64_SHORT = dict(position=1e-9, velocity=1e-9, F=1e-9, B=1e-8, damage=1e-9, alpha=1e-7, psi_max=1e-6,
                      stress=1e-6, volume=1e-9, FP=1e-7, pf_flux=1e-5)
# short horizon, FP32 GPU vs FP64 oracle
TOL_FP32_SHORT = dict(position=2e-3, velocity=1e-3, F=1e-4, damage=1e-4, B=2e-2, volume=1e-4)
# first 100 substeps of the notched bar
TOL_100 = {1: dict(position=1e-3, velocity=5e-3, F=1e-2, damage=1e-3),   # FP64
           0: dict(position=3e-3, velocity=1e-2, F=3e-2, damage=3e-3)}   # FP32


def run_pair(pkg, ctx, oracle, sp, steps):
    gpu = sp.build(ctx)
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    gpu.substep(steps)
    orc.substep(steps)
    assert gpu.sync() == pkg.gmpm.OK
    return gpu, orc


SHORT = [("blob", lambda S, p: S.blob(precision=p), 20), ("notched_bar", lambda S, p: S.notched_bar(precision=p), 10),
         ("plates32", lambda S, p: S.plates_small(32, precision=p), 20)]

# Fields that are pure rounding noise in a scene at this horizon are not
# compared: the plates are in free fall for the first 20 substeps (F = I,
# B = 0, no stress), and the blob is elastic at strains ~1e-6, where the FP32
# Hencky strain log(sigma) itself carries ~10% relative error.
SKIP64 = {"plates32": {"B", "stress", "psi_max", "pf_flux"}}
SKIP32 = {"plates32": {"B", "stress", "psi_max", "pf_flux", "position"},
          "blob": {"psi_max", "stress", "pf_flux", "FP", "position"}}


@pytest.mark.parametrize("name,make,steps", SHORT, ids=[s[0] for s in SHORT])
def test_fp64_short_horizon(pkg, ctx, oracle, name, make, steps):
    G = pkg.gmpm
    sp = make(pkg.scenes, G.PRECISION_FP64)
    gpu, orc = run_pair(pkg, ctx, oracle, sp, steps)
    e = errors(G, gpu, orc, sp.positions, dx=sp.desc.dx)
    print(f"\n[{name} FP64 {steps} substeps] {format_errors(e)}")
    assert e["position_dx"] <= 1e-9
    for k, tol in TOL_FP64_SHORT.items():
        if k not in SKIP64.get(name, set()):
            assert e[k] <= tol, (k, e[k], tol)


@pytest.mark.parametrize("name,make,steps", SHORT, ids=[s[0] for s in SHORT])
def test_fp32_short_horizon(pkg, ctx, oracle, name, make, steps):
    G = pkg.gmpm
    sp = make(pkg.scenes, G.PRECISION_FP32)
    gpu, orc = run_pair(pkg, ctx, oracle, sp, steps)
    e = errors(G, gpu, orc, sp.positions, dx=sp.desc.dx)
    print(f"\n[{name} FP32 {steps} substeps] {format_errors(e)}")
    assert e["position_dx"] <= 1e-4  # FP32 positions near 0.5 carry ~6e-8 / dx ~ 1e-5 cells of rounding
    for k, tol in TOL_FP32_SHORT.items():
        if k not in SKIP32.get(name, set()):
            assert e[k] <= tol, (k, e[k], tol)


@pytest.mark.parametrize("prec", [1, 0], ids=["fp64", "fp32"])
def test_notched_bar_100_substeps(pkg, ctx, oracle, prec):
    G = pkg.gmpm
    sp = pkg.scenes.notched_bar(precision=prec)
    gpu, orc = run_pair(pkg, ctx, oracle, sp, 100)
    e = errors(G, gpu, orc, sp.positions, fields=CORE)
    # the oracle against itself with its input perturbed at the precision's rounding level
    eps = 1e-15 if prec == 1 else 6e-8
    pert = oracle.OracleScene(sp.desc, sp.positions * (1 + eps), sp.masses, sp.velocities, sp.material_ids)
    pert.substep(100)
    floor = {}
    for f in CORE:
        a = pert.field_by_id(G.FIELD[f])
        b = orc.field_by_id(G.FIELD[f])
        if f == "position":
            a, b = a - sp.positions, b - sp.positions
        floor[f] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    print(f"\n[notched_bar prec={prec} 100 substeps] gpu: {format_errors(e)}\n    oracle spread: {format_errors(floor)}")
    for k, tol in TOL_100[prec].items():
        assert e[k] <= tol, (k, e[k], tol)
        assert e[k] <= 20 * floor[k] + 1e-12, (k, e[k], floor[k])


def test_fp32_with_fp64_svd_fallback(pkg, ctx, oracle):
    """Precision form: FP32 bulk with FP64 SVD/return map for ill-conditioned F
    is at least as close to the oracle as plain FP32 on the plate scene."""
    G = pkg.gmpm
    res = {}
    for prec in (G.PRECISION_FP32, G.PRECISION_FP32_FP64SVD):
        sp = pkg.scenes.plates_small(32, precision=prec)
        gpu, orc = run_pair(pkg, ctx, oracle, sp, 30)
        res[prec] = errors(G, gpu, orc, sp.positions, fields=CORE)
        print(f"\n[plates32 prec={prec} 30 substeps] {format_errors(res[prec])}")
    for k in CORE:
        assert res[G.PRECISION_FP32_FP64SVD][k] <= 2 * res[G.PRECISION_FP32][k] + 1e-7


def test_adaptive_dt_matches_oracle(pkg, ctx, oracle):
    """Adaptive (CFL) time step computed on the device from G2P's maximum speed:
    FP64 GPU and oracle take the same steps and agree to 1e-9."""
    G = pkg.gmpm
    sp = pkg.scenes.blob(n_side=8, velocity=(3.0, -2.0, 1.0), precision=G.PRECISION_FP64)
    sp.desc.dt = 5e-3
    sp.desc.adaptive_dt = 1
    gpu, orc = run_pair(pkg, ctx, oracle, sp, 10)
    dg, do = gpu.diagnostics(), orc.diagnostics(G.Diag)
    assert dg["dt"] < 5e-3 and dg["dt"] == pytest.approx(do["dt"], rel=1e-12)
    assert dg["time"] == pytest.approx(do["time"], rel=1e-12)
    e = errors(G, gpu, orc, sp.positions, dx=sp.desc.dx, fields=CORE)
    print(f"\n[blob adaptive dt FP64 10 substeps] dt={dg['dt']:.6g} {format_errors(e)}")
    for k in CORE:
        assert e[k] <= 1e-9, (k, e[k])
