"""The reference's other energy models (Setting.h:38 Energy_Model 0 and 1),
selected per material: elastic fixed-corotated
(computeContributionFixedCorotated, ExplicitTimeIntegrator.cu:22-47) and
Neo-Hookean with phase-field fracture driving
(computeContributionNeoHookean, :372-446).  FP64 on the GPU against the
oracle's restatement on a box stretched along x and squeezed along y, alone
and mixed with a von Mises material."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from parity import errors, format_errors

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "F", "B", "stress", "psi_max", "damage", "volume")
TOL = dict(position=1e-9, velocity=1e-9, F=1e-9, B=1e-8, stress=1e-8, psi_max=1e-7, damage=1e-9, volume=1e-9)


def _stretched_box(pkg, models, precision):
    G, S = pkg.gmpm, pkg.scenes
    sp = S.blob(n_side=10, precision=precision, velocity=(0.0, 0.0, 0.0), spin=0.0)
    d = sp.desc
    d.n_materials = len(models)
    for k, model in enumerate(models):
        if k > 0:  # the reference defaults are set for material 0 only
            ctypes.memmove(ctypes.addressof(d.materials[k]), ctypes.addressof(d.materials[0]),
                           ctypes.sizeof(d.materials[0]))
        S.config_material(d.materials[k], d.dx, E=2e4)
        d.materials[k].yield_stress = 1e9 if model == G.ENERGY_VON_MISES_FRACTURE else 200.0
        d.materials[k].energy_model = model
    d.phase_field = G.PHASE_FIELD_EXPLICIT
    c = sp.positions.mean(axis=0)
    r = sp.positions - c
    sp.velocities[:, 0] = 4.0 * r[:, 0]    # stretch along x
    sp.velocities[:, 1] = -2.0 * r[:, 1]   # squeeze along y
    sp.velocities[:, 2] = 0.5 * r[:, 0]    # and shear
    # materials by half-space when mixed
    sp.material_ids[:] = 0
    if len(models) > 1:
        sp.material_ids[r[:, 2] > 0] = 1
    return sp


def _run(pkg, ctx, oracle, sp, steps=20):
    gpu = sp.build(ctx)
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    gpu.substep(steps)
    orc.substep(steps)
    assert gpu.sync() == pkg.gmpm.OK
    return gpu, orc


@pytest.mark.parametrize("model", [1, 2], ids=["fixed_corotated", "neo_hookean_fracture"])
def test_energy_model_fp64_matches_oracle(pkg, ctx, oracle, model):
    G = pkg.gmpm
    sp = _stretched_box(pkg, [model], G.PRECISION_FP64)
    gpu, orc = _run(pkg, ctx, oracle, sp)
    fields = FIELDS if model == G.ENERGY_NEO_HOOKEAN_FRACTURE else tuple(f for f in FIELDS if f != "psi_max")
    e = errors(G, gpu, orc, sp.positions, fields=fields, dx=sp.desc.dx)
    print(f"\n[energy model {model}] {format_errors(e)}")
    for k in fields:
        assert e[k] <= TOL[k], (model, k, e[k])
    F = gpu.read("F")
    assert np.abs(F - np.eye(3).ravel()).max() > 1e-3  # the box did deform
    if model == G.ENERGY_NEO_HOOKEAN_FRACTURE:
        assert gpu.read("psi_max").max() > 0  # tension drives the phase field
    else:
        assert np.array_equal(gpu.read("psi_max"), np.zeros(sp.n))  # no fracture driving


def test_mixed_models_fp64_matches_oracle_and_fp32_is_deterministic(pkg, ctx, oracle):
    G = pkg.gmpm
    models = [G.ENERGY_VON_MISES_FRACTURE, G.ENERGY_NEO_HOOKEAN_FRACTURE]
    sp = _stretched_box(pkg, models, G.PRECISION_FP64)
    gpu, orc = _run(pkg, ctx, oracle, sp)
    e = errors(G, gpu, orc, sp.positions, fields=FIELDS, dx=sp.desc.dx)
    print(f"\n[von Mises + Neo-Hookean] {format_errors(e)}")
    for k in FIELDS:
        assert e[k] <= TOL[k], (k, e[k])
    sp32 = _stretched_box(pkg, models, G.PRECISION_FP32_FP64SVD)
    a, b = sp32.build(ctx), sp32.build(ctx)
    a.substep(20)
    b.substep(20)
    for f in ("position", "F", "damage", "stress"):
        x = a.read(f)
        assert np.isfinite(x).all() and np.array_equal(x, b.read(f)), f


def test_unknown_energy_model_is_rejected(pkg, ctx):
    G = pkg.gmpm
    sp = _stretched_box(pkg, [G.ENERGY_FIXED_COROTATED], G.PRECISION_FP32)
    sp.desc.materials[0].energy_model = 7
    with pytest.raises(G.GmpmError) as e:
        sp.build(ctx)
    assert e.value.status == G.INVALID_ARG
