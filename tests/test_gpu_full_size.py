"""Full-size precision checks.

Precision configuration: the 8,388,608-particle plate scene (4 plates of
128x128x16 cells at dx = 1/128, 8 particles per cell, a sphere impactor at
5 m/s that reaches the top plate after about 62 substeps), over its first 100
substeps, compared three ways by relative L2 over particles matched by id
(positions as displacement):

* the production form (FP32 with compensated grid sums and the FP64 SVD
  fallback below sigma_min/sigma_max = 1e-3) against an FP64 run of the same
  scene on the GPU;
* the production form against the FP64 CPU oracle (OpenMP on the host cores;
  about 3 s per substep on 8 cores, 1.6 s on 16);
* the FP64 GPU run against the oracle.

Plastic flow under the impactor amplifies rounding (the reference's return
map divides by tr tau and caps dlambda at 100), so each comparison is also
held against the spread of the FP64 GPU run under an input rounding of the
compared precision: positions moved by half an FP32 ulp for the FP32 form,
by 1e-15 relative for FP64.  A comparison passes within a fixed tolerance
(about 10x the measured errors) or within 20x that spread, whichever is
larger.  Particle mass, momentum and kinetic energy of the two precisions
agree to 1e-5 relative.

Headline configuration: the 33,554,432-particle plates at dx = 1/256, FP32
against FP64 on the GPU over 40 substeps, through the first contact of the
impactor (its lowest point starts 2 cells above the top plate and moves
0.064 cells per substep)."""
from __future__ import annotations

import numpy as np
import pytest

from parity import rel_l2

pytestmark = pytest.mark.gpu

STEPS = 100
FIELDS = ("position", "velocity", "F", "damage")
TOL32 = dict(position_dx=1e-3, position=3e-3, velocity=1e-3, F=2e-5, damage=2e-5)
# FP64 GPU against the oracle, about 10x the measured 7.5e-11 cells, 1.3e-11, 1.2e-10, 1.1e-9, 3e-13
TOL64 = dict(position_dx=1e-9, position=1e-9, velocity=2e-9, F=1e-8, damage=1e-9)


def _perturbed(sp, kind: str) -> np.ndarray:
    x0 = sp.positions.astype(np.float64)
    rng = np.random.default_rng(7)
    sign = np.where(rng.random(x0.shape) < 0.5, -1.0, 1.0)
    if kind == "fp32":
        return x0 + sign * 0.5 * np.spacing(np.abs(x0).astype(np.float32)).astype(np.float64)
    return x0 * (1.0 + sign * 1e-15)


def _gpu_run(pkg, ctx, make, precision, steps, perturb=None):
    G = pkg.gmpm
    sp = make(precision=precision)
    x0 = sp.positions.astype(np.float64).copy()
    if perturb:
        sp.positions = _perturbed(sp, perturb)
    sc = sp.build(ctx)
    sc.substep(steps)
    assert sc.sync() == G.OK
    out = {f: sc.read(f) for f in FIELDS}
    diag = sc.diagnostics()
    sc.close()
    return sp, x0, out, diag


def _compare(a: dict, b: dict, x0: np.ndarray, dx: float) -> dict:
    err = {}
    for f in FIELDS:
        u, w = a[f], b[f]
        assert np.isfinite(u).all() and np.isfinite(w).all(), f
        if f == "position":
            err["position_dx"] = float(np.abs(u - w).max() / dx)
            u, w = u - x0, w - x0
        err[f] = rel_l2(u, w)
    return err


def _fmt(e: dict) -> str:
    return " ".join(f"{k}={v:.2e}" for k, v in e.items())


@pytest.fixture(scope="module")
def plates_8m_runs(pkg, ctx, oracle):
    G, S = pkg.gmpm, pkg.scenes
    sp, x0, ref64, d64 = _gpu_run(pkg, ctx, S.plates_8m, G.PRECISION_FP64, STEPS)
    assert sp.n == 8_388_608
    _, _, f32, d32 = _gpu_run(pkg, ctx, S.plates_8m, G.PRECISION_FP32_FP64SVD, STEPS)
    _, _, per32, _ = _gpu_run(pkg, ctx, S.plates_8m, G.PRECISION_FP64, STEPS, perturb="fp32")
    _, _, per64, _ = _gpu_run(pkg, ctx, S.plates_8m, G.PRECISION_FP64, STEPS, perturb="fp64")
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    orc.substep(STEPS)
    ora = {f: orc.field_by_id(G.FIELD[f]) for f in FIELDS}
    dorc = orc.diagnostics(G.Diag)
    del orc
    return dict(sp=sp, x0=x0, ref64=ref64, f32=f32, per32=per32, per64=per64, ora=ora, d64=d64, d32=d32, dorc=dorc)


def test_plates_8m_fp32_against_fp64(plates_8m_runs):
    r = plates_8m_runs
    dx = r["sp"].desc.dx
    err = _compare(r["f32"], r["ref64"], r["x0"], dx)
    spread = _compare(r["per32"], r["ref64"], r["x0"], dx)
    print(f"\n[plates_8m, {STEPS} substeps] FP32 vs FP64 GPU: {_fmt(err)}")
    print(f"[plates_8m, {STEPS} substeps] FP64 GPU, input moved by FP32 half-ulps: {_fmt(spread)}")
    d32, d64 = r["d32"], r["d64"]
    keys = ("particle_mass", "grid_mass", "particle_momentum", "kinetic_energy", "max_speed", "min_damage",
            "n_blocks", "flags")
    print("[diag] fp64:", {k: d64[k] for k in keys})
    print("[diag] fp32:", {k: d32[k] for k in keys})
    assert d32["flags"] == 0 and d64["flags"] == 0
    assert d32["particle_mass"] == d64["particle_mass"]
    assert abs(d32["grid_mass"] / d64["grid_mass"] - 1) < 1e-6
    for k in ("kinetic_energy", "max_speed"):
        assert abs(d32[k] / d64[k] - 1) < 1e-5, k
    assert abs(d32["particle_momentum"][1] / d64["particle_momentum"][1] - 1) < 1e-5
    f32 = r["f32"]
    assert ((f32["damage"] >= 0) & (f32["damage"] <= 1)).all()
    assert np.abs(f32["velocity"]).max() > 1.0  # the impactor has reached the plates
    assert d64["min_damage"] < 0.9  # and started to drive the phase field
    for k, tol in TOL32.items():
        assert err[k] <= max(tol, 20 * spread[k]), (k, err[k], spread[k])


def test_plates_8m_against_oracle(plates_8m_runs):
    """The precision configuration's oracle leg: the FP32 production form and
    the FP64 GPU run, each against the FP64 CPU oracle over 100 substeps."""
    r = plates_8m_runs
    dx = r["sp"].desc.dx
    e32 = _compare(r["f32"], r["ora"], r["x0"], dx)
    e64 = _compare(r["ref64"], r["ora"], r["x0"], dx)
    s32 = _compare(r["per32"], r["ref64"], r["x0"], dx)
    s64 = _compare(r["per64"], r["ref64"], r["x0"], dx)
    print(f"\n[plates_8m, {STEPS} substeps] FP32 vs oracle: {_fmt(e32)}")
    print(f"[plates_8m, {STEPS} substeps] FP64 GPU vs oracle: {_fmt(e64)}")
    print(f"[plates_8m, {STEPS} substeps] FP64 GPU spread under 1e-15 input rounding: {_fmt(s64)}")
    do, d64 = r["dorc"], r["d64"]
    print("[diag] oracle:", {k: do[k] for k in ("particle_mass", "grid_mass", "kinetic_energy", "max_speed",
                                                "min_damage", "flags")})
    assert do["particle_mass"] == pytest.approx(d64["particle_mass"], rel=1e-12)
    assert do["kinetic_energy"] == pytest.approx(d64["kinetic_energy"], rel=1e-6)
    assert do["min_damage"] < 0.9
    for k, tol in TOL32.items():
        assert e32[k] <= max(tol, 20 * s32[k]), ("fp32", k, e32[k], s32[k])
    for k, tol in TOL64.items():
        assert e64[k] <= max(tol, 20 * s64[k]), ("fp64", k, e64[k], s64[k])


def test_plates_33m_fp32_against_fp64(pkg, ctx):
    """The headline scene at its own size (dx = 1/256): FP32 against FP64 on
    the GPU through the impactor's first contact."""
    G, S = pkg.gmpm, pkg.scenes
    steps = 40
    sp, x0, ref64, d64 = _gpu_run(pkg, ctx, S.plates, G.PRECISION_FP64, steps)
    assert sp.n == 33_554_432
    _, _, f32, d32 = _gpu_run(pkg, ctx, S.plates, G.PRECISION_FP32, steps)
    err = _compare(f32, ref64, x0, sp.desc.dx)
    print(f"\n[plates_33m, {steps} substeps] FP32 vs FP64 GPU: {_fmt(err)}; max |v| {d64['max_speed']:.3f}")
    assert d32["flags"] == 0 and d64["flags"] == 0
    assert d64["max_speed"] > 1.0  # the impactor has touched the top plate
    assert d32["particle_mass"] == d64["particle_mass"]
    assert abs(d32["kinetic_energy"] / d64["kinetic_energy"] - 1) < 1e-4
    for k, tol in dict(position_dx=1e-3, position=1e-3, velocity=1e-3, F=1e-5, damage=1e-5).items():
        assert err[k] <= tol, (k, err[k], tol)
