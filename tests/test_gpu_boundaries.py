"""Velocity conditions against the FP64 oracle, acting on nodes with mass
within the compared horizon:

* the moving sphere (the plate scenes' impactor; it generalises the spheres of
  PullGrid_kernal, TimeIntegrator.cu:169-214): its lowest point starts half a
  cell above the top plate, so the top layer of nodes with mass is inside it
  from the first substep and particles under it are driven towards -5 m/s
  while the rest of the plates fall at g t (about 0.01 m/s);
* the sticky walls (collideWithGround, TimeIntegrator.cu:117-165): a box
  slides diagonally into the low or the high corner of the domain, its
  stencils inside the 4-node wall layers from the first substep, where a node
  moving outwards stops in all three components.

Each test also shows that the condition did act: particles whose velocity it
set are counted against an oracle run without it.  FP64 on the GPU agrees
with the oracle to 1e-9 (relative L2 per field), FP32 to the short-horizon
FP32 tolerances."""
from __future__ import annotations

import numpy as np
import pytest

from parity import errors, format_errors

pytestmark = pytest.mark.gpu

CORE = ("position", "velocity", "F", "B", "damage", "stress")
TOL = {1: dict(position=1e-9, velocity=1e-9, F=1e-9, B=1e-8, damage=1e-9, stress=1e-6),
       0: dict(position=2e-3, velocity=1e-3, F=1e-4, B=2e-2, damage=1e-4, stress=2e-2)}
STEPS = 20


def run_pair(pkg, ctx, oracle, sp, steps):
    gpu = sp.build(ctx)
    orc = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    gpu.substep(steps)
    orc.substep(steps)
    assert gpu.sync() == pkg.gmpm.OK
    return gpu, orc


@pytest.mark.parametrize("prec", [1, 0], ids=["fp64", "fp32"])
def test_sphere_impactor_matches_oracle(pkg, ctx, oracle, prec):
    G = pkg.gmpm
    sp = pkg.scenes.plates_small(32, precision=prec, sphere_gap=0.5)
    gpu, orc = run_pair(pkg, ctx, oracle, sp, STEPS)
    e = errors(G, gpu, orc, sp.positions, fields=CORE, dx=sp.desc.dx)
    v_orc = orc.field_by_id(G.FIELD["velocity"])
    v_gpu = gpu.read("velocity", order=G.ORDER_ORIGINAL)
    # the same scene without the sphere: free fall
    sp.desc.n_sphere_bcs = 0
    free = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    free.substep(STEPS)
    v_free = free.field_by_id(G.FIELD["velocity"])
    set_by_sphere = np.abs(v_orc[:, 1] - v_free[:, 1]) > 0.5
    print(f"\n[plates32 sphere contact prec={prec} {STEPS} substeps] {format_errors(e)}; "
          f"{int(set_by_sphere.sum())} particles driven by the sphere, min v_y {v_orc[:, 1].min():.3f}")
    assert set_by_sphere.sum() > 100
    assert v_orc[:, 1].min() < -2.0 and np.abs(v_free[:, 1]).max() < 0.05
    assert (np.abs(v_gpu[:, 1] - v_free[:, 1]) > 0.5).sum() == pytest.approx(set_by_sphere.sum(), rel=0.01)
    for k, tol in TOL[prec].items():
        assert e[k] <= tol, (k, e[k], tol)
    if prec == 1:
        assert e["position_dx"] <= 1e-9


@pytest.mark.parametrize("corner", ["low", "high"])
@pytest.mark.parametrize("prec", [1, 0], ids=["fp64", "fp32"])
def test_sticky_walls_match_oracle(pkg, ctx, oracle, prec, corner):
    G = pkg.gmpm
    sp = pkg.scenes.wall_slide(corner, precision=prec)
    gpu, orc = run_pair(pkg, ctx, oracle, sp, STEPS)
    e = errors(G, gpu, orc, sp.positions, fields=CORE, dx=sp.desc.dx)
    v_orc = orc.field_by_id(G.FIELD["velocity"])
    sp.desc.wall_bc = 0
    free = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    free.substep(STEPS)
    v_free = free.field_by_id(G.FIELD["velocity"])
    set_by_wall = np.linalg.norm(v_orc - v_free, axis=1) > 0.2
    print(f"\n[wall_slide {corner} prec={prec} {STEPS} substeps] {format_errors(e)}; "
          f"{int(set_by_wall.sum())} of {sp.n} particles slowed by the walls")
    assert set_by_wall.sum() > 100
    # the walls only remove velocity towards them
    speed0 = np.linalg.norm(sp.velocities[0])
    assert np.linalg.norm(v_orc[set_by_wall], axis=1).max() < speed0
    for k, tol in TOL[prec].items():
        assert e[k] <= tol, (k, e[k], tol)
    if prec == 1:
        assert e["position_dx"] <= 1e-9
