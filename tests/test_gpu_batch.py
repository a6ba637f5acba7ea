"""Batched stepping (gmpm_batch): every scene of a batch ends bitwise equal to
the same scene stepped alone (deterministic P2G), through autotuning, graph
replays and recaptures after a scene is stepped outside the batch."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "F", "damage", "B", "alpha", "stress")


def _specs(pkg):
    S = pkg.scenes
    specs = S.notched_bar_batch(5, seed=7, lo=8_000, hi=120_000, substeps=40)
    specs.append(S.plates_small(32, precision=pkg.gmpm.PRECISION_FP32))
    specs.append(S.blob(precision=pkg.gmpm.PRECISION_FP64))
    return specs


def _same(a, b, name):
    for f in FIELDS:
        x, y = a.read(f), b.read(f)
        assert np.array_equal(x, y), (name, f, float(np.abs(x - y).max()))


def test_batch_equals_scenes_alone(pkg, ctx):
    G = pkg.gmpm
    specs = _specs(pkg)
    alone = [sp.build(ctx) for sp in specs]
    mixed = [sp.build(ctx) for sp in specs]
    steps = 40
    for sc in alone:
        sc.substep(steps)
    batch = G.Batch(ctx, mixed, autotune=True, trial_substeps=2)
    batch.substep(steps)
    info = batch.info()
    print("\n[batch]", info)
    assert info["tuned"] == 1 and info["captures"] >= 2 and info["graph_nodes"] > 0
    assert info["substeps"] == steps
    for sp, a, b in zip(specs, alone, mixed):
        assert a.sync() == G.OK and b.sync() == G.OK
        _same(a, b, sp.name)
        assert a.diagnostics()["substeps"] == b.diagnostics()["substeps"] == steps
    batch.close()


def test_batch_recaptures_after_outside_step(pkg, ctx):
    G = pkg.gmpm
    specs = _specs(pkg)[:3]
    alone = [sp.build(ctx) for sp in specs]
    mixed = [sp.build(ctx) for sp in specs]
    batch = G.Batch(ctx, mixed, autotune=False)
    batch.substep(3)
    mixed[1].substep(1)            # one scene alone: parities no longer match the graphs
    batch.substep(4)
    c1 = batch.info()["captures"]
    assert c1 >= 4                 # two graphs, then two more after the outside step
    for k, sc in enumerate(alone):
        sc.substep(7 + (1 if k == 1 else 0))
    for sp, a, b in zip(specs, alone, mixed):
        _same(a, b, sp.name)
    batch.close()


def test_batched_workload_scene_stays_finite(pkg, ctx):
    """The batched workload's scene 6 (a grip particle reaches a hydrostatic
    trial state with equal FP32 singular values) stays finite in FP32."""
    G = pkg.gmpm
    sp = pkg.scenes.notched_bar_batch(64, seed=0, precision=G.PRECISION_FP32)[6]
    sc = sp.build(ctx)
    sc.substep(40)
    assert sc.sync() == G.OK


def test_batch_is_one_launch_per_stage_over_its_scenes(pkg, ctx):
    """Scenes of one kernel kind advance with one launch per stage, so the
    graph's kernel count depends on the kinds present, not on the number of
    scenes: 40 bars of one kind give the same 23 kernel nodes as 3."""
    G, S = pkg.gmpm, pkg.scenes
    nodes = {}
    for count in (3, 40):
        specs = S.notched_bar_batch(count, seed=3, lo=4_000, hi=30_000, substeps=4)
        scenes = [sp.build(ctx) for sp in specs]
        batch = G.Batch(ctx, scenes, autotune=False)
        batch.substep(4)
        info = batch.info()
        assert info["table_scenes"] == count
        nodes[count] = info["kernel_nodes"]
        if count == 40:  # two of them against the same scenes alone
            for k in (0, 27):
                alone = specs[k].build(ctx)
                alone.substep(4)
                _same(alone, scenes[k], specs[k].name)
                alone.close()
        batch.close()
        for sc in scenes:
            sc.close()
    assert nodes[3] == nodes[40] == 23


def test_batch_with_implicit_scene_on_a_branch(pkg, ctx):
    """A scene with the implicit phase field (its solve stops on a device flag)
    runs its own launch sequence on a branch beside the scene table; both
    kinds of scene still end equal to themselves alone."""
    G, S = pkg.gmpm, pkg.scenes
    specs = S.notched_bar_batch(3, seed=9, lo=6_000, hi=20_000, substeps=6)
    imp = S.notched_bar_sized(10_000, seed=5, precision=G.PRECISION_FP64, substeps=6)
    imp.desc.phase_field = G.PHASE_FIELD_IMPLICIT
    specs.append(imp)
    alone = [sp.build(ctx) for sp in specs]
    mixed = [sp.build(ctx) for sp in specs]
    for sc in alone:
        sc.substep(6)
    batch = G.Batch(ctx, mixed, autotune=False)
    batch.substep(6)
    info = batch.info()
    assert info["table_scenes"] == 3 and info["kernel_nodes"] > 23
    for sp, a, b in zip(specs, alone, mixed):
        assert a.sync() == G.OK and b.sync() == G.OK
        _same(a, b, sp.name)
    batch.close()
