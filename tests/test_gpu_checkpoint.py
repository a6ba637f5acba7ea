"""Checkpoint/resume (gmpm_scene_save / gmpm_scene_load): a scene saved after
k substeps and loaded continues bitwise like the uninterrupted run."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "F", "damage", "B", "alpha", "psi_max", "stress", "volume", "FP", "pf_flux")


def _resume_matches(pkg, ctx, sp, k, m, tmp_path):
    G = pkg.gmpm
    ref = sp.build(ctx)
    ref.substep(k + m)
    a = sp.build(ctx)
    a.substep(k)
    path = tmp_path / "scene.gmpm"
    a.save(path)
    a.close()
    b = G.Scene.load(ctx, path)
    db = b.diagnostics()
    assert db["substeps"] == k
    b.substep(m)
    assert b.sync() == G.OK and ref.sync() == G.OK
    for f in FIELDS:
        x, y = ref.read(f), b.read(f)
        assert np.array_equal(x, y), (sp.name, f, float(np.abs(x - y).max()))
    dr, db = ref.diagnostics(), b.diagnostics()
    for key in ("time", "substeps", "dt", "n_blocks", "n_grid_blocks"):
        assert dr[key] == db[key], key


def test_resume_fp32_notched_bar(pkg, ctx, tmp_path):
    _resume_matches(pkg, ctx, pkg.scenes.notched_bar(), 12, 9, tmp_path)


def test_resume_fp64_adaptive_dt(pkg, ctx, tmp_path):
    G = pkg.gmpm
    sp = pkg.scenes.blob(n_side=8, velocity=(3.0, -2.0, 1.0), precision=G.PRECISION_FP64)
    sp.desc.dt = 5e-3
    sp.desc.adaptive_dt = 1
    _resume_matches(pkg, ctx, sp, 5, 5, tmp_path)


def test_load_rejects_bad_files(pkg, ctx, tmp_path):
    G = pkg.gmpm
    with pytest.raises(G.GmpmError) as e:
        G.Scene.load(ctx, tmp_path / "missing.gmpm")
    assert e.value.status == G.IO_ERROR
    bad = tmp_path / "bad.gmpm"
    bad.write_bytes(b"not a checkpoint" * 8)
    with pytest.raises(G.GmpmError) as e:
        G.Scene.load(ctx, bad)
    assert e.value.status == G.IO_ERROR


def test_load_rejects_other_format_versions_and_precisions(pkg, ctx, tmp_path):
    """A valid file with its format version (uint32 at byte 8) or its real
    size (uint32 at byte 12) changed is refused: a file from a build with
    another particle layout must not be read as this one's."""
    G = pkg.gmpm
    sc = pkg.scenes.notched_bar(cells=(8, 8, 16), res=32, dx=1.0 / 32).build(ctx)
    sc.substep(2)
    good = tmp_path / "good.gmpm"
    sc.save(good)
    sc.close()
    G.Scene.load(ctx, good).close()  # the unchanged file loads
    data = bytearray(good.read_bytes())
    version = int.from_bytes(data[8:12], "little")
    real_bytes = int.from_bytes(data[12:16], "little")
    assert version >= 2 and real_bytes in (4, 8)
    for offset, value in ((8, version - 1), (8, version + 1), (12, 12 - real_bytes)):
        bad = bytearray(data)
        bad[offset:offset + 4] = int(value).to_bytes(4, "little")
        path = tmp_path / f"patched_{offset}_{value}.gmpm"
        path.write_bytes(bytes(bad))
        with pytest.raises(G.GmpmError) as e:
            G.Scene.load(ctx, path)
        assert e.value.status == G.IO_ERROR, (offset, value)
