"""The C-ABI surface: symbols, struct layouts, argument checking and the host
scene generator.  No GPU needed (nothing here launches a kernel)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gmpm.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:gmpm_status|const char\*|void)\s+(gmpm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.gmpm.lib()
    names = declared_functions()
    assert len(names) >= 13
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg.gmpm.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT\s+(gmpm_\w+)", out))
    assert set(names) <= exported
    # the binding declares exactly the header's entry points
    assert set(pkg.gmpm.SIGNATURES) == set(names)


def test_struct_layouts_match_header(pkg, tmp_path):
    G = pkg.gmpm
    structs = {"gmpm_material": G.Material, "gmpm_slab_bc": G.SlabBC, "gmpm_sphere_bc": G.SphereBC,
               "gmpm_scene_desc": G.SceneDesc, "gmpm_particle_init": G.ParticleInit, "gmpm_diag": G.Diag,
               "gmpm_scene_geometry": G.Geometry, "gmpm_stage_times": G.StageTimes,
               "gmpm_batch_options": G.BatchOptions, "gmpm_batch_info": G.BatchInfo,
               "gmpm_server_options": G.ServerOptions, "gmpm_request_status": G.RequestStatus,
               "gmpm_server_stats": G.ServerStats}
    probe = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gmpm.h"', "int main(void){"]
    for cname, ct in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    probe.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(probe), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for cname, ct in structs.items():
        assert int(got[cname]) == C.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(ct, fname).offset, (cname, fname)


def test_status_strings(pkg):
    L = pkg.gmpm.lib()
    for s in range(10):
        assert L.gmpm_status_string(s)
    assert L.gmpm_status_string(0) == b"ok"


def test_null_arguments_are_rejected(pkg):
    L = pkg.gmpm.lib()
    G = pkg.gmpm
    assert L.gmpm_context_create(0, None) == G.INVALID_ARG
    assert L.gmpm_substep(None, 1, None) == G.INVALID_ARG
    assert L.gmpm_scene_destroy(None) == G.INVALID_ARG
    assert L.gmpm_read_particles(None, 0, 0, 0, None, 0, None) == G.INVALID_ARG
    assert L.gmpm_diagnostics(None, None) == G.INVALID_ARG
    assert L.gmpm_scene_desc_reference_defaults(None, 1.0, 8, 8, 8) == G.INVALID_ARG
    assert L.gmpm_batch_create(None, None, 0, None, None) == G.INVALID_ARG
    assert L.gmpm_batch_substep(None, 1, None) == G.INVALID_ARG
    assert L.gmpm_batch_get_info(None, None) == G.INVALID_ARG
    assert L.gmpm_batch_destroy(None) == G.INVALID_ARG
    assert L.gmpm_server_create(None, None, None) == G.INVALID_ARG
    assert L.gmpm_server_step(None, 1, None) == G.INVALID_ARG
    assert L.gmpm_server_poll(None, 1, None) == G.INVALID_ARG
    assert L.gmpm_server_destroy(None) == G.INVALID_ARG


def test_batch_option_defaults(pkg):
    G = pkg.gmpm
    o = G.BatchOptions()
    G.lib().gmpm_batch_options_defaults(C.byref(o))
    assert (o.autotune, o.trial_substeps, o.streams, o.sm_share) == (1, 2, 0, 0)


def test_reference_defaults(pkg):
    d = pkg.gmpm.reference_defaults(1.0 / 256, (256, 256, 256))
    m = d.materials[0]
    # constants of Setting.h / applyVonMises / Materials.cpp
    assert d.dt == 1e-4 and d.gravity[1] == -10.0 and d.wall_layers == 4
    assert m.yield_stress == 800.0 and m.hardening == 3.0 and m.alpha_cap == 1.0 and m.dlambda_cap == 100.0
    assert m.strain_cap == 3.0 and m.fracture_energy == 3.0 and m.softening_onset == 0.01
    assert m.residual_fracture == 0.1 and m.mobility == 50.0
    assert m.theta == float(np.float32(1e-4)) and m.length_scale == 0.5 / 256


def test_generator_counts_and_layout(pkg):
    G, S = pkg.gmpm, pkg.scenes
    bar = S.notched_bar()
    assert bar.n == 131072 - 1 * 4 * 16 * 8  # notch: 1 cell wide, 4 deep, full x extent
    # the 33.5M and 8.4M plate scenes: count without allocating
    L = G.lib()
    for cells, dx, expect in [(256, 1 / 256, 33554432), (128, 1 / 128, 8388608)]:
        g = G.Geometry(kind=1, cells=(cells, 16, cells), ppc=8, n_plates=4, gap_cells=4, dx=dx, seed=0)
        n = C.c_int64()
        assert L.gmpm_generate_particles(C.byref(g), C.byref(n), None, None, 0) == G.OK
        assert n.value == expect
    pos = bar.positions
    assert np.all(pos.astype(np.float32).astype(np.float64) == pos)  # FP32-representable
    dx = bar.desc.dx
    cells = np.floor(pos / dx).astype(np.int64)
    _, counts = np.unique(cells, axis=0, return_counts=True)
    assert np.all(counts == 8)  # 8 particles in every cell of the body


def test_generator_deterministic_and_seeded(pkg):
    S = pkg.scenes
    a = S.notched_bar(seed=0).positions
    b = S.notched_bar(seed=0).positions
    c = S.notched_bar(seed=1).positions
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    p = S.plates_small(32)
    assert set(np.unique(p.material_ids)) == {0, 1, 2, 3}
    assert p.desc.n_materials == 4


def test_generator_rejects_bad_geometry(pkg):
    G = pkg.gmpm
    L = G.lib()
    n = C.c_int64()
    for g in [G.Geometry(kind=5, cells=(4, 4, 4), ppc=8, dx=0.1), G.Geometry(kind=0, cells=(0, 4, 4), ppc=8, dx=0.1),
              G.Geometry(kind=0, cells=(4, 4, 4), ppc=0, dx=0.1), G.Geometry(kind=1, cells=(4, 4, 4), ppc=1, dx=0.1,
                                                                             n_plates=0)]:
        assert L.gmpm_generate_particles(C.byref(g), C.byref(n), None, None, 0) == G.INVALID_ARG
    g = G.Geometry(kind=2, cells=(4, 4, 4), ppc=2, dx=0.1)
    assert L.gmpm_generate_particles(C.byref(g), C.byref(n), None, None, 0) == G.OK
    buf = np.empty((n.value - 1, 3))
    assert L.gmpm_generate_particles(C.byref(g), C.byref(n), buf.ctypes.data_as(C.POINTER(C.c_double)), None,
                                     n.value - 1) == G.INVALID_ARG


def test_no_device_is_reported_not_fatal(pkg):
    """On a machine without a GPU the context call returns NO_DEVICE."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    G = pkg.gmpm
    h = C.c_void_p()
    assert G.lib().gmpm_context_create(0, C.byref(h)) == G.NO_DEVICE
