"""The reference's scene samplers (GPU_MPM/LoadSample.cpp) restated in the
library's C-ABI, against fixtures recorded from the reference's own
LoadSample.cpp compiled by oracle/Makefile (tests/golden/make_golden.py):
particle counts and SHA-1 of the positions as float64, bit for bit."""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden"
GOLD = json.loads((GOLDEN / "reference_kats.json").read_text())
# the reference's one shipped OBJ asset, where the reference project is present
# (its root in the environment variable GMPM_REFERENCE_DIR)
_REF = os.environ.get("GMPM_REFERENCE_DIR", "")
TUBE = Path(_REF) / "Assets" / "sample" / "tube_10.obj" if _REF else None


def _check(pos: np.ndarray, rec: dict):
    assert len(pos) == rec["count"]
    if rec["count"]:
        assert [x.hex() for x in pos[0]] == rec["first"]
        assert [x.hex() for x in pos[-1]] == rec["last"]
    assert hashlib.sha1(np.ascontiguousarray(pos, dtype=np.float64).tobytes()).hexdigest() == rec["sha1"]


def test_obj_records_match_reference(pkg):
    # vertex records, then two face records (read as particles by the
    # reference's "<char> x y z" loop), more vertices, and a normal record
    # that ends the list
    pos = pkg.gmpm.sample_obj(GOLDEN / "sample_records.obj")
    _check(pos, GOLD["sample_records_obj"])
    assert len(pos) == 112


@pytest.mark.skipif(TUBE is None or not TUBE.exists(), reason="the reference's tube_10.obj asset is not present")
def test_tube_10_obj_matches_reference(pkg):
    _check(pkg.gmpm.sample_obj(TUBE), GOLD["sample_tube_10_obj"])


def test_cube_matches_reference(pkg):
    # the reference's grid: N = 256 (Setting.h)
    _check(pkg.gmpm.sample_cube(256), GOLD["sample_cube"])


def test_sdf_rejection_samples_match_reference(pkg):
    rec = GOLD["sample_sdf"]
    pos = pkg.gmpm.sample_sdf(GOLDEN / "sample_sphere.sdf", rec["center"], rec["res"], dx=1.0 / 256, seed=1)
    _check(pos, rec)
    # and the samples are inside the placed sphere's box
    assert np.all(pos > 0) and np.all(pos < 1)


def test_sampler_errors(pkg):
    G = pkg.gmpm
    with pytest.raises(G.GmpmError) as e:
        G.sample_obj(GOLDEN / "missing.obj")
    assert e.value.status == G.IO_ERROR
    with pytest.raises(G.GmpmError) as e:
        G.sample_sdf(GOLDEN / "sample_records.obj", (128, 64, 128), (8, 8, 8), 1.0 / 256)
    assert e.value.status == G.IO_ERROR
    with pytest.raises(G.GmpmError):
        G.sample_cube(2)


def test_facade_sample_class_matches_reference(pkg, tmp_path):
    """The C++ facade's Sample (the reference's class and method names) gives
    the same particles as the reference's own LoadSample.cpp."""
    import subprocess

    root = Path(__file__).resolve().parents[1]
    lib = pkg.gmpm.LIB_PATH
    exe = tmp_path / "samples"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", str(root / "include"), str(root / "tests" / "cpp" /
                    "samples.cpp"), str(lib), f"-Wl,-rpath,{lib.parent}", "-o", str(exe)], check=True)

    def run(*args) -> np.ndarray:
        out = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, check=True).stdout
        lines = out.splitlines()
        n = int(lines[0].split()[1])
        return np.array([[float.fromhex(x) for x in l.split()] for l in lines[1:1 + n]], dtype=np.float64).reshape(-1, 3)

    _check(run("obj", GOLDEN / "sample_records.obj"), GOLD["sample_records_obj"])
    rec = GOLD["sample_sdf"]
    _check(run("sdf", GOLDEN / "sample_sphere.sdf", *rec["center"], *rec["res"]), rec)
