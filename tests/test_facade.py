"""The C++ host side (include/gmpm_simulator.hpp): it compiles against the
C-ABI, and on a GPU its frame loop (MPMSimulator::simulateStick) reproduces
the direct C-ABI run bit for bit."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def build_headless(pkg, out_dir: Path) -> Path:
    exe = out_dir / "headless"
    lib = pkg.gmpm.LIB_PATH
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" /
                    "headless.cpp"), str(lib), f"-Wl,-rpath,{lib.parent}", "-o", str(exe)], check=True)
    return exe


def test_facade_compiles_and_links(pkg, tmp_path):
    exe = build_headless(pkg, tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_headless_frame_loop_matches_direct_run(pkg, ctx, tmp_path):
    exe = build_headless(pkg, tmp_path)
    out = tmp_path / "pos.bin"
    r = subprocess.run([str(exe), "0", "12", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    pos_cpp = np.fromfile(out, dtype=np.float64).reshape(-1, 3)
    sp = pkg.scenes.notched_bar()
    scene = sp.build(ctx)
    scene.substep(12)
    assert np.array_equal(pos_cpp, scene.read("position"))
