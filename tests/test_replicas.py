"""The multi-GPU form of the path is independent replicas, one per rank, with
no collective on the data path: ranks meet only at the timing barriers, and
the job's time is the slowest rank's.  These tests run that host-side logic
of bench.py as two gloo ranks on the CPU."""
from __future__ import annotations

import importlib.util
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = _load_bench()
        local_ms = 100.0 + 25.0 * rank  # rank 1 is the slow one
        dist.barrier()
        ms_max = bench.max_over_ranks(local_ms, dist)
        rate = bench.job_rate(world, 1000, 10, ms_max)
        dist.barrier()
        Path(out_dir, f"rank{rank}.txt").write_text(f"{ms_max} {rate}")
    finally:
        dist.destroy_process_group()


def test_slowest_rank_sets_the_job_time(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for rank in range(world):
        ms_max, rate = map(float, Path(tmp_path, f"rank{rank}.txt").read_text().split())
        assert ms_max == 125.0
        # two replicas of 1000 particles, 10 substeps each, in 125 ms
        assert rate == pytest.approx(2 * 1000 * 10 / 0.125)


def test_single_process_needs_no_group():
    bench = _load_bench()
    assert bench.max_over_ranks(42.5, None) == 42.5
    assert bench.job_rate(1, 500, 4, 2.0) == pytest.approx(1e6)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference (CPU) arm prints its line from rank 0 only;
    other ranks exit 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_line_contract():
    """Rank 0's reference line: the same metric, unit and workload as the
    CUDA arm, at least 3 warm-up steps, impl "reference", and cpu_baseline
    and e2e objects that repeat the line's own value with no transfers."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--reference-sample"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "particle-substeps/sec" and line["unit"] == "particle-substeps/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["warmup"] >= 3 and line["steps"] == 1
    assert line["config"]["workload"].startswith("plates_33m: 4 plates of 256x256x16 cells")
    cpu, e2e = line["cpu_baseline"], line["e2e"]
    assert cpu["value"] == line["value"] and cpu["kind"] in ("port", "reference") and cpu["cores"] >= 1
    assert cpu["sample"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["same_config"] is False


def test_reference_arm_times_the_whole_workload():
    """By default the reference arm runs the CUDA arm's own scene (here the
    notched bar, small enough for a CPU test), not a sample of it."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "notched_bar",
                        "--steps", "2", "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["config"]["same_config"] is True and line["config"]["timed_steps"] == 2
    assert line["config"]["particles"] == 130_560  # the notched bar, notch removed
    assert line["config"]["workload"].startswith("notched_bar: 16x16x64 cells")


def test_reference_arm_does_not_load_the_product_library():
    """The reference arm sets its sample up through the oracle, so the process
    maps oracle/liboracle.so and never the library under test."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--reference-sample'];\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('LIBGMPM', 'libgmpm.so' in maps, 'LIBORACLE', 'liboracle.so' in maps)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "LIBGMPM False LIBORACLE True" in r.stdout, r.stdout[-500:]


def test_oracle_scene_setup_equals_the_librarys(pkg, oracle):
    """The CPU legs' set-up (oracle) gives the library's scene description
    byte for byte and its seeded particles bit for bit."""
    import ctypes as C

    import numpy as np

    G = pkg.gmpm
    setup = oracle.SceneSetup(G)
    for dx, res in ((1.0 / 256, (272, 160, 272)), (1.0 / 128, (128, 128, 128))):
        a, b = G.reference_defaults(dx, res), setup.reference_defaults(dx, res)
        assert C.string_at(C.addressof(a), C.sizeof(a)) == C.string_at(C.addressof(b), C.sizeof(b))
    geoms = [G.Geometry(kind=1, cells=(12, 16, 10), ppc=8, n_plates=4, gap_cells=8, notch_width=0, notch_depth=0,
                        dx=1.0 / 256, origin=(8 / 256, 8 / 256, 8 / 256), seed=0),
             G.Geometry(kind=0, cells=(16, 16, 64), ppc=8, n_plates=1, gap_cells=0, notch_width=1, notch_depth=4,
                        dx=1.0 / 128, origin=(0.4375, 0.4375, 0.25), seed=3),
             G.Geometry(kind=2, cells=(5, 7, 3), ppc=3, n_plates=1, gap_cells=0, notch_width=0, notch_depth=0,
                        dx=1.0 / 64, origin=(0.25, 0.3, 0.35), seed=11)]
    for g in geoms:
        pa, ma = G.generate_particles(g)
        pb, mb = setup.generate_particles(g)
        assert np.array_equal(pa, pb) and np.array_equal(ma, mb)
