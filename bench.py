#!/usr/bin/env python
"""Benchmark: particle-substeps per second of the explicit MPM substep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one substep (binning, P2G, grid update with explicit phase field,
G2P with SVD + return map) of the whole scene.  Default workload: 4 stacked
plates of 256x256x16 cells at dx=1/256, 8 particles per cell (33,554,432
particles), sphere impactor r=0.1 at 5 m/s, gravity -9.8, dt=5e-5, FP32,
deterministic P2G.  Synthetic seeded data (the reference's sampled assets are
not shipped).  The resident state (about 9 GB) is far larger than L2.

With N>1 (torchrun, one process per GPU) every rank advances its own replica
of the scene: the path has no exchange step, scaling is weak and `value` is
the sum over ranks, timed as the max over ranks.

`--impl reference` times the oracle (the FP64 CPU restatement of the
reference's algorithm; the reference itself has no CPU path) on the host
cores, on a bounded sample of the same workload (4 plates of 48x48x16 cells,
same dx, ppc and materials).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "explicit-gpumpm-ductile-fracture_b200"

# Algorithmic bytes (FP32 state layout; one read or write of each byte the
# kernel must touch).  Per particle / per grid node of a grid page.
ALGO_BYTES = {
    "sort": dict(particle=20, node=0),    # read x (12) + write key and slot (8)
    "p2g": dict(particle=112, node=36),   # read x v B sigma c m V FP q; write 9 channels per node
    "grid": dict(particle=0, node=56),    # read 9 channels, write 5 channels per node
    "g2p": dict(particle=224, node=20),   # read x F c alpha psi m id; write x v F B c alpha psi sigma V FP q m id
}
STAGE_KEY = {"sort": "bin_ms", "p2g": "p2g_ms", "grid": "grid_ms", "g2p": "g2p_ms"}
CPU_SAMPLE_CELLS = 48


def load_package():
    spec = importlib.util.spec_from_file_location("gmpm_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gmpm_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402  (test/baseline infrastructure)
    oracle.build()
    return oracle


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=6650.0, source="fallback")


def clocks_median_mhz(clocks) -> float | None:
    """Median SM clock sampled during the timed region, if any."""
    try:
        v = clocks.summary().get("sm_mhz")
        return float(v) if v else None
    except Exception:
        return None


def measured_traffic() -> dict:
    """DRAM bytes per particle per kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic_per_particle.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


WORKLOADS = {
    "plates_33m": "plates_33m: 4 plates of 256x256x16 cells, dx=1/256, 8 ppc, sphere impactor r=0.1 at 5 m/s, "
                  "g=-9.8, dt=5e-5",
    "plates_8m": "plates_8m: 4 plates of 128x128x16 cells, dx=1/128, 8 ppc, sphere impactor r=0.1 at 5 m/s, "
                 "g=-9.8, dt=5e-5",
    "notched_bar": "notched_bar: 16x16x64 cells, dx=1/128, 8 ppc, pulled at +/-0.5 m/s, dt=1e-4",
}


def workload(pkg, name: str, seed: int = 0):
    S = pkg.scenes
    make = {"plates_33m": S.plates, "plates_8m": S.plates_8m, "notched_bar": S.notched_bar}.get(name)
    if make is None:
        raise SystemExit(f"unknown workload {name}")
    return make(seed=seed), WORKLOADS[name]


def cpu_sample(pkg, oracle, name: str):
    """The CPU legs' sample of the workload, set up through the oracle (the
    same description and particles as the library's set-up), so that these
    legs do not load the product library."""
    S = pkg.scenes
    setup = oracle.SceneSetup(pkg.gmpm)
    if name.startswith("plates"):
        dx = 1.0 / 256 if name == "plates_33m" else 1.0 / 128
        sp = S._plate_scene("plates_sample", CPU_SAMPLE_CELLS, dx, 8, 8, 8 if dx < 1 / 200 else 4,
                            160 if dx < 1 / 200 else 96, 0, pkg.gmpm.PRECISION_FP64, 10, setup=setup)
        return sp, f"4 plates of {CPU_SAMPLE_CELLS}x{CPU_SAMPLE_CELLS}x16 cells (same dx, ppc, materials), {sp.n} particles"
    sp = S.notched_bar(precision=pkg.gmpm.PRECISION_FP64, setup=setup)
    return sp, f"the full notched bar, {sp.n} particles"


def full_sample(pkg, oracle, name: str):
    """The whole workload (the same scene as the CUDA arm, in FP64), set up through the oracle."""
    S = pkg.scenes
    setup = oracle.SceneSetup(pkg.gmpm)
    make = {"plates_33m": S.plates, "plates_8m": S.plates_8m, "notched_bar": S.notched_bar}[name]
    sp = make(precision=pkg.gmpm.PRECISION_FP64, setup=setup)
    return sp, f"the full workload, {sp.n} particles"


def time_oracle(pkg, oracle, name: str, steps: int, warmup: int, budget_s: float | None = None,
                full: bool = False):
    """Substeps of the oracle on all host cores.  full: the whole workload,
    with the number of timed substeps cut to what fits in budget_s (each
    substep is the whole workload, so the rate stays per substep)."""
    sp, what = full_sample(pkg, oracle, name) if full else cpu_sample(pkg, oracle, name)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.OracleScene(sp.desc, sp.positions, sp.masses, sp.velocities, sp.material_ids)
    o.substep(max(0, warmup))
    per = []
    t_all = time.perf_counter()
    for _ in range(steps):
        t = time.perf_counter()
        o.substep(1)
        per.append(time.perf_counter() - t)
        if budget_s is not None and time.perf_counter() - t_all > budget_s:
            break
    total = sum(per)
    return dict(value=sp.n * len(per) / total, unit="particle-substeps/s", cores=oracle.get_threads(),
                kind="port", sample=f"{what}; {len(per)} substeps after {warmup} warm-up",
                ms_per_step=1e3 * total / len(per), timed_steps=len(per), particles=sp.n)


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which: str):
        setattr(self, which, time.time())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        # samples inside the timed region (plus the one straddling its start)
        inside = [l for t, l in self.lines if t0 - 0.2 <= t <= t1 + 0.05]
        for l in inside:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=mx, reasons=sorted(reasons),
                    samples=len(sm))


def max_over_ranks(value: float, dist, device=None) -> float:
    """Largest per-rank value over all ranks: a job's time is its slowest rank's.
    The reduction runs on `device` under NCCL and on the host under gloo."""
    if dist is None:
        return float(value)
    import torch
    on = device if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=on)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, particles: int, steps: int, ms_max: float) -> float:
    """Whole-job particle-substeps/s of `world` replicas of `particles` particles
    stepped `steps` substeps, timed as the slowest rank's `ms_max`."""
    return world * particles * steps / (ms_max / 1e3)


def run_ours(args, pkg, rank: int, local_rank: int, world: int, dist):
    import torch

    G = pkg.gmpm
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = G.Context(local_rank)
    sp, what = workload(pkg, args.workload)
    if getattr(args, "implicit", False):
        sp.desc.phase_field = G.PHASE_FIELD_IMPLICIT
        what += ", implicit phase field (Jacobi-PCG, tol 1e-6, <= 100 iterations)"
    if getattr(args, "atomic_p2g", False):
        sp.desc.deterministic = 0
        what += ", P2G node sums with shared-memory atomics (not bitwise reproducible)"
    t0 = time.perf_counter()
    scene = sp.build(ctx)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    scene.substep(args.warmup, sh)
    torch.cuda.synchronize(dev)
    launches0 = scene.diagnostics()["kernel_launches"]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        barrier()
        torch.cuda.synchronize(dev)
        clocks.mark("t0")
        start.record(stream)
        scene.substep(args.steps, sh)
        end.record(stream)
        end.synchronize()
        clocks.mark("t1")
        torch.cuda.synchronize(dev)
        barrier()
    ms = start.elapsed_time(end)
    diag = scene.diagnostics()
    launches = diag["kernel_launches"] - launches0
    status = scene.sync()
    ms_max = max_over_ranks(ms, dist, dev)
    value = job_rate(world, sp.n, args.steps, ms_max)

    # per-stage device times (CUDA events on the same stream) for the roofline
    stages = scene.substep_timed(min(5, max(1, args.steps)), sh)
    nsub = max(1, stages["substeps"])
    nodes = 64 * diag["n_grid_blocks"]
    peaks = measured_peaks()
    traffic = measured_traffic()
    kernels = {}
    for k, key in STAGE_KEY.items():
        t = stages[key] / nsub / 1e3
        b = ALGO_BYTES[k]["particle"] * sp.n + ALGO_BYTES[k]["node"] * nodes
        gbs = b / t / 1e9 if t > 0 else 0.0
        tr = traffic.get(k)
        kernels[k] = dict(ms=round(t * 1e3, 4), algo_bytes=b, achieved_gbs=round(gbs, 1),
                          frac=round(gbs / peaks["hbm_gbs"], 4),
                          traffic=(int(tr * sp.n) if tr is not None else None))
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    # Issue roofline of the transfer kernels: warp instructions per particle (ncu,
    # the committed profile) x particles / (SMs x 4 schedulers x SM clock).  P2G
    # and G2P are bound by issue and latency, not by HBM, so this is the ceiling
    # that explains their time.
    issue = {}
    ipp = traffic.get("warp_instructions_per_particle", {})
    props = torch.cuda.get_device_properties(dev)
    sm_hz = 1e6 * (clocks_median_mhz(clocks) or 1965.0)
    peak_ips = props.multi_processor_count * 4 * sm_hz
    for k in ("p2g", "g2p"):
        if k in ipp and kernels[k]["ms"] > 0:
            bound_ms = 1e3 * ipp[k] * sp.n / peak_ips
            issue[k] = dict(warp_instructions_per_particle=ipp[k], bound_ms=round(bound_ms, 4),
                            achieved=round(ipp[k] * sp.n / (kernels[k]["ms"] / 1e3) / 1e12, 4),
                            peak=round(peak_ips / 1e12, 4), unit="warp instr/ns",
                            frac=round(bound_ms / kernels[k]["ms"], 4))

    # end to end through the C-ABI, the reference's frame loop: host-set velocity
    # conditions (H2D), one substep, positions + damage back to pinned host memory (D2H).
    # The headline form reads with gmpm_read_particles_async into two alternating
    # sets of host buffers, so a step's copy travels while the next step computes;
    # the timed region ends after gmpm_read_wait, when every copy has landed.  The
    # blocking form (gmpm_read_particles, a stall per read) is reported beside it.
    e2e = None
    if not args.no_e2e:
        pos_h = [torch.empty(sp.n * 3, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        dmg_h = [torch.empty(sp.n, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        nsph = sp.desc.n_sphere_bcs
        nslab = sp.desc.n_slab_bcs
        sph_h = torch.empty(max(1, nsph) * 56, dtype=torch.uint8, pin_memory=True)
        slab_h = torch.empty(max(1, nslab) * 48, dtype=torch.uint8, pin_memory=True)
        import ctypes as C
        C.memmove(sph_h.data_ptr(), C.addressof(sp.desc.spheres), max(1, nsph) * 56)
        C.memmove(slab_h.data_ptr(), C.addressof(sp.desc.slabs), max(1, nslab) * 48)

        def frame_loop(overlapped: bool) -> float:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier()
            torch.cuda.synchronize(dev)
            e0.record(stream)
            for i in range(args.steps):
                scene.set_velocity_conditions_raw(slab_h.data_ptr(), nslab, sph_h.data_ptr(), nsph, sh)
                scene.substep(1, sh)
                p, d = pos_h[i & 1], dmg_h[i & 1]
                read = scene.read_into_async if overlapped else scene.read_into
                read("position", p.data_ptr(), p.numel() * 4, order=G.ORDER_INTERNAL, dtype=G.DTYPE_F32, stream=sh)
                read("damage", d.data_ptr(), d.numel() * 4, order=G.ORDER_INTERNAL, dtype=G.DTYPE_F32, stream=sh)
            if overlapped:
                scene.read_wait()
            e1.record(stream)
            e1.synchronize()
            barrier()
            return max_over_ranks(e0.elapsed_time(e1), dist, dev)

        e_ms = frame_loop(True)
        b_ms = frame_loop(False)
        bc_bytes = sizeof_velocity_conditions(np.float32)
        e2e = dict(value=job_rate(world, sp.n, args.steps, e_ms), unit="particle-substeps/s",
                   h2d_bytes_per_step=bc_bytes, d2h_bytes_per_step=sp.n * 16,
                   blocking_value=job_rate(world, sp.n, args.steps, b_ms),
                   note="per step: velocity conditions H2D (pinned), gmpm_substep, positions+damage FP32 D2H "
                        "(pinned) through the C-ABI, as MPMSimulator::simulateStick + Attribs_Back_Host (which "
                        "copies the same two fields as FP64 plus a colour word, 36 B/particle); reads "
                        "overlapped with the next substep (gmpm_read_particles_async, all landed at the end); "
                        "blocking_value: the same loop with gmpm_read_particles")
    return dict(sp=sp, what=what, value=value, ms_max=ms_max, launches=launches, clocks=clocks.summary(), issue=issue,
                kernels=kernels, dom=dom, peaks=peaks, e2e=e2e, status=status, build_s=build_s, diag=diag)


def run_batched(pkg, local_rank: int, steps: int, plain_steps: int, n_scenes: int = 64, seed: int = 0) -> dict:
    """The batched workload: 64 independent notched bars (10k-500k particles,
    log-uniform; parameters within +/-50%; FP32 with FP64 SVD fallback).
    Aggregate particle-substeps/s of the same scenes (a) one at a time through
    the plain path (each scene's substeps, scene after scene) and (b) advanced
    together by one autotuned CUDA-graph launch per substep."""
    import torch

    G = pkg.gmpm
    dev = torch.device("cuda", local_rank)
    ctx = G.Context(local_rank)
    specs = pkg.scenes.notched_bar_batch(n_scenes, seed=seed)
    total = sum(sp.n for sp in specs)
    stream = torch.cuda.Stream(dev)
    sh = stream.cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    plain = [sp.build(ctx) for sp in specs]
    for sc in plain:
        sc.substep(2, sh)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for sc in plain:
        sc.substep(plain_steps, sh)
    e1.record(stream)
    e1.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain_status = max(sc.sync() for sc in plain)
    for sc in plain:
        sc.close()
    del plain

    scenes = [sp.build(ctx) for sp in specs]
    batch = G.Batch(ctx, scenes, autotune=True, trial_substeps=2)
    batch.substep(2, sh)
    tune = batch.info()["n_candidates"] * 2
    batch.substep(tune + 2, sh)
    torch.cuda.synchronize(dev)
    info = batch.info()
    # the scenes' own launches (branch scenes) plus the batch's launches over many scenes
    launches0 = sum(sc.diagnostics()["kernel_launches"] for sc in scenes)
    with ClockSampler(local_rank) as clocks:
        clocks.mark("t0")
        e0.record(stream)
        batch.substep(steps, sh)
        e1.record(stream)
        e1.synchronize()
        clocks.mark("t1")
    b_ms = e0.elapsed_time(e1)
    info = batch.info()
    own = sum(sc.diagnostics()["kernel_launches"] for sc in scenes) - launches0
    launches = own if info["table_scenes"] == 0 else info["kernel_nodes"] * steps
    status = max(sc.sync() for sc in scenes)
    batch.close()
    for sc in scenes:
        sc.close()
    rate = total * steps / (b_ms / 1e3)
    plain_rate = total * plain_steps / (plain_ms / 1e3)
    return dict(value=rate, unit="particle-substeps/s", scenes=n_scenes, particles=total, steps=steps,
                ms_per_step=b_ms / steps, plain_sequential=dict(value=plain_rate, steps=plain_steps,
                                                                ms_per_round=plain_ms / plain_steps),
                speedup_vs_plain=rate / plain_rate, autotune=info, gpu_launches=launches, clocks=clocks.summary(),
                status=pkg.gmpm.STATUS_NAMES.get(max(status, plain_status), max(status, plain_status)),
                workload="64 notched bars, 10k-500k particles log-uniform, params +/-50%, pull U[0.2,1.0] m/s, "
                         "FP32 + FP64 SVD fallback, dx=1/128, 8 ppc")


SERVED_MIX = ("notched bar or plate impact 50/50, 20k-2M particles log-uniform, horizons U[200,2000] substeps, "
              "params +/-50%, 120 GB budget, FP32 + FP64 SVD fallback")


def run_served(pkg, local_rank: int, duration_s: float, rate_hz: float = 20.0, drain_s: float = 0.0,
               plain: bool = True) -> dict:
    """The served workload: Poisson arrivals of notched-bar and plate-impact
    solves (50/50; 20k-2M particles log-uniform; horizons 200-2000 substeps),
    admitted against a 120 GB budget into one continuous batch.  Latency =
    finish - submit of each completed request; the *_all figures also count
    every unfinished request at its age when the run ends (lower bounds)."""
    import torch

    G = pkg.gmpm
    torch.cuda.set_device(local_rank)
    ctx = G.Context(local_rank)
    stream = torch.cuda.Stream(torch.device("cuda", local_rank))
    from gmpm_b200 import serving  # noqa: E402  (package loaded by load_package)
    r = serving.run_served(ctx, duration_s=duration_s, rate_hz=rate_hz, seed=0, stream=stream.cuda_stream,
                           drain_s=drain_s)
    r["workload"] = f"Poisson {rate_hz:g} req/s, " + SERVED_MIX
    if plain:
        p = served_plain_sequential(pkg, ctx, stream)
        r["plain_sequential"] = p
        r["speedup_vs_plain"] = r["particle_substeps_per_s"] / p["value"]
    return r


def served_plain_sequential(pkg, ctx, stream, n_requests: int = 32, substeps: int = 10, seed: int = 0) -> dict:
    """The first requests of the served workload's generator, one at a time
    through the plain path: each scene alone for a fixed number of substeps,
    CUDA events around each scene's substeps, summed."""
    import torch

    prng = np.random.default_rng(seed + 1)  # the served run's request generator
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    work, ms = 0, 0.0
    for k in range(n_requests):
        sp, _ = pkg.scenes.served_request(prng, k)
        sc = sp.build(ctx)
        sc.substep(2, stream.cuda_stream)
        e0.record(stream)
        sc.substep(substeps, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        work += sp.n * substeps
        sc.close()
    return dict(value=work / (ms / 1e3), requests=n_requests, substeps_each=substeps,
                particles=int(work // substeps))


def sizeof_velocity_conditions(dt) -> int:
    # int n_slabs, n_spheres, slab_axis[4]; Real lo[4], hi[4], vel[4][3], c[2][3], r[2], v[2][3]
    r = np.dtype(dt).itemsize
    ints = 4 * (2 + 4)
    reals = r * (4 + 4 + 12 + 6 + 2 + 6)
    return ints + reals


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="plates_33m",
                    choices=["plates_33m", "plates_8m", "notched_bar", "batched64", "served"])
    ap.add_argument("--duration", type=float, default=600.0, help="served workload: seconds of arrivals")
    ap.add_argument("--rate", type=float, default=20.0, help="served workload: arrivals per second")
    ap.add_argument("--drain", type=float, default=0.0,
                    help="served workload: seconds to keep stepping after the last arrival")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-workload object of the line")
    ap.add_argument("--implicit", action="store_true",
                    help="the reference's implicit (Jacobi-PCG) phase field instead of the explicit update")
    ap.add_argument("--no-served", action="store_true", help="skip the served-workload object of the line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-sample", action="store_true",
                    help="reference arm: time the bounded CPU sample instead of the whole workload")
    ap.add_argument("--atomic-p2g", action="store_true",
                    help="P2G's fast mode (shared-memory atomics) instead of the fixed-order, reproducible sums")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    pkg = load_package()

    if args.impl == "reference":
        if rank != 0:
            return
        oracle = load_oracle()
        if args.workload not in WORKLOADS:
            raise SystemExit(f"unknown workload {args.workload}")
        # the whole workload (same configuration as the CUDA arm); timed substeps bounded so the run
        # ends within a few minutes, or the bounded sample with --reference-sample
        r = time_oracle(pkg, oracle, args.workload, args.steps, args.warmup,
                        budget_s=None if args.reference_sample else 120.0, full=not args.reference_sample)
        what = WORKLOADS[args.workload]
        line = dict(metric="particle-substeps/sec", value=r["value"], unit="particle-substeps/s", n_gpus=0,
                    steps=args.steps, warmup=args.warmup, ms_per_step=r["ms_per_step"], higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                    config=dict(workload=what, sample=r["sample"], particles=r["particles"],
                                same_config=not args.reference_sample, timed_steps=r["timed_steps"]),
                    impl="reference",
                    cpu_baseline=dict(value=r["value"], unit=r["unit"], cores=r["cores"], kind=r["kind"],
                                      sample=r["sample"]),
                    e2e=dict(value=r["value"], unit=r["unit"], h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line))
        return

    if args.workload == "batched64":
        if rank != 0:
            return
        import torch
        torch.cuda.set_device(local_rank)
        b = run_batched(pkg, local_rank, steps=args.steps, plain_steps=max(5, args.steps // 4))
        line = dict(metric="particle-substeps/sec", value=b["value"], unit="particle-substeps/s", n_gpus=1,
                    steps=args.steps, warmup=args.warmup, ms_per_step=b["ms_per_step"], higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                    config=dict(workload=b["workload"], particles_per_gpu=b["particles"], scenes=b["scenes"],
                                parallelism="batched scenes, one CUDA graph per substep",
                                l2="resident state larger than L2 (no flush needed)"),
                    plain_sequential=b["plain_sequential"], speedup_vs_plain=b["speedup_vs_plain"],
                    autotune=b["autotune"], gpu_launches=b["gpu_launches"], clocks=b["clocks"], status=b["status"])
        print(json.dumps(line))
        return

    if args.workload == "served":
        if rank != 0:
            return
        r = run_served(pkg, local_rank, args.duration, rate_hz=args.rate, drain_s=args.drain)
        line = dict(metric="particle-substeps/sec", value=r["particle_substeps_per_s"], unit="particle-substeps/s",
                    n_gpus=1, steps=r["substeps"], warmup=0, ms_per_step=None, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
                    config=dict(workload=r["workload"], parallelism="continuous batching"),
                    p50_latency_s=r["p50_latency_s"], p99_latency_s=r["p99_latency_s"],
                    p50_latency_all_s=r["p50_latency_all_s"], p99_latency_all_s=r["p99_latency_all_s"], served=r)
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        res = run_ours(args, pkg, rank, local_rank, world, dist)
    finally:
        pass
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        oracle = load_oracle()
        r = time_oracle(pkg, oracle, args.workload, steps=50, warmup=1, budget_s=20.0)
        cpu = dict(value=r["value"], unit=r["unit"], cores=r["cores"], kind=r["kind"], sample=r["sample"])
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        b = run_batched(pkg, local_rank, steps=30, plain_steps=6)
        batched = {k: b[k] for k in ("value", "unit", "scenes", "particles", "steps", "ms_per_step",
                                     "plain_sequential", "speedup_vs_plain", "gpu_launches", "status", "workload")}
        batched["autotune"] = {k: b["autotune"][k] for k in ("streams", "n_candidates", "sm_share_small",
                                                              "sm_share_medium", "sm_share_large", "graph_nodes",
                                                              "kernel_nodes", "table_scenes")}
    served = sustainable = None
    if rank == 0 and world == 1 and not args.no_served:
        served = run_served(pkg, local_rank, duration_s=20.0)
        # a load the GPU sustains (about two thirds of its capacity on this mix): the queue drains, so
        # every request finishes and p50/p99 are uncensored
        sustainable = run_served(pkg, local_rank, duration_s=30.0, rate_hz=2.0, drain_s=90.0, plain=False)
    if rank == 0:
        sp = res["sp"]
        k = res["kernels"][res["dom"]]
        line = dict(
            metric="particle-substeps/sec", value=res["value"], unit="particle-substeps/s", n_gpus=world,
            steps=args.steps, warmup=args.warmup, ms_per_step=res["ms_max"] / args.steps, higher_is_better=True,
            scaling="weak", vs_baseline=None, dtype="f32", data="synthetic",
            config=dict(workload=res["what"], particles_per_gpu=sp.n, precision="fp32",
                        deterministic_p2g=not args.atomic_p2g,
                        parallelism=f"replicas x{world}" if world > 1 else "single scene",
                        l2="resident state larger than L2 (no flush needed)"),
            roofline=dict(bound="hbm", kernel=res["dom"], achieved=k["achieved_gbs"], peak=res["peaks"]["hbm_gbs"],
                          unit="GB/s", frac=k["frac"], traffic=k["traffic"],
                          peak_source=res["peaks"]["source"]),
            issue_roofline=res["issue"], kernels=res["kernels"], cpu_baseline=cpu, e2e=res["e2e"], clocks=res["clocks"],
            gpu_launches=res["launches"], status=pkg.gmpm.STATUS_NAMES.get(res["status"], res["status"]),
            n_blocks=res["diag"]["n_blocks"], n_grid_blocks=res["diag"]["n_grid_blocks"], batched=batched, served=served,
            served_sustainable=sustainable)
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
