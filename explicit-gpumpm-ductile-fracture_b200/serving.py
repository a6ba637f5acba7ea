"""Driver of the served workload: Poisson arrivals of fracture solves into a
gmpm_server (continuous batching), with request latency percentiles and the
aggregate particle-substeps/s.

Arrivals are generated ahead of time by a background thread (the request's
particles are part of the request, not of the server's work); the main thread
submits each request when its arrival time comes, advances the server in
chunks of substeps, and collects finished requests.
"""
from __future__ import annotations

import queue
import threading
import time

import numpy as np

from . import gmpm as G
from . import scenes as S


def run_served(ctx: G.Context, duration_s: float = 600.0, rate_hz: float = 20.0, seed: int = 0,
               lo: int = 20_000, hi: int = 2_000_000, budget_bytes: int = 120 * 10**9, chunk: int = 20,
               max_live: int = 64, stream: int | None = None, drain_s: float = 0.0) -> dict:
    rng = np.random.default_rng(seed)
    # arrival times (Poisson process) over the run
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        arrivals.append(t)
    specs: queue.Queue = queue.Queue(maxsize=64)

    def produce():
        prng = np.random.default_rng(seed + 1)
        for k in range(len(arrivals)):
            specs.put(S.served_request(prng, k, lo, hi))
        specs.put(None)

    threading.Thread(target=produce, daemon=True).start()
    srv = G.Server(ctx, hbm_budget_bytes=budget_bytes, max_live=max_live)
    t0 = time.perf_counter()
    pending = {}  # request id -> (particles, horizon)
    done = []
    submitted = 0
    peak_queue = 0
    nxt = specs.get()
    while True:
        now = time.perf_counter() - t0
        while nxt is not None and submitted < len(arrivals) and arrivals[submitted] <= now:
            sp, horizon = nxt
            rid = srv.submit_spec(sp, horizon)
            pending[rid] = (sp.n, horizon)
            submitted += 1
            nxt = specs.get()
        if now > duration_s + drain_s:
            break
        st = srv.stats()
        peak_queue = max(peak_queue, st["queued"])
        if st["live"] == 0 and st["queued"] == 0:
            if nxt is None or submitted >= len(arrivals):
                break
            time.sleep(min(0.002, max(0.0, arrivals[submitted] - now)))
            continue
        srv.step(chunk, stream)
        for rid in list(pending):
            p = srv.poll(rid)
            if p["state"] in (G.REQUEST_DONE, G.REQUEST_FAILED):
                done.append(dict(latency=p["finish_time"] - p["submit_time"], queue=p["admit_time"] - p["submit_time"],
                                 n=p["n_particles"], horizon=p["horizon"], ok=p["state"] == G.REQUEST_DONE))
                srv.release(rid)
                del pending[rid]
    elapsed = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = np.array([d["latency"] for d in done if d["ok"]]) if done else np.zeros(0)
    return dict(
        duration_s=elapsed, arrivals=len(arrivals), submitted=submitted, completed=int(sum(d["ok"] for d in done)),
        failed=int(sum(not d["ok"] for d in done)), unfinished=len(pending),
        p50_latency_s=float(np.percentile(lat, 50)) if len(lat) else None,
        p99_latency_s=float(np.percentile(lat, 99)) if len(lat) else None,
        mean_queue_s=float(np.mean([d["queue"] for d in done])) if done else None,
        particle_substeps_per_s=st["particle_substeps"] / elapsed, batches=st["batches"],
        capture_s=st["capture_microseconds"] / 1e6, max_live=max_live, peak_queue=peak_queue,
        substeps=st["substeps"], rate_hz=rate_hz, sizes=[lo, hi], horizons=[200, 2000],
        budget_bytes=budget_bytes)
