"""Driver of the served workload: Poisson arrivals of fracture solves into a
gmpm_server (continuous batching), with request latency percentiles and the
aggregate particle-substeps/s.

Latency is reported over every accepted arrival, not only the requests that
finished: a request still queued or running when the run ends is counted at
its age then (a lower bound on its latency; "censored"), and one never
submitted is counted at the time left after its arrival.  With drain_s > 0
the loop keeps stepping after the last arrival until every request has
finished (or drain_s has passed), so that at a sustainable load no latency is
censored.

The queue is bounded (max_queue): an arrival that finds max_queue requests
waiting is rejected and counted, as a server sheds load under overload.
Every queued request holds its particle arrays in host memory, so without a
bound an overloaded run grows without limit; a rejected request's particles
are never generated.

A producer thread generates each request (its particles are part of the
request, not of the server's work) and submits it at its arrival time; the
main thread advances the server in chunks of substeps and collects finished
requests.  The server accepts submissions while it is being stepped.
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
               max_live: int = 64, stream: int | None = None, drain_s: float = 0.0,
               max_queue: int = 256) -> dict:
    rng = np.random.default_rng(seed)
    # arrival times (Poisson process) over the run
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        arrivals.append(t)
    srv = G.Server(ctx, hbm_budget_bytes=budget_bytes, max_live=max_live)
    submitted: queue.Queue = queue.Queue()
    t0 = time.perf_counter()
    submit_s = [0.0]
    rejected = [0]

    def produce():
        # draws each request, generates its particles if the queue has room when
        # it arrives, and submits it on time (the server accepts submissions while
        # another thread steps it)
        prng = np.random.default_rng(seed + 1)
        for k, t_arr in enumerate(arrivals):
            params = S.served_request_params(prng, lo, hi)
            wait = t_arr - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            if max_queue > 0 and srv.stats()["queued"] >= max_queue:
                rejected[0] += 1
                submitted.put(-1)
                continue
            sp, horizon = S.served_request_build(params, k)
            t1 = time.perf_counter()
            rid = srv.submit_spec(sp, horizon)
            submit_s[0] += time.perf_counter() - t1
            submitted.put(rid)
        submitted.put(None)

    producer = threading.Thread(target=produce, daemon=True)
    producer.start()
    pending = set()
    done = []
    n_submitted = 0
    n_handled = 0  # arrivals the producer has submitted or rejected
    producer_done = False
    peak_queue = 0
    step_s = poll_s = 0.0
    while True:
        while True:
            try:
                rid = submitted.get_nowait()
            except queue.Empty:
                break
            if rid is None:
                producer_done = True
                continue
            n_handled += 1
            if rid >= 0:
                pending.add(rid)
                n_submitted += 1
        now = time.perf_counter() - t0
        if now > duration_s + drain_s:
            break
        st = srv.stats()
        peak_queue = max(peak_queue, st["queued"])
        if st["live"] == 0 and st["queued"] == 0:
            if producer_done and not pending:
                break
            time.sleep(0.001)
            continue
        t1 = time.perf_counter()
        srv.step(chunk, stream)
        t2 = time.perf_counter()
        step_s += t2 - t1
        for rid in list(pending):
            p = srv.poll(rid)
            if p["state"] in (G.REQUEST_DONE, G.REQUEST_FAILED):
                done.append(dict(latency=p["finish_time"] - p["submit_time"], queue=p["admit_time"] - p["submit_time"],
                                 n=p["n_particles"], horizon=p["horizon"], ok=p["state"] == G.REQUEST_DONE))
                srv.release(rid)
                pending.discard(rid)
        poll_s += time.perf_counter() - t2
    elapsed = time.perf_counter() - t0
    # requests left at the end: their age on the server's clock (a lower bound on their latency)
    ages = []
    for rid in pending:
        p = srv.poll(rid)
        ages.append(max(0.0, elapsed - p["submit_time"]))
    # arrivals the producer had not reached: the time since their arrival
    ages += [max(0.0, elapsed - t_arr) for t_arr in arrivals[n_handled:]]
    st = srv.stats()
    srv.close()
    lat = np.array([d["latency"] for d in done if d["ok"]]) if done else np.zeros(0)
    everyone = np.concatenate([lat, np.array(ages)])

    def pct(a, q):
        return float(np.percentile(a, q)) if len(a) else None

    return dict(
        duration_s=elapsed, arrivals=len(arrivals), submitted=n_submitted, rejected=rejected[0],
        rejected_fraction=float(rejected[0] / max(1, len(arrivals))), max_queue=max_queue,
        completed=int(sum(d["ok"] for d in done)), failed=int(sum(not d["ok"] for d in done)), unfinished=len(ages),
        p50_latency_s=pct(lat, 50), p99_latency_s=pct(lat, 99),
        # over every arrival, unfinished ones censored at their age at the end (lower bounds)
        p50_latency_all_s=pct(everyone, 50), p99_latency_all_s=pct(everyone, 99),
        unfinished_age_p50_s=pct(np.array(ages), 50), unfinished_age_p99_s=pct(np.array(ages), 99),
        censored_fraction=float(len(ages) / max(1, len(arrivals) - rejected[0])),
        mean_queue_s=float(np.mean([d["queue"] for d in done])) if done else None,
        particle_substeps_per_s=st["particle_substeps"] / elapsed, batches=st["batches"],
        capture_s=st["capture_microseconds"] / 1e6, admit_s=st["admit_microseconds"] / 1e6,
        retire_s=st["retire_microseconds"] / 1e6, launch_s=st["launch_microseconds"] / 1e6,
        step_s=step_s, poll_s=poll_s, submit_s=submit_s[0], max_live=max_live, peak_queue=peak_queue,
        substeps=st["substeps"], rate_hz=rate_hz, sizes=[lo, hi], horizons=[200, 2000],
        budget_bytes=budget_bytes)
