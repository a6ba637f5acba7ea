"""Serving loop (gmpm_server): requests admitted under a device-memory budget
as others finish, advanced together, retired at their horizons; each result
equals the same scene run alone (bitwise, deterministic P2G)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEPT = ("position", "velocity", "F", "damage")


def test_served_results_equal_alone(pkg, ctx):
    G, S = pkg.gmpm, pkg.scenes
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(6):
        if k % 2 == 0:
            sp = S.notched_bar_sized(int(rng.integers(8_000, 40_000)), seed=k, pull=float(rng.uniform(0.2, 1.0)))
        else:
            sp = S.plates_sized(int(rng.integers(10_000, 40_000)), seed=k)
        reqs.append((sp, int(rng.integers(10, 40))))
    # a budget that holds about three of these scenes at a time
    srv = G.Server(ctx, hbm_budget_bytes=3 * 60_000_000)
    ids = [srv.submit_spec(sp, h) for sp, h in reqs]
    seen_queued = False
    for _ in range(200):
        st = srv.stats()
        seen_queued |= st["queued"] > 0 and st["live"] > 0
        if st["completed"] + st["failed"] == len(reqs):
            break
        srv.step(7)
    st = srv.stats()
    print("\n[serve]", st)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert seen_queued                     # admission waited for memory
    assert st["batches"] >= 2              # the live set changed
    assert st["particle_substeps"] == sum(sp.n * h for sp, h in reqs)
    for rid, (sp, h) in zip(ids, reqs):
        p = srv.poll(rid)
        assert p["state"] == G.REQUEST_DONE and p["substeps_done"] == h
        assert p["submit_time"] <= p["admit_time"] <= p["finish_time"]
        alone = sp.build(ctx)
        alone.substep(h)
        assert alone.sync() == G.OK
        for f in KEPT:
            a = alone.read(f, dtype=G.DTYPE_F32)
            b = srv.read(rid, f)
            assert np.array_equal(a, b), (sp.name, f)
        alone.close()
        srv.release(rid)
    srv.close()


def test_server_rejects_oversized_request(pkg, ctx):
    G, S = pkg.gmpm, pkg.scenes
    srv = G.Server(ctx, hbm_budget_bytes=1_000_000)
    sp = S.notched_bar_sized(20_000)
    with pytest.raises(G.GmpmError):
        srv.submit_spec(sp, 10)
    srv.close()


def test_served_driver_reports_every_arrival(pkg, ctx):
    """The serving driver's latency covers every arrival: drained at a light
    load nothing is censored; cut off under overload, the unfinished requests
    are counted at their age at the end, so the all-arrival percentiles are
    at least the completed-only ones."""
    from gmpm_b200 import serving  # noqa: E402  (loaded by the pkg fixture)

    light = serving.run_served(ctx, duration_s=2.0, rate_hz=3.0, seed=4, lo=20_000, hi=40_000, drain_s=60.0)
    assert light["arrivals"] > 0 and light["completed"] == light["arrivals"] and light["unfinished"] == 0
    assert light["censored_fraction"] == 0.0
    assert light["p50_latency_all_s"] == pytest.approx(light["p50_latency_s"])
    assert light["p99_latency_all_s"] == pytest.approx(light["p99_latency_s"])
    heavy = serving.run_served(ctx, duration_s=2.0, rate_hz=40.0, seed=5, lo=200_000, hi=400_000)
    assert heavy["unfinished"] > 0
    assert heavy["completed"] + heavy["unfinished"] + heavy["failed"] + heavy["rejected"] == heavy["arrivals"]
    assert heavy["p99_latency_all_s"] >= heavy["unfinished_age_p50_s"] > 0
    # a bounded queue sheds the arrivals that find it full, and counts them
    shed = serving.run_served(ctx, duration_s=2.0, rate_hz=40.0, seed=6, lo=200_000, hi=400_000, max_queue=4)
    assert shed["rejected"] > 0 and shed["submitted"] + shed["rejected"] <= shed["arrivals"]
    assert shed["completed"] + shed["unfinished"] + shed["failed"] + shed["rejected"] == shed["arrivals"]
