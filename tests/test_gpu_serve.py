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
