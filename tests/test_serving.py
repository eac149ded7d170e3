"""Continuous-batching server.

CPU: the request trace is a seeded Poisson stream with the stated ranges.
GPU: requests that overlap on the device (several active in one launch,
admitted and retired between rounds) give, each, the same result as the
request tracked alone through the drop-in entry point, bit for bit (same
kernel and arithmetic; the turn counter carries across rounds).
"""
import numpy as np
import pytest

from at_b200 import rings, serving


def test_trace_is_seeded_poisson():
    names = ["a", "b", "c"]
    t1 = serving.make_trace(names, 200, rate_hz=200.0, seed=3)
    t2 = serving.make_trace(names, 200, rate_hz=200.0, seed=3)
    assert [r.arrival for r in t1] == [r.arrival for r in t2]
    arr = np.array([r.arrival for r in t1])
    assert np.all(np.diff(arr) > 0)
    gaps = np.diff(np.concatenate(([0.0], arr)))
    assert 0.5 / 200 < gaps.mean() < 2.0 / 200
    ns = np.array([r.n for r in t1])
    ts = np.array([r.nturns for r in t1])
    assert ns.min() >= 1000 and ns.max() <= 2_000_000
    assert ts.min() >= 100 and ts.max() <= 10_000
    assert {r.kind for r in t1} == {"da", "ma", "bunch"}
    assert all(r.particles.flags.f_contiguous and r.particles.shape == (6, r.n) for r in t1)


@pytest.mark.gpu
def test_served_results_equal_alone():
    from at_b200.tracking import gpupass

    lats, orbits = rings.serving_pool(2, 2)
    reqs = serving.make_trace(list(lats), 10, rate_hz=400.0, seed=5, n_range=(200, 3000),
                              t_range=(10, 120), centre_of=orbits.get)
    srv = serving.TrackingServer(lats, hbm_budget_bytes=1.2e6, round_flops=5e8)
    try:
        srv.serve(reqs)
    finally:
        srv.close()
    assert len(srv.done) == len(reqs)
    assert srv.rounds > 1
    # at least two requests were on the device together
    spans = [(r.admitted, r.finished) for r in reqs]
    overlap = any(a1 < f2 and a2 < f1 for i, (a1, f1) in enumerate(spans)
                  for (a2, f2) in spans[i + 1:])
    assert overlap
    for req in reqs:
        r = np.asfortranarray(req.particles.copy())
        _, ld = gpupass(lats[req.lattice], r, req.nturns, losses=True, mode="fast")
        np.testing.assert_array_equal(req.result, r)
        for k in ("islost", "turn", "elem", "coord"):
            np.testing.assert_array_equal(req.losses[k], ld[k])
    st = serving.latency_stats(reqs)
    assert st["completed"] == len(reqs) and st["p99_s"] >= st["p50_s"] > 0
