"""Continuous-batching servers.

CPU: the request trace is a seeded Poisson stream with the stated ranges.
GPU: requests that overlap on the device give, each, the same result as the
request tracked alone through the drop-in entry point, bit for bit (same
kernel and arithmetic; the turn counter carries across chunks) -- for the
round server (one batched launch per round) and for the device-resident one
(one persistent kernel fed by a host-appended queue).
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


def test_admission_order_shortest_work_first_with_aging():
    """The device-resident server's admission order (host logic, no GPU):
    least work first, requests older than max_wait ahead in arrival order."""
    srv = serving.TrackingServer.__new__(serving.TrackingServer)
    srv.fpt = {"a": 1.0, "b": 10.0}
    srv.policy, srv.max_wait = "sjf", 5.0
    srv.live_work, srv.horizon_s, srv.gpu_flops = 0.0, 1.0, 1.0    # overloaded
    mk = lambda k, lat, n, t, arr: serving.Request(k, lat, np.zeros((6, n)), t, arr)
    srv.waiting = [mk(0, "a", 100, 100, 0.0), mk(1, "b", 10, 10, 1.0), mk(2, "a", 5, 5, 2.0),
                   mk(3, "b", 1000, 1000, 9.0), mk(4, "a", 1, 1, 9.5)]
    assert [r.rid for r in srv._order(now=10.0)] == [0, 1, 2, 4, 3]
    assert [r.rid for r in srv._order(now=6.5)] == [0, 1, 4, 2, 3]
    srv.policy = "fifo"
    assert [r.rid for r in srv._order(now=10.0)] == [0, 1, 2, 3, 4]
    srv.policy, srv.horizon_s = "sjf", 1e8                         # within the horizon
    assert [r.rid for r in srv._order(now=10.0)] == [0, 1, 2, 3, 4]


def _check_alone(lats, reqs, mode):
    from at_b200.tracking import gpupass
    for req in reqs:
        r = np.asfortranarray(req.particles.copy())
        _, ld = gpupass(lats[req.lattice], r, req.nturns, losses=True, mode=mode)
        np.testing.assert_array_equal(req.result, r)
        for k in ("islost", "turn", "elem", "coord"):
            np.testing.assert_array_equal(req.losses[k], ld[k])


def _overlap(reqs):
    spans = [(r.admitted, r.finished) for r in reqs]
    return any(a1 < f2 and a2 < f1 for i, (a1, f1) in enumerate(spans)
               for (a2, f2) in spans[i + 1:])


@pytest.mark.gpu
def test_round_server_results_equal_alone():
    lats, orbits = rings.serving_pool(2, 2)
    reqs = serving.make_trace(list(lats), 10, rate_hz=400.0, seed=5, n_range=(200, 3000),
                              t_range=(10, 120), centre_of=orbits.get)
    srv = serving.RoundServer(lats, hbm_budget_bytes=1.2e6, round_flops=5e8, mode="fast")
    try:
        srv.serve(reqs)
    finally:
        srv.close()
    assert len(srv.done) == len(reqs)
    assert srv.rounds > 1
    assert _overlap(reqs)                   # requests were on the device together
    _check_alone(lats, reqs, "fast")
    st = serving.latency_stats(reqs)
    assert st["completed"] == len(reqs) and st["p99_s"] >= st["p50_s"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_device_resident_server_results_equal_alone(mode):
    """The persistent serving kernel: requests are published into the running
    launch as they arrive (no round barrier), each tile advances by chunks of
    turns through the device-side continuation queue, and each result equals
    the request tracked alone, bit for bit."""
    lats, orbits = rings.serving_pool(2, 2)
    reqs = serving.make_trace(list(lats), 14, rate_hz=300.0, seed=6, n_range=(200, 4000),
                              t_range=(10, 150), centre_of=orbits.get)
    srv = serving.TrackingServer(lats, hbm_budget_bytes=2e6, chunk_flops=1e8, mode=mode)
    try:
        srv.serve(reqs)
        c = srv.counters()
        jobs = srv.jobs
    finally:
        srv.close()
    assert len(srv.done) == len(reqs) == jobs           # one job per request
    assert c["claimed"] == c["published"]
    assert c["resumed"] == c["requeued"] > c["published"]   # tiles ran in several chunks
    assert _overlap(reqs)
    _check_alone(lats, reqs, mode)


@pytest.mark.gpu
@pytest.mark.parametrize("pack", [True, False])
def test_device_resident_chunks_keep_results_with_losses(pack):
    """Chunks of one turn on a bunch that loses particles along the way: the
    loss turn, element and coordinates carry over from chunk to chunk, with
    the tiles packed to their live particles at every chunk end or not."""
    lats, orbits = rings.serving_pool(1, 1)
    reqs = serving.make_trace(list(lats), 3, rate_hz=1000.0, seed=11, n_range=(600, 1500),
                              t_range=(40, 60), centre_of=orbits.get)
    for r in reqs:                                          # far out: losses over many turns
        c = orbits[r.lattice][[0, 2], None]
        r.particles[[0, 2]] = c + 6.0 * (r.particles[[0, 2]] - c)
    srv = serving.TrackingServer(lats, chunk_flops=1.0, pack=pack)   # one turn per claim
    try:
        srv.serve(reqs)
        c = srv.counters()
    finally:
        srv.close()
    assert len(srv.done) == 3
    assert c["requeued"] > 10 * c["published"]
    assert any(r.losses["islost"].any() and not r.losses["islost"].all() for r in reqs)
    _check_alone(lats, reqs, "exact")


@pytest.mark.gpu
def test_device_resident_server_survives_idle_gaps():
    """Arrivals separated by more than the kernel's idle time: the kernel
    leaves while the queue is empty and the next submit launches it again."""
    lats, orbits = rings.serving_pool(1, 1)
    reqs = serving.make_trace(list(lats), 3, rate_hz=1.0, seed=8, n_range=(500, 800),
                              t_range=(5, 10), centre_of=orbits.get)
    for k, r in enumerate(reqs):
        r.arrival = 0.45 * k                 # gaps of 0.45 s > 0.2 s idle limit
    srv = serving.TrackingServer(lats, chunk_flops=1e12)
    try:
        srv.serve(reqs)
    finally:
        srv.close()
    assert len(srv.done) == 3
    _check_alone(lats, reqs, "exact")


def test_sharded_server_deals_requests_to_the_least_loaded():
    """Host logic of the one-server-per-GPU dispatcher, on stand-in servers:
    each arrival goes to the server with the least work outstanding."""
    class Stub:
        def __init__(self):
            self.waiting, self.staging, self.active = [], [], []
            self.fpt = {"a": 1.0}

        def _work(self, r):
            return r.n * r.nturns * self.fpt[r.lattice]

    sh = serving.ShardedTrackingServer.__new__(serving.ShardedTrackingServer)
    sh.servers = [Stub(), Stub(), Stub()]
    mk = lambda k, n, t: serving.Request(k, "a", np.zeros((6, n)), t, 0.0)
    got = [sh.servers.index(sh._assign(mk(k, n, t)))
           for k, (n, t) in enumerate([(100, 10), (10, 10), (10, 10), (50, 1), (10, 1)])]
    assert got == [0, 1, 2, 1, 2]          # loads 1000 / 150 / 110 at the end
    assert [len(s.waiting) for s in sh.servers] == [1, 2, 2]


@pytest.mark.gpu
def test_sharded_server_on_one_device_equals_alone():
    lats, orbits = rings.serving_pool(1, 1)
    reqs = serving.make_trace(list(lats), 6, rate_hz=300.0, seed=12, n_range=(200, 2000),
                              t_range=(10, 60), centre_of=orbits.get)
    sh = serving.ShardedTrackingServer(lats, [0], chunk_flops=1e8)
    try:
        sh.serve(reqs)
        done = sh.done
    finally:
        sh.close()
    assert len(done) == len(reqs)
    _check_alone(lats, reqs, "exact")


@pytest.mark.gpu
def test_device_resident_queue_classes_equal_alone():
    """With continuations queued by remaining time (eight device rings, taken
    lowest first) every result still equals the request tracked alone."""
    lats, orbits = rings.serving_pool(1, 1)
    reqs = serving.make_trace(list(lats), 8, rate_hz=400.0, seed=13, n_range=(200, 3000),
                              t_range=(10, 120), centre_of=orbits.get)
    srv = serving.TrackingServer(lats, chunk_flops=1e8, classes=True)
    try:
        srv.serve(reqs)
        c = srv.counters()
    finally:
        srv.close()
    assert len(srv.done) == len(reqs)
    assert c["resumed"] == c["requeued"] > c["published"]
    _check_alone(lats, reqs, "exact")
