"""Batched lattice variants (the DA-scan workload) and the autotuner.

CPU: the workload generators are seeded and within their stated ranges.
GPU: every job of one batched launch (replayed from a CUDA graph) equals the
same particles tracked alone through the drop-in entry point, bit for bit
(same kernel and arithmetic; the launch shape does not enter a particle's
arithmetic).
"""
import numpy as np
import pytest

from at_b200 import rings
from conftest import scale_rel_diff


def test_batch_workload_ranges_and_determinism():
    w = rings.batch_workload(256)
    assert w == rings.batch_workload(256)
    seeds = [s for s, _, _ in w]
    assert seeds == list(range(2, 258))
    ns = np.array([n for _, n, _ in w])
    ts = np.array([t for _, _, t in w])
    assert ns.min() >= 1024 and ns.max() <= 16384
    assert ts.min() >= 500 and ts.max() <= 5000
    assert len(set(ns)) > 100


def test_da_grid_layout():
    r = rings.da_grid(1000, seed=4)
    assert r.shape == (6, 1000) and r.flags.f_contiguous
    d = np.round(r[4] - rings.LARGE_ORBIT[4], 12)
    assert set(np.unique(d)) == {-0.03, 0.0, 0.03}
    assert np.all(r[2] - rings.LARGE_ORBIT[2] > 0)


def test_variant_changes_only_errors():
    a = rings.large_ring_variant(2)
    b = rings.large_ring_variant(3)
    assert len(a) == len(b) == len(rings.large_ring())
    assert [e.PassMethod for e in a] == [e.PassMethod for e in b]
    qa = [e for e in a if e.FamName == "QF"][0]
    qb = [e for e in b if e.FamName == "QF"][0]
    assert qa.PolynomB[1] != qb.PolynomB[1]
    assert abs(qa.PolynomB[1] / rings.LARGE_KF - 1) < 1e-2
    assert not np.array_equal(qa.T1, qb.T1)
    # the design (dipole gradients) is seed 1's; only the errors differ
    d1 = [e.PolynomB[1] for e in rings.large_ring(seed=1) if e.FamName == "B"][:7]
    da = [e.PolynomB[1] for e in a if e.FamName == "B"][:7]
    np.testing.assert_allclose(da, d1, rtol=1e-2)


def test_variant_is_stable_on_the_oracle():
    """An error-seeded copy keeps a DA grid's core alive (oracle, 5 turns)."""
    from oracle import oracle
    lat = rings.large_ring_variant(7)
    r = rings.da_grid(60, seed=7, deltas=(0.0,), xmax=1e-3, ymax=5e-4)
    _, ld = oracle.track(lat, r, 5, energy=lat.energy, rest_energy=lat.particle.rest_energy,
                         losses=True)
    assert ld["islost"].mean() < 0.2


@pytest.mark.gpu
def test_batched_variants_equal_individual_runs(tmp_path, monkeypatch):
    monkeypatch.setenv("AT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from at_b200 import tracking
    from at_b200.batch import BatchTracker

    work = rings.batch_workload(6, turn_scale=0.006, seed=1)
    lats = [rings.large_ring_variant(s) for s, _, _ in work]
    parts = [rings.da_grid(max(200, n // 10), seed=s) for s, n, _ in work]
    turns = [t for _, _, t in work]
    bt = BatchTracker(lats, parts, turns, mode="fast", tune=True, graph=True)
    try:
        assert bt.tuning is not None
        bt.run()
        res1 = bt.results()
        bt.reset()
        bt.run()                                   # graph replay
        res2 = bt.results()
    finally:
        bt.close()
    for (ra, la), (rb, lb) in zip(res1, res2):
        np.testing.assert_array_equal(ra, rb)
        np.testing.assert_array_equal(la["islost"], lb["islost"])
    one_per_thread = isinstance(bt.tuning, dict) or bt.tuning[2] == 1
    for (r, ld), lat, p, t in zip(res1, lats, parts, turns):
        ref = p.copy(order="F")
        _, lr = tracking.gpupass(lat, ref, t, losses=True, mode="fast")
        if one_per_thread:
            np.testing.assert_array_equal(r, ref)
        else:   # fast-mode contraction may differ by an ulp with two per thread
            ok = ~lr["islost"]
            assert scale_rel_diff(r[:, ok], ref[:, ok]) <= 2e-13
        for k in ("islost", "turn", "elem") + (("coord",) if one_per_thread else ()):
            np.testing.assert_array_equal(ld[k], lr[k])
    assert any(ld["islost"].any() for _, ld in res1)       # +/-3 % particles get lost
    assert (tmp_path / "tune.json").exists()


@pytest.mark.gpu
def test_refill_claims_give_the_same_results(tmp_path, monkeypatch):
    """Jobs large enough that the launch starts on one block per several
    tiles (refill factor 8, halved to keep two claims per resident block):
    blocks take the rest of each job into the lanes that lost particles free
    at turn boundaries.  Every particle's result and loss record equal the
    run with one claim per tile and the plain drop-in call."""
    monkeypatch.setenv("AT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from at_b200 import tracking
    from at_b200.batch import BatchTracker
    from at_b200.engine import Engine

    lats = [rings.large_ring_variant(s) for s in (2, 3, 4, 5)]
    parts = [rings.da_grid(160000, seed=s) for s in (2, 3, 4, 5)]
    turns = [6, 4, 5, 3]
    eng = Engine.get(0)
    out = {}
    try:
        for k in (1, 8):
            eng.set_launch(threads=256, seg_cap_words=3072, particles_per_thread=1,
                           refill_factor=k)
            bt = BatchTracker(lats, parts, turns, mode="fast", tune=False, graph=True)
            try:
                bt.run()
                out[k] = bt.results()
            finally:
                bt.close()
    finally:
        eng.set_launch(threads=256, seg_cap_words=6144, particles_per_thread=1, refill_factor=8)
    lost = 0
    for (ra, la), (rb, lb) in zip(out[1], out[8]):
        np.testing.assert_array_equal(ra, rb)
        for key in ("islost", "turn", "elem", "coord"):
            np.testing.assert_array_equal(la[key], lb[key])
        lost += int(la["islost"].sum())
    assert 0 < lost < sum(p.shape[1] for p in parts)
    ref = parts[0].copy(order="F")
    _, lr = tracking.gpupass(lats[0], ref, turns[0], losses=True, mode="fast")
    np.testing.assert_array_equal(out[8][0][0], ref)
    np.testing.assert_array_equal(out[8][0][1]["islost"], lr["islost"])


def test_partition_jobs_longest_first_balanced():
    """Variants split over devices (host logic): every job once, each
    device's list ascending, and the LPT makespan within 4/3 of the bound."""
    from at_b200.batch import partition_jobs
    rng = np.random.default_rng(0)
    work = rng.uniform(1.0, 100.0, 257)
    for nd in (1, 2, 3, 8):
        parts = partition_jobs(work, nd)
        assert len(parts) == nd
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(257))
        assert all(p == sorted(p) for p in parts)
        loads = [work[p].sum() for p in parts]
        bound = max(work.sum() / nd, work.max())
        assert max(loads) <= 4.0 / 3.0 * bound
    assert partition_jobs([5.0, 1.0, 1.0, 1.0, 1.0, 1.0], 2) == [[0], [1, 2, 3, 4, 5]]
    with pytest.raises(ValueError):
        partition_jobs([1.0], 0)


@pytest.mark.gpu
def test_sharded_batch_on_one_device_equals_one_batch(tmp_path, monkeypatch):
    """The sharded tracker over a device list (here the one GPU twice:
    two shards, two launches at once) returns, in the caller's order, the
    results of one batched launch."""
    monkeypatch.setenv("AT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from at_b200.batch import BatchTracker, ShardedBatchTracker

    work = rings.batch_workload(5, turn_scale=0.004, seed=2)
    lats = [rings.large_ring_variant(s) for s, _, _ in work]
    parts = [rings.da_grid(max(200, n // 10), seed=s) for s, n, _ in work]
    turns = [t for _, _, t in work]
    one = BatchTracker(lats, parts, turns, mode="exact", tune=False, graph=False)
    try:
        one.run()
        ref = one.results()
    finally:
        one.close()
    sh = ShardedBatchTracker(lats, parts, turns, devices=[0, 0], mode="exact", tune=False,
                             graph=False)
    try:
        assert all(p for p in sh.parts)
        sh.run()
        got = sh.results()
    finally:
        sh.close()
    for (ra, la), (rb, lb) in zip(got, ref):
        np.testing.assert_array_equal(ra, rb)
        for key in ("islost", "turn", "elem", "coord"):
            np.testing.assert_array_equal(la[key], lb[key])
