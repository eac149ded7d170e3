"""Multi-process (world size 2, gloo on CPU) and multi-device coverage of the
sharded path.

Each rank tracks its shard of the bunch and the results -- final coordinates,
refpts snapshots and the loss map -- are gathered in rank order; they must
equal a single-process run of the whole bunch.  The oracle stands in for the
per-GPU engine here (no GPU on this machine); the shard, gather and timing
logic is the product's.  The in-process multi-device path
(``gpupass(gpu_pool=[...])``) is checked the same way with a stand-in engine
per device.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from at_b200 import shard

NP, NT = 301, 40
REFS = np.array([0, 7, 100], dtype=np.uint32)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _bunch():
    from at_b200 import rings
    return np.asfortranarray(rings.gaussian(NP, seed=5) * 3.0)


def _worker(rank, world, port, results):
    import torch.distributed as dist

    from at_b200 import rings
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ring = rings.fodo_ring()
        mine = shard.local_shard(_bunch(), rank, world)
        rout, ld = oracle.track(ring, mine, NT, refpts=REFS, energy=ring.energy,
                                rest_energy=ring.particle.rest_energy, losses=True, nthreads=1)
        full, full_rout, full_ld = shard.gather_results(mine, rout, ld)
        t = shard.max_over_ranks(float(rank + 1))
        alive, moments = shard.reduce_stats(*_stats(mine, ld))
        if rank == 0:
            results.put((np.ascontiguousarray(full), np.ascontiguousarray(full_rout),
                         {k: np.ascontiguousarray(v) for k, v in full_ld.items()}, float(t),
                         alive, moments))
    finally:
        dist.destroy_process_group()


def _stats(r, ld):
    """Per-turn statistics of a tracked set, as gpupass(stats=True) gives
    them: survivors after each turn (from the loss map) and, per turn, the
    sums and sums of squares of the survivors' final coordinates."""
    alive = np.array([np.sum(~ld["islost"] | (ld["turn"] > t)) for t in range(NT)])
    ok = ~ld["islost"]
    row = np.concatenate([r[:, ok].sum(axis=1), (r[:, ok] ** 2).sum(axis=1)])
    return alive, np.tile(row, (NT, 1))


def _single():
    from at_b200 import rings
    from oracle import oracle
    ring = rings.fodo_ring()
    ref = _bunch()
    rout, ld = oracle.track(ring, ref, NT, refpts=REFS, energy=ring.energy,
                            rest_energy=ring.particle.rest_energy, losses=True)
    return ref, rout, ld


def test_shard_bounds_match_array_split():
    for n in (0, 1, 7, 300, 301):
        for k in (1, 2, 3, 8):
            b = shard.shard_bounds(n, k)
            sizes = [len(a) for a in np.array_split(np.arange(n), k)]
            assert list(np.diff(b)) == sizes


def test_two_rank_gloo_shards_equal_single_process():
    port = _free_port()
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    full, full_rout, full_ld, t, alive, moments = results.get(timeout=300)   # rank 0's
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    ref, rout, ld = _single()
    np.testing.assert_array_equal(full, ref)
    np.testing.assert_array_equal(full_rout, rout)
    assert set(full_ld) == set(ld)
    for k in ld:
        assert full_ld[k].dtype == ld[k].dtype and full_ld[k].shape == ld[k].shape, k
        np.testing.assert_array_equal(full_ld[k], ld[k], err_msg=k)
    assert t == 2.0
    assert ld["islost"].any() and not ld["islost"].all()     # lost and surviving shards
    a1, m1 = _stats(ref, ld)                                  # statistics summed over ranks
    np.testing.assert_array_equal(alive, a1)
    np.testing.assert_allclose(moments, m1, rtol=1e-13, atol=0)


class _OracleEngine:
    """Stand-in for one device's engine: the oracle with Engine.track's
    signature and results."""

    def __init__(self, calls):
        self.calls = calls

    def track(self, lid, r, nturns, turn0=0, start_elem=0, end_elem=0, refpts=None,
              losses=False, stats=False, mode=None, element=False):
        from at_b200 import rings
        from oracle import oracle
        ring = rings.fodo_ring()
        self.calls.append(r.shape[1])
        rout, ld = oracle.track(ring, r, nturns, refpts=refpts, turn=turn0, energy=ring.energy,
                                rest_energy=ring.particle.rest_energy, losses=losses,
                                start_elem=start_elem, end_elem=end_elem, nthreads=1)
        st = None
        if stats:
            alive = np.array([np.sum(~np.isnan(r[0]))] * nturns, dtype=np.uint32)
            st = (alive, np.zeros((nturns, 12)))
        return rout, ld, st


def test_in_process_device_shards_assemble_like_format_results(monkeypatch):
    """gpupass(gpu_pool=[0, 1, 2]) path: three contiguous shards, each on its
    own (stand-in) engine, concatenated into the caller's r_in, rout and loss
    dict exactly as one call over the whole bunch."""
    from at_b200 import engine as _eng
    from at_b200 import tracking

    calls = []
    eng = _OracleEngine(calls)
    monkeypatch.setattr(_eng.Engine, "get", classmethod(lambda cls, d=0: eng))
    monkeypatch.setattr(tracking._state, "lids", {0: 0, 1: 0, 2: 0})
    r = _bunch()
    rout, ld, st = tracking._track_sharded([0, 1, 2], r, NT, 0, 0, 0, REFS, True, True, None)
    ref, rout1, ld1 = _single()
    assert sorted(calls) == [100, 100, 101]
    np.testing.assert_array_equal(r, ref)
    np.testing.assert_array_equal(rout, rout1)
    assert rout.flags.f_contiguous and ld["coord"].flags.f_contiguous
    for k in ld1:
        np.testing.assert_array_equal(ld[k], ld1[k], err_msg=k)
    assert st[0].shape == (NT,)
