"""Multi-process (world size 2, gloo on CPU) coverage of the sharded path.

Each rank tracks its shard of the bunch and the results are gathered in rank
order; the gathered state and loss flags must equal a single-process run
of the whole bunch.  The oracle stands in for the per-GPU engine here (no GPU
on this machine); the shard/gather/timing logic is the product's.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from at_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, results):
    import torch.distributed as dist

    from at_b200 import rings
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ring = rings.fodo_ring()
        r = rings.gaussian(301, seed=5) * 3.0
        mine = shard.local_shard(np.asfortranarray(r), rank, world)
        oracle.track(ring, mine, 40, energy=ring.energy, rest_energy=ring.particle.rest_energy,
                     nthreads=1)
        full = shard.gather_shards(mine)
        t = shard.max_over_ranks(float(rank + 1))
        if rank == 0:
            results.put((np.ascontiguousarray(full), float(t)))
    finally:
        dist.destroy_process_group()


def test_shard_bounds_match_array_split():
    for n in (0, 1, 7, 300, 301):
        for k in (1, 2, 3, 8):
            b = shard.shard_bounds(n, k)
            sizes = [len(a) for a in np.array_split(np.arange(n), k)]
            assert list(np.diff(b)) == sizes


def test_two_rank_gloo_shards_equal_single_process():
    from at_b200 import rings
    from oracle import oracle

    port = _free_port()
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    full, t = results.get(timeout=300)        # rank 0's gathered state
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    g = {"full": full, "t": t}
    ring = rings.fodo_ring()
    ref = np.asfortranarray(rings.gaussian(301, seed=5) * 3.0)
    oracle.track(ring, ref, 40, energy=ring.energy, rest_energy=ring.particle.rest_energy)
    np.testing.assert_array_equal(g["full"], ref)
    assert float(g["t"]) == 2.0
    assert np.isnan(ref[0]).any()          # some particles were lost on the way
