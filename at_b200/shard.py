"""Particle sharding across GPUs.

Particles are independent, so a bunch is split into contiguous shards, one
per GPU, tracked with no exchange, and the results are concatenated in
order -- the same split and gather as pyat's ``patpass``
(``numpy.array_split`` over the particle axis, ``pyat/at/tracking/track.py:71-88``;
``format_results``, ``pyat/at/tracking/utils.py:118-130``).  Within one
process ``gpupass(gpu_pool=[...])`` drives one engine per device from a
thread each; across processes (one per GPU, ``torch.distributed``) each
rank tracks its shard and the final state is gathered once at the end.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(n: int, nshards: int) -> np.ndarray:
    """Boundaries of ``nshards`` contiguous, nearly equal shards of ``n``
    particles (the sizes of numpy.array_split)."""
    if nshards <= 0:
        raise ValueError("nshards must be positive")
    q, r = divmod(int(n), int(nshards))
    sizes = [q + 1] * r + [q] * (nshards - r)
    return np.concatenate(([0], np.cumsum(sizes))).astype(np.int64)


def local_shard(r: np.ndarray, rank: int, world: int) -> np.ndarray:
    """This rank's (6, n_rank) Fortran-ordered copy of the bunch."""
    b = shard_bounds(r.shape[1], world)
    return np.asfortranarray(r[:, b[rank]:b[rank + 1]])


def gather_shards(local: np.ndarray, group=None) -> np.ndarray:
    """Concatenate every rank's (6, n_rank) result in rank order
    (torch.distributed; works on gloo and nccl)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    n_local = torch.tensor([local.shape[1]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    nmax = int(max(s.item() for s in sizes))
    buf = torch.zeros((nmax, 6), dtype=torch.float64, device=dev)
    buf[: local.shape[1]] = torch.from_numpy(np.ascontiguousarray(local.T)).to(dev)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    parts = [o[: int(s.item())].cpu().numpy().T for o, s in zip(outs, sizes)]
    return np.asfortranarray(np.concatenate(parts, axis=1))


def max_over_ranks(seconds: float, group=None) -> float:
    """Step time of a multi-GPU run: the slowest rank's."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
