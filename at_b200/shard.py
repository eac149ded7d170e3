"""Particle sharding across GPUs.

Particles are independent, so a bunch is split into contiguous shards, one
per GPU, tracked with no exchange, and the results are concatenated in
order -- the same split and gather as pyat's ``patpass``
(``numpy.array_split`` over the particle axis, ``pyat/at/tracking/track.py:71-88``;
``format_results``, ``pyat/at/tracking/utils.py:118-130``).  Within one
process ``gpupass(gpu_pool=[...])`` drives one engine per device from a
thread each; across processes (one per GPU, ``torch.distributed``) each
rank tracks its shard and the results (final state, refpts snapshots, loss
map) are gathered once at the end.
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


def _device(group):
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_along(arr: np.ndarray, axis: int, group=None) -> np.ndarray:
    """Every rank's ``arr`` concatenated along ``axis`` (the particle axis) in
    rank order; the other dimensions must agree.  Ranks may hold different
    particle counts (their rows are padded for one all_gather).  Works on gloo
    and nccl; bool and unsigned arrays travel as wider signed integers."""
    import torch
    import torch.distributed as dist

    a = np.moveaxis(np.asarray(arr), axis, 0)
    n, rest = a.shape[0], a.shape[1:]
    width = int(np.prod(rest)) if rest else 1
    wire = {np.dtype(bool): np.uint8, np.dtype(np.uint32): np.int64,
            np.dtype(np.uint16): np.int32}.get(a.dtype, a.dtype)
    dev = _device(group)
    world = dist.get_world_size(group)
    n_local = torch.tensor([n], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    counts = [int(c.item()) for c in sizes]
    rows = torch.from_numpy(np.ascontiguousarray(a.reshape(n, width).astype(wire)))
    buf = torch.zeros((max(counts + [1]), width), dtype=rows.dtype, device=dev)
    buf[:n] = rows.to(dev)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    full = np.concatenate([o[:c].cpu().numpy() for o, c in zip(outs, counts)], axis=0)
    full = full.astype(a.dtype).reshape((sum(counts),) + rest)
    return np.moveaxis(full, 0, axis)


def gather_shards(local: np.ndarray, group=None) -> np.ndarray:
    """Concatenate every rank's (6, n_rank) final coordinates in rank order."""
    return np.asfortranarray(gather_along(local, 1, group))


def gather_results(r: np.ndarray, rout: np.ndarray | None = None, losses: dict | None = None,
                   group=None):
    """All of one sharded tracking call, assembled as the reference's
    ``format_results`` does for its process pool
    (pyat/at/tracking/utils.py:118-130): the final coordinates (6, N), the
    refpts snapshots (6, N, R, T) and every loss-map key, each concatenated
    along its particle axis in rank order.  Returns (r, rout, losses)."""
    full_r = gather_shards(r, group)
    full_rout = None if rout is None else np.asfortranarray(gather_along(rout, 1, group))
    full_ld = None
    if losses is not None:
        full_ld = {}
        for k in losses:
            v = np.asarray(losses[k])
            ax = v.ndim - 1                      # (N,) flags and turns, (6, N) coordinates
            full_ld[k] = gather_along(v, ax, group)
        if "coord" in full_ld:
            full_ld["coord"] = np.asfortranarray(full_ld["coord"])
    return full_r, full_rout, full_ld


def reduce_stats(alive: np.ndarray, moments: np.ndarray, group=None):
    """The per-turn statistics of a sharded call (``gpupass(stats=True)``)
    summed over ranks in ONE all-reduce: survivor counts (T,) and the twelve
    coordinate sums and sums of squares per turn (T, 12), from which the
    bunch's mean and rms follow.  Counts travel as float64 (exact below
    2**53).  Returns (alive (T,) int64, moments (T, 12) float64)."""
    import torch
    import torch.distributed as dist

    a = np.asarray(alive, dtype=np.float64).reshape(-1)
    m = np.asarray(moments, dtype=np.float64).reshape(a.size, 12)
    buf = torch.from_numpy(np.concatenate([a[:, None], m], axis=1)).to(_device(group))
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return out[:, 0].astype(np.int64), np.ascontiguousarray(out[:, 1:])


def max_over_ranks(seconds: float, group=None) -> float:
    """Step time of a multi-GPU run: the slowest rank's."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([seconds], dtype=torch.float64, device=_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
