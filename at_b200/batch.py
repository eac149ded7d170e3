"""Batched tracking: many lattice variants and particle sets in one launch.

The reference tracks one lattice and one particle array per ``atpass`` call
(``pyat/at.c:340-681``); a study over error-seeded lattice variants is a
Python loop of such calls.  ``BatchTracker`` uploads every variant's table
once, keeps all particle sets in one device buffer, and runs them as the jobs
of a single persistent kernel launch (tiles of the longest jobs first),
recorded once as a CUDA graph and replayed.  Launch parameters (threads per
block, shared-memory segment size) come from the autotuner.
"""
from __future__ import annotations

import numpy as np

from . import autotune
from .engine import Engine, device_info, mode_code
from .lattice import compile_lattice


class BatchTracker:
    """Jobs ``(lattice, particles (6, N_i), nturns_i)`` tracked in one launch.

    ``lattices`` may repeat the same object (it is compiled and uploaded once);
    ``particles`` are host arrays copied to one device buffer.  ``run()``
    tracks every job for its turns and returns the device time; ``results()``
    returns the final coordinates and loss maps per job.
    """

    def __init__(self, lattices, particles, nturns, turn0=0, mode="exact", device: int = 0,
                 tune: bool = True, graph: bool = True, tune_turns: int = 2):
        import torch

        if not (len(lattices) == len(particles) == len(nturns)):
            raise ValueError("lattices, particles and nturns must have the same length")
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.eng = Engine.get(device)
        self.mode = mode_code(mode)
        self.stream = torch.cuda.Stream(self.dev)
        self._lids = {}
        self.lids = []
        self.words = 0
        for lat in lattices:
            k = id(lat)
            if k not in self._lids:
                cl = compile_lattice(lat, getattr(lat, "energy", 0.0),
                                     getattr(getattr(lat, "particle", None), "rest_energy", 0.0))
                self._lids[k] = (self.eng.upload(cl), lat)
                self.words = max(self.words, int(cl.words.size))
            self.lids.append(self._lids[k][0])
        self.sizes = [int(np.asarray(p).shape[1]) for p in particles]
        self.offsets = np.concatenate(([0], np.cumsum(self.sizes))).astype(np.int64)
        ntot = int(self.offsets[-1])
        host = np.zeros((ntot, 6), dtype=np.float64)
        for k, p in enumerate(particles):
            host[self.offsets[k]:self.offsets[k + 1]] = np.asarray(p, dtype=np.float64).T
        self.r0 = host
        self.r = torch.from_numpy(host).to(self.dev)
        self.lost = torch.zeros(ntot, dtype=torch.uint8, device=self.dev)
        self.lturn = torch.zeros(ntot, dtype=torch.int32, device=self.dev)
        self.lelem = torch.zeros(ntot, dtype=torch.int32, device=self.dev)
        self.lcoord = torch.zeros((ntot, 6), dtype=torch.float64, device=self.dev)
        self.nturns = [int(t) for t in nturns]
        self.turn0 = turn0
        self.tuning = None
        if tune:
            self._tune(tune_turns)
        self.bid = self.eng.batch_prepare(self._jobs(self.r, self.lost, self.lturn, self.lelem,
                                                     self.lcoord, self.nturns), self.mode)
        if graph:
            self.eng.batch_capture(self.bid)
        self.graph = graph

    def _jobs(self, r, lost, lturn, lelem, lcoord, nturns):
        jobs = []
        for k, (lid, n, t) in enumerate(zip(self.lids, self.sizes, nturns)):
            o = int(self.offsets[k])
            jobs.append({"lattice_id": lid, "nturns": t, "turn0": self.turn0,
                         "r": r.data_ptr() + 48 * o, "np": n,
                         "losses": (lost.data_ptr() + o, lturn.data_ptr() + 4 * o,
                                    lelem.data_ptr() + 4 * o, lcoord.data_ptr() + 48 * o)})
        return jobs

    def _tune(self, turns):
        torch = self.torch
        scratch = [self.r.clone(), torch.zeros_like(self.lost), torch.zeros_like(self.lturn),
                   torch.zeros_like(self.lelem), torch.zeros_like(self.lcoord)]
        jobs = self._jobs(*scratch, [min(t, turns) for t in self.nturns])

        def sample():
            scratch[0].copy_(self.r)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(self.stream):
                e0.record(self.stream)
                self.eng.track_batch(jobs, self.mode, stream=self.stream.cuda_stream)
                e1.record(self.stream)
            e1.synchronize()
            return e0.elapsed_time(e1) * 1e-3

        name = device_info(self.eng.device)[0]
        key = autotune.cache_key(name, self.words, len(self.lids), int(self.offsets[-1]),
                                 self.mode)
        try:
            self.tuning = autotune.tune(self.eng, sample, key)
        except RuntimeError as exc:
            # another prepared batch pins this engine's launch shape
            self.tuning = {"skipped": str(exc)}

    def run(self) -> float:
        """Track every job for its turns (one persistent launch); returns the
        device time in seconds."""
        torch = self.torch
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            e0.record(self.stream)
            self.eng.batch_launch(self.bid, stream=self.stream.cuda_stream)
            e1.record(self.stream)
        e1.synchronize()
        self.eng.sync(self.stream.cuda_stream)
        return e0.elapsed_time(e1) * 1e-3

    def reset(self):
        """Restore the initial particles and clear the loss maps."""
        self.r.copy_(self.torch.from_numpy(self.r0).to(self.dev))
        for t in (self.lost, self.lturn, self.lelem, self.lcoord):
            t.zero_()
        self.torch.cuda.synchronize(self.dev)

    def particle_turns(self) -> int:
        return int(sum(n * t for n, t in zip(self.sizes, self.nturns)))

    def results(self):
        """[(r (6, N_i) Fortran order, {"islost", "turn", "elem", "coord"})]."""
        r = self.r.cpu().numpy()
        lost = self.lost.cpu().numpy().astype(bool)
        lt = self.lturn.cpu().numpy().view(np.uint32)
        le = self.lelem.cpu().numpy().view(np.uint32)
        lc = self.lcoord.cpu().numpy()
        out = []
        for k in range(len(self.sizes)):
            a, b = int(self.offsets[k]), int(self.offsets[k + 1])
            out.append((np.asfortranarray(r[a:b].T),
                        {"islost": lost[a:b], "turn": lt[a:b], "elem": le[a:b],
                         "coord": np.asfortranarray(lc[a:b].T)}))
        return out

    def close(self):
        if getattr(self, "bid", None) is not None:
            self.eng.batch_free(self.bid)
            self.bid = None
        for lid, _ in self._lids.values():
            self.eng.free(lid)
        self._lids = {}


def partition_jobs(work, ndev: int) -> list[list[int]]:
    """Split jobs of the given ``work`` (e.g. particles x turns x flops per
    particle-turn) over ``ndev`` devices: longest processing time first, each
    job to the device with the least work so far (Graham's LPT rule, within
    4/3 of the optimal makespan).  Returns the job indices of each device in
    ascending order."""
    if ndev < 1:
        raise ValueError("ndev must be at least 1")
    load = [0.0] * ndev
    parts: list[list[int]] = [[] for _ in range(ndev)]
    for k in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        d = min(range(ndev), key=lambda j: (load[j], j))
        parts[d].append(k)
        load[d] += float(work[k])
    return [sorted(p) for p in parts]


class ShardedBatchTracker:
    """The batched workload over several GPUs of one process: the variants
    are split by :func:`partition_jobs` (there is no exchange between them),
    each device runs its share as one :class:`BatchTracker` launch, all
    devices at once from a thread each, and ``results()`` returns every job's
    result in the caller's order."""

    def __init__(self, lattices, particles, nturns, devices, turn0=0, mode="exact",
                 tune: bool = True, graph: bool = True):
        from . import flops

        self.devices = list(devices)
        fpt = {}
        work = []
        for lat, p, t in zip(lattices, particles, nturns):
            k = id(lat)
            if k not in fpt:
                cl = compile_lattice(lat, getattr(lat, "energy", 0.0),
                                     getattr(getattr(lat, "particle", None), "rest_energy",
                                             0.0))
                fpt[k] = flops.flops_per_particle_turn(cl)[0]
            work.append(np.asarray(p).shape[1] * int(t) * fpt[k])
        self.parts = [p for p in partition_jobs(work, len(self.devices))]
        self.trackers = []
        for dev, idx in zip(self.devices, self.parts):
            if not idx:
                self.trackers.append(None)
                continue
            self.trackers.append(BatchTracker([lattices[i] for i in idx],
                                              [particles[i] for i in idx],
                                              [nturns[i] for i in idx], turn0=turn0, mode=mode,
                                              device=dev, tune=tune, graph=graph))

    def _each(self, fn):
        from concurrent.futures import ThreadPoolExecutor
        live = [t for t in self.trackers if t is not None]
        with ThreadPoolExecutor(max_workers=max(1, len(live))) as ex:
            return list(ex.map(fn, live))

    def run(self) -> float:
        """Every device's launch at once; returns the longest device time."""
        return max(self._each(lambda t: t.run()), default=0.0)

    def reset(self):
        self._each(lambda t: t.reset())

    def results(self):
        out = [None] * sum(len(p) for p in self.parts)
        for idx, t in zip(self.parts, self.trackers):
            if t is None:
                continue
            for i, res in zip(idx, t.results()):
                out[i] = res
        return out

    def close(self):
        for t in self.trackers:
            if t is not None:
                t.close()
        self.trackers = []
