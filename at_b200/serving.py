"""Continuous-batching tracking server.

Requests (a lattice, a particle set, a turn count) arrive over time.  The
server keeps every admitted request's particles in HBM (admitted in arrival
order under an HBM budget, smaller requests allowed to pass a head that does
not fit) and advances all of them together.

``TrackingServer`` is device-resident: ONE persistent kernel
(``atb_serve_*``) claims tiles from a queue that the host appends to while it
runs.  A request joins as soon as its particles are in HBM -- its tiles are
published into the running launch -- and is one job for all its turns.  A
tile runs a chunk of turns per claim (a few tens of ms of one block's work)
and then puts itself back in a device-side continuation ring that the blocks
take from after new work, so long requests share the GPU with short ones
tile by tile (processor sharing) with no host step and no barrier between
chunks.  Admission copies and result copies run on a side stream (copy
engine) beside the kernel.  By default ("sjf") requests are admitted in
arrival order while the admitted and waiting work would take the GPU at
most ``horizon_s`` seconds, so a burst the GPU can absorb is admitted whole
and shared tile by tile; beyond that (overload) admission takes the waiting
requests with the least work first (any request that has waited longer than
``max_wait`` goes ahead of them) and only while fewer than ``waves`` waves of
the persistent grid's tiles are in flight, so the short requests run first
and finish instead of every request sharing the GPU and few finishing.  With ``classes=True`` re-enqueued tiles wait in one of eight
device queues by the decade of their remaining time instead of one (measured
slower on the bench traces, kept as an option).  ``RoundServer`` is the earlier form: one
``atb_track_batch`` launch per round over every active request, new arrivals
joining at the next round.

Either way the absolute turn counter carries over from chunk to chunk, so
the RF phase is the same as in one long call and a request's result is the
one it gets alone.  The reference has no serving layer: each request would be
one blocking ``atpass`` call (``pyat/at.c:340-681``); ``serve_sequential``
runs a trace that way through the drop-in entry point, for comparison.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import flops
from .engine import Engine, mode_code
from .lattice import compile_lattice
from .tracking import gpupass

BYTES_PER_PARTICLE = 48 + 1 + 4 + 4 + 48 + 4  # state + loss map + particle index


@dataclass
class Request:
    rid: int
    lattice: str
    particles: np.ndarray           # (6, N) Fortran order (host)
    nturns: int
    arrival: float                  # seconds from the start of the trace
    kind: str = "bunch"
    # filled by the server
    admitted: float | None = None
    finished: float | None = None
    result: np.ndarray | None = None
    losses: dict | None = None
    done_turns: int = 0
    dev: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.particles.shape[1])

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class RoundServer:
    """Continuous batching at round granularity (one batched launch per
    round)."""

    def __init__(self, lattices: dict, hbm_budget_bytes: float = 150e9, device: int = 0,
                 mode="exact", round_flops: float = 2e12, max_chunk: int = 512):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.eng = Engine.get(device)
        self.mode = mode_code(mode)
        self.budget = float(hbm_budget_bytes)
        self.round_flops = float(round_flops)
        self.max_chunk = int(max_chunk)
        self.stream = torch.cuda.Stream(self.dev)
        self.lids = {}
        self.fpt = {}
        for name, lat in lattices.items():
            cl = compile_lattice(lat, getattr(lat, "energy", 0.0),
                                 getattr(getattr(lat, "particle", None), "rest_energy", 0.0))
            self.lids[name] = self.eng.upload(cl)
            self.fpt[name] = flops.flops_per_particle_turn(cl)[0]
        self.waiting: list[Request] = []
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.used = 0.0
        self.rounds = 0
        self.particle_turns = 0

    # -- admission / retirement ------------------------------------------------
    def _admit(self, now: float):
        torch = self.torch
        keep = []
        for req in self.waiting:
            need = req.n * BYTES_PER_PARTICLE
            if self.used + need <= self.budget:
                n = req.n
                req.dev = {
                    "r": torch.from_numpy(np.ascontiguousarray(req.particles.T)).to(self.dev),
                    "lost": torch.zeros(n, dtype=torch.uint8, device=self.dev),
                    "lturn": torch.zeros(n, dtype=torch.int32, device=self.dev),
                    "lelem": torch.zeros(n, dtype=torch.int32, device=self.dev),
                    "lcoord": torch.zeros((n, 6), dtype=torch.float64, device=self.dev),
                }
                self.used += need
                req.admitted = now
                self.active.append(req)
            else:
                keep.append(req)
        self.waiting = keep

    def _retire(self, now: float):
        still = []
        for req in self.active:
            if req.done_turns >= req.nturns:
                d = req.dev
                req.result = np.asfortranarray(d["r"].cpu().numpy().T)
                req.losses = {"islost": d["lost"].cpu().numpy().astype(bool),
                              "turn": d["lturn"].cpu().numpy().view(np.uint32),
                              "elem": d["lelem"].cpu().numpy().view(np.uint32),
                              "coord": np.asfortranarray(d["lcoord"].cpu().numpy().T)}
                req.dev = {}
                req.finished = now
                self.used -= req.n * BYTES_PER_PARTICLE
                self.done.append(req)
            else:
                still.append(req)
        self.active = still

    # -- one round ---------------------------------------------------------------
    def _round(self):
        cost = sum(r.n * self.fpt[r.lattice] for r in self.active)
        chunk = int(max(1, min(self.max_chunk, self.round_flops // max(cost, 1))))
        jobs = []
        for req in self.active:
            t = min(chunk, req.nturns - req.done_turns)
            d = req.dev
            jobs.append({"lattice_id": self.lids[req.lattice], "nturns": t,
                         "turn0": req.done_turns, "r": d["r"].data_ptr(), "np": req.n,
                         "losses": (d["lost"].data_ptr(), d["lturn"].data_ptr(),
                                    d["lelem"].data_ptr(), d["lcoord"].data_ptr())})
            req._step = t
        with self.torch.cuda.stream(self.stream):
            self.eng.track_batch(jobs, self.mode, stream=self.stream.cuda_stream)
        self.stream.synchronize()
        self.eng.sync(self.stream.cuda_stream)
        for req in self.active:
            req.done_turns += req._step
            self.particle_turns += req.n * req._step
        self.rounds += 1

    def serve(self, requests: list[Request], time_limit: float | None = None):
        """Replay a trace: request k becomes visible at ``arrival`` seconds after
        the start; rounds run back to back while there is work.  Returns the
        wall time of the whole trace."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        i = 0
        while i < len(pending) or self.waiting or self.active:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                self.waiting.append(pending[i])
                i += 1
            self._admit(now)
            if self.active:
                self._round()
                self._retire(time.perf_counter() - t0)
            elif i < len(pending):
                time.sleep(max(0.0, min(0.01, pending[i].arrival - now)))
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
        return time.perf_counter() - t0

    def close(self):
        for lid in self.lids.values():
            self.eng.free(lid)
        self.lids = {}


class TrackingServer:
    """Device-resident continuous batching over one persistent kernel."""

    def __init__(self, lattices: dict, hbm_budget_bytes: float = 150e9, device: int = 0,
                 mode="exact", chunk_flops: float = 1e9, max_chunk: int = 512,
                 max_jobs: int = 1 << 16, max_tiles: int = 1 << 22, policy: str = "sjf",
                 horizon_s: float = 30.0, max_wait: float = 30.0, pack: bool = True,
                 classes: bool = False, waves: float = 4.0):
        import ctypes as C

        import torch

        from . import _lib

        self.C = C
        self.lib = _lib.lib()
        self.check = _lib.check
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.eng = Engine.get(device)
        self.mode = mode_code(mode)
        self.budget = float(hbm_budget_bytes)
        self.chunk_flops = float(chunk_flops)
        self.max_chunk = int(max_chunk)
        self.copy = torch.cuda.Stream(self.dev)           # admission and result copies
        self.lids, self.fpt = {}, {}
        for name, lat in lattices.items():
            cl = compile_lattice(lat, getattr(lat, "energy", 0.0),
                                 getattr(getattr(lat, "particle", None), "rest_energy", 0.0))
            self.lids[name] = self.eng.upload(cl)
            self.fpt[name] = flops.flops_per_particle_turn(cl)[0]
        ids = (C.c_int32 * len(self.lids))(*self.lids.values())
        self.srv = C.c_void_p()
        self.check(self.lib.atb_serve_open(self.eng.h, ids, len(self.lids), self.mode,
                                           int(max_jobs), int(max_tiles), C.byref(self.srv)))
        self.waiting: list[Request] = []
        self.staging: list[Request] = []      # admitted, particles on their way to HBM
        self.active: list[Request] = []       # a chunk in the queue
        self.retiring: list[Request] = []     # results on their way back
        self.done: list[Request] = []
        self.used = 0.0
        self.jobs = 0                         # queue slots used
        self.particle_turns = 0
        if policy not in ("sjf", "fifo"):
            raise ValueError("policy must be 'sjf' or 'fifo'")
        self.policy = policy
        self.max_wait = float(max_wait)
        #: algorithmic flops the GPU tracks per second in this arithmetic (the
        #: large-ring bench rates: exact 10 TFLOP/s, fast 24 TFLOP/s), and the
        #: admission horizon: under "sjf" nothing more is admitted while the
        #: admitted, unfinished work would take longer than horizon_s
        self.gpu_flops = 1.0e13 if mode_code(mode) == mode_code("exact") else 2.4e13
        self.horizon_s = float(horizon_s)
        self.live_work = 0.0
        sms = torch.cuda.get_device_properties(self.dev).multi_processor_count
        #: under overload, tiles in flight (admitted, not finished) above which
        #: nothing more is admitted: a few waves of the persistent grid (two
        #: blocks per SM)
        self.max_live_tiles = int(waves * 2 * sms)
        self.live_tiles = 0
        self.classes = bool(classes)
        #: re-enqueued tiles keep only their live particles (a per-request
        #: particle index, filled from a pinned 0..n-1 on the copy stream)
        self.pack = bool(pack)
        self._iota = torch.empty(0, dtype=torch.int32)

    # -- admission ----------------------------------------------------------------
    def _work(self, req) -> float:
        return req.n * req.nturns * self.fpt[req.lattice]

    def _overloaded(self) -> bool:
        """The admitted, unfinished work plus the waiting work would take the
        GPU longer than the horizon."""
        total = self.live_work + sum(self._work(r) for r in self.waiting)
        return total > self.horizon_s * self.gpu_flops

    def _order(self, now: float) -> list:
        """Admission order.  "fifo", and "sjf" while the GPU is not
        overloaded: arrival order.  "sjf" under overload: requests that have
        waited longer than ``max_wait`` first (in arrival order), then the
        others by increasing work (N x T x flops per particle-turn), which
        keeps short requests from queueing behind long ones when the offered
        load exceeds the GPU."""
        if self.policy == "fifo" or not self._overloaded():
            return list(self.waiting)
        old = [r for r in self.waiting if now - r.arrival > self.max_wait]
        new = sorted((r for r in self.waiting if now - r.arrival <= self.max_wait),
                     key=self._work)
        return old + new

    #: flops of one particle-turn that count as one unit of tile time
    TURN_UNIT = 2e5

    def _turn_cost(self, req) -> float:
        """Relative cost of one turn of the request's lattice (a FODO turn is
        about 1, a large-ring turn 10).  With classes a re-enqueued tile waits
        in the device queue of the decade of (turns left) x this cost, so the
        tiles closest to their end -- what bounds a request's latency, as a
        tile needs all its turns whatever the particle count -- go first.
        0 (one queue, round robin) unless the server was opened with
        ``classes=True``."""
        if not self.classes:
            return 0.0
        return max(self.fpt[req.lattice] / self.TURN_UNIT, 1e-3)

    def _tiles(self, req) -> int:
        return (req.n + self.TILE - 1) // self.TILE

    def _admit(self, now: float):
        """Admit waiting requests (particles copied to HBM on the side stream)
        while the HBM budget holds and, under "sjf" when overloaded, while
        fewer than ``max_live_tiles`` tiles are in flight (one request is
        always admitted into an idle server)."""
        torch = self.torch
        keep = []
        capped = self.policy == "sjf" and self._overloaded()
        for req in self._order(now):
            need = req.n * BYTES_PER_PARTICLE
            busy = self.live_tiles > 0
            over = capped and busy and self.live_tiles + self._tiles(req) > self.max_live_tiles
            if self.used + need > self.budget or over:
                keep.append(req)
                continue
            n = req.n
            host = {"r": torch.from_numpy(np.ascontiguousarray(req.particles.T)).pin_memory(),
                    "lost": torch.zeros(n, dtype=torch.uint8).pin_memory(),
                    "lturn": torch.zeros(n, dtype=torch.int32).pin_memory(),
                    "lelem": torch.zeros(n, dtype=torch.int32).pin_memory(),
                    "lcoord": torch.zeros((n, 6), dtype=torch.float64).pin_memory()}
            d = {k: torch.empty(v.shape, dtype=v.dtype, device=self.dev) for k, v in host.items()}
            if self.pack:
                if self._iota.numel() < n:
                    self._iota = torch.arange(max(n, 2 * self._iota.numel()),
                                              dtype=torch.int32).pin_memory()
                d["pidx"] = torch.empty(n, dtype=torch.int32, device=self.dev)
            with torch.cuda.stream(self.copy):
                for k in host:
                    d[k].copy_(host[k], non_blocking=True)    # copy engine, beside the kernel
                if self.pack:
                    d["pidx"].copy_(self._iota[:n], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.copy)
            req.dev, req._host, req._event = d, host, ev
            self.used += need
            self.live_work += self._work(req)
            self.live_tiles += self._tiles(req)
            req.admitted = now
            self.staging.append(req)
        self.waiting = sorted(keep, key=lambda r: r.arrival)

    TILE = 256                                # particles per tile (the kernel's block)

    def _chunk(self, req) -> int:
        """Turns a tile runs per claim: about ``chunk_flops`` of work (a few
        tens of ms on one block), so a tile of a long request goes back to
        the device queue often enough for newer requests' tiles to start."""
        per = min(req.n, self.TILE) * self.fpt[req.lattice]
        return int(max(1, min(self.max_chunk, req.nturns, self.chunk_flops // max(per, 1.0))))

    def _submit(self, req):
        C = self.C
        from ._lib import AtbJobDesc
        d = req.dev
        jd = AtbJobDesc()
        jd.lattice_id = self.lids[req.lattice]
        jd.nturns = req.nturns
        jd.turn0 = 0
        jd.losses = 1
        jd.r = d["r"].data_ptr()
        jd.np = req.n
        jd.islost, jd.lturn = d["lost"].data_ptr(), d["lturn"].data_ptr()
        jd.lelem, jd.lcoord = d["lelem"].data_ptr(), d["lcoord"].data_ptr()
        slot = C.c_int32(-1)
        pidx = d["pidx"].data_ptr() if "pidx" in d else None
        self.check(self.lib.atb_serve_submit(self.srv, C.byref(jd), self._chunk(req),
                                             self._turn_cost(req), pidx, C.byref(slot)))
        req._slot = slot.value
        self.jobs = slot.value + 1

    # -- progress -------------------------------------------------------------------
    def _poll(self) -> int:
        """Publish staged requests and start the result copy of every request
        whose particles are all done; returns how many moved."""
        C, torch = self.C, self.torch
        moved = 0
        for req in list(self.staging):
            if req._event.query():
                self.staging.remove(req)
                self._submit(req)
                self.active.append(req)
                moved += 1
        if self.active:
            first = min(r._slot for r in self.active)
            n = self.jobs - first
            buf = np.zeros(n, dtype=np.uint64)
            running = C.c_int32(0)
            self.check(self.lib.atb_serve_poll(self.srv, first, n, buf.ctypes.data,
                                               C.byref(running)))
            for req in list(self.active):
                if int(buf[req._slot - first]) != req.n:
                    continue
                moved += 1
                req.done_turns = req.nturns
                self.particle_turns += req.n * req.nturns
                self.live_work -= self._work(req)
                self.live_tiles -= self._tiles(req)
                self.active.remove(req)
                with torch.cuda.stream(self.copy):
                    for k in req._host:
                        req._host[k].copy_(req.dev[k], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(self.copy)
                req._event = ev
                self.retiring.append(req)
        return moved

    def _retire(self, now: float):
        for req in list(self.retiring):
            if not req._event.query():
                continue
            self.retiring.remove(req)
            h = req._host
            req.result = np.asfortranarray(h["r"].numpy().T)
            req.losses = {"islost": h["lost"].numpy().astype(bool),
                          "turn": h["lturn"].numpy().view(np.uint32),
                          "elem": h["lelem"].numpy().view(np.uint32),
                          "coord": np.asfortranarray(h["lcoord"].numpy().T)}
            req.dev, req._host = {}, None
            req.finished = now
            self.used -= req.n * BYTES_PER_PARTICLE
            self.done.append(req)

    def _maybe_reset(self):
        """An idle queue is emptied so its slots can be used again."""
        C = self.C
        if self.jobs > (1 << 15) and not (self.staging or self.active or self.retiring):
            self.check(self.lib.atb_serve_reset(self.srv))
            self.jobs = 0

    def serve(self, requests: list[Request], time_limit: float | None = None):
        """Replay a trace: request k becomes visible at ``arrival`` seconds
        after the start.  Returns the wall time of the whole trace."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        i = 0
        while i < len(pending) or self.waiting or self.staging or self.active or self.retiring:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                self.waiting.append(pending[i])
                i += 1
            self._admit(now)
            moved = self._poll()
            self._retire(time.perf_counter() - t0)
            self._maybe_reset()
            if not moved:
                time.sleep(2e-4)
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
        return time.perf_counter() - t0

    def counters(self) -> dict:
        """Tiles published and claimed from the host queue and continuations
        written to and taken from the device queue since the last reset."""
        out = (self.C.c_int32 * 4)()
        self.check(self.lib.atb_serve_counters(self.srv, out))
        return dict(zip(("published", "claimed", "requeued", "resumed"), list(out)))

    def close(self):
        if self.srv:
            self.check(self.lib.atb_serve_close(self.srv))
            self.srv = None
        for lid in self.lids.values():
            self.eng.free(lid)
        self.lids = {}


class ShardedTrackingServer:
    """One device-resident server per GPU of the process, requests dealt out
    as they arrive to the server with the least work outstanding (admitted
    or waiting, N x T x flops per particle-turn).  The devices share nothing:
    a request runs whole on one GPU, as in the reference a call runs whole
    on one process."""

    def __init__(self, lattices: dict, devices, **kw):
        self.servers = [TrackingServer(lattices, device=d, **kw) for d in devices]

    @staticmethod
    def _outstanding(srv) -> float:
        return sum(srv._work(r) for r in srv.waiting + srv.staging + srv.active)

    def _assign(self, req):
        srv = min(self.servers, key=lambda s: (self._outstanding(s), self.servers.index(s)))
        srv.waiting.append(req)
        return srv

    @property
    def done(self) -> list[Request]:
        return [r for s in self.servers for r in s.done]

    def serve(self, requests: list[Request], time_limit: float | None = None):
        """Replay a trace over all servers; returns the wall time."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        i = 0

        def busy():
            return any(s.waiting or s.staging or s.active or s.retiring for s in self.servers)

        while i < len(pending) or busy():
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i].arrival <= now:
                self._assign(pending[i])
                i += 1
            moved = 0
            for s in self.servers:
                s._admit(now)
                moved += s._poll()
                s._retire(time.perf_counter() - t0)
                s._maybe_reset()
            if not moved:
                time.sleep(2e-4)
            if time_limit is not None and time.perf_counter() - t0 > time_limit:
                break
        return time.perf_counter() - t0

    def close(self):
        for s in self.servers:
            s.close()
        self.servers = []


def serve_sequential(lattices: dict, requests: list[Request], mode="exact", device: int = 0,
                     time_limit: float | None = None):
    """The plain drop-in as a server: one blocking ``gpupass`` call per request,
    in arrival order (a request waits for all earlier ones)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    for req in pending:
        if time_limit is not None and time.perf_counter() - t0 > time_limit:
            break
        now = time.perf_counter() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        r = np.asfortranarray(req.particles.copy())
        req.admitted = time.perf_counter() - t0
        _, ld = gpupass(lattices[req.lattice], r, req.nturns, losses=True, mode=mode,
                        gpu_pool=[device])
        req.result, req.losses = r, ld
        req.finished = time.perf_counter() - t0
    return time.perf_counter() - t0


def latency_stats(reqs: list[Request]) -> dict:
    lat = np.array([r.latency for r in reqs if r.finished is not None])
    if lat.size == 0:
        return {"completed": 0}
    return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "max_s": float(lat.max())}


def make_trace(lattice_names: list[str], nreq: int, rate_hz: float = 200.0, seed: int = 0,
               n_range=(1e3, 2e6), t_range=(100, 10_000), centre_of=None):
    """A Poisson stream: exponential inter-arrival times at ``rate_hz``; each
    request picks a lattice uniformly, N and T log-uniform in their ranges and
    one of three kinds: a dynamic-aperture grid scan (x-y grid x 5 momentum
    offsets), a momentum-aperture scan (small x-y offset, delta spread over
    +/-5 %), or a Gaussian bunch.  ``centre_of(name)`` gives each lattice's
    orbit to centre the particles on."""
    from . import rings

    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for k in range(nreq):
        t += rng.exponential(1.0 / rate_hz)
        name = lattice_names[int(rng.integers(len(lattice_names)))]
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        nt = int(round(np.exp(rng.uniform(np.log(t_range[0]), np.log(t_range[1])))))
        kind = ("da", "ma", "bunch")[int(rng.integers(3))]
        c = np.zeros(6) if centre_of is None else np.asarray(centre_of(name), dtype=np.float64)
        if kind == "da":
            p = rings.da_grid(n, seed=k, deltas=(-0.02, -0.01, 0.0, 0.01, 0.02), centre=c)
        elif kind == "ma":
            p = np.zeros((6, n))
            p[:] = c[:, None]
            p[0] += 1e-5
            p[2] += 1e-5
            p[4] += np.linspace(-0.05, 0.05, n)
            p = np.asfortranarray(p)
        else:
            p = rings.gaussian(n, rings.LARGE_SIGMA, seed=k, centre=c)
        reqs.append(Request(k, name, p, nt, t, kind))
    return reqs
