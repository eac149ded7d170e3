"""Benchmark: particle-turns/s of the FP64 tracking path on B200.

Workload (default): the radiating large ring (``at_b200.rings.large_ring``,
1954 elements, misaligned, 3 GeV electrons) with a 1,000,000-particle
Gaussian bunch around its closed orbit per GPU.  One step tracks the bunch
for ``--turns-per-step`` turns (default 10); the bunch keeps evolving from
step to step with the absolute turn counter advancing, so K steps are K*T
consecutive turns of the 10,000-turn run.

Arms:
  default            this engine.  ``value``: device time (CUDA events on the
                     launching stream, L2 flushed between steps) with the
                     particles resident in HBM; ``e2e``: the drop-in call
                     ``at_b200.gpupass`` on pinned host arrays (host->device
                     and device->host copies of the bunch and loss map inside
                     the timed region).
  --impl reference   the reference's own compiled C engine (pyat/at.c +
                     atintegrators, built by oracle/build_ref.py) through its
                     atpass entry, OpenMP over all host cores, on a bounded
                     sample of the same workload each step.

Multi-GPU (torchrun): one process per GPU, each tracks its own bunch (weak
scaling, particles are independent: no collective on the data path); the
step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "particle-turns/s FP64 vs FP64 peak; served p50/p99 latency vs plain drop-in"
UNIT = "particle-turns/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-step-seconds", type=float, default=10.0,
                    help="reference arm: CPU seconds of tracking per step")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own GPU backend")
    ap.add_argument("--workload", default="large", choices=["large", "fodo"])
    ap.add_argument("--particles", type=int, default=None)
    ap.add_argument("--turns-per-step", type=int, default=None)
    ap.add_argument("--mode", default="exact", choices=["fast", "exact"],
                    help="arithmetic of the headline (exact: the reference's operation order)")
    ap.add_argument("--threads", type=int, default=0, help="threads per block (0: default)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving trace")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-full", action="store_true",
                    help="serving trace at the stated sizes (N up to 2e6, T up to 1e4)")
    ap.add_argument("--serve-time-limit", type=float, default=None,
                    help="end each served trace after this many seconds")
    ap.add_argument("--serve-only", action="store_true",
                    help="only the serving comparison (one JSON object)")
    ap.add_argument("--serve-chunk-flops", type=float, default=None,
                    help="device-resident server: algorithmic flops per tile chunk")
    ap.add_argument("--serve-forms", default="device,rounds,sequential",
                    help="comma-separated serving forms to run")
    ap.add_argument("--serve-opts", default="{}",
                    help="device-resident server: keyword arguments as JSON")
    ap.add_argument("--no-diff", action="store_true", help="skip the tangent-kernel timing")
    ap.add_argument("--diff-only", action="store_true",
                    help="only the tangent-kernel timing (one JSON object)")
    ap.add_argument("--diff-particles", type=int, default=65536)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-variant run")
    ap.add_argument("--no-acceptance", action="store_true", help="skip the acceptance scan")
    ap.add_argument("--batch-turn-scale", type=float, default=0.01,
                    help="scale of the batched variants' turn counts (1.0: 500-5000 turns)")
    ap.add_argument("--batch-sample", type=int, default=None,
                    help="time the per-variant drop-in on this many seeded variants")
    ap.add_argument("--batch-only", action="store_true",
                    help="only the batched-variant comparison (one JSON object)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fodo-line", action="store_true",
                    help="skip the FODO (10,000 particles x 1000 turns) line")
    ap.add_argument("--no-alt-line", action="store_true",
                    help="skip timing the other arithmetic mode beside the headline's")
    ap.add_argument("--refpts-line", action="store_true",
                    help="also time snapshots at every element (FODO, 10,000 particles)")
    return ap.parse_args()


def _defaults(a):
    if a.particles is None:
        a.particles = 1_000_000 if a.workload == "large" else 10_000
    if a.turns_per_step is None:
        a.turns_per_step = 10 if a.workload == "large" else 100
    return a


def _ring(workload):
    from at_b200 import rings
    if workload == "large":
        return rings.large_ring()
    return rings.fodo_ring()


def _bunch(workload, n, seed):
    from at_b200 import rings
    if workload == "large":
        return rings.large_ring_bunch(n, seed=seed)
    return rings.gaussian(n, seed=seed)


def _config(a, ring):
    return {"workload": "%s ring, %d particles/GPU, %d turns/step" % (
                "radiating large (1954 elements)" if a.workload == "large" else "FODO (385 elements)",
                a.particles, a.turns_per_step),
            "elements": len(ring), "particles_per_gpu": a.particles,
            "turns_per_step": a.turns_per_step, "arithmetic": a.mode,
            "losses": True, "l2": "flushed between timed steps",
            "parallelism": "particle shards, one per GPU"}


# --------------------------------------------------------------------------- #
# reference (CPU) runs                                                         #
# --------------------------------------------------------------------------- #
def _ref_sample(workload, particles, turns, threads):
    """Time the reference engine once in a subprocess; returns the JSON dict."""
    from oracle import ref_runner
    if not ref_runner.available():
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    cmd = [sys.executable, os.path.join(REPO, "oracle", "ref_runner.py"), workload,
           "--particles", str(particles), "--turns", str(turns), "--threads", str(threads)]
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=900)
    if out.returncode != 0:
        raise RuntimeError("reference run failed: %s" % out.stderr[-2000:])
    return json.loads(out.stdout.strip().splitlines()[-1])


def _port_sample(workload, particles, turns, threads):
    """The oracle restatement (when the reference build is absent)."""
    from oracle import oracle
    ring = _ring(workload)
    r = _bunch(workload, particles, 0)
    t0 = time.perf_counter()
    oracle.track(ring, r, turns, energy=ring.energy, rest_energy=ring.particle.rest_energy,
                 losses=True, nthreads=threads)
    dt = time.perf_counter() - t0
    return {"particle_turns": particles * turns, "seconds": dt, "rate": particles * turns / dt,
            "threads": threads, "sample": "%d particles x %d turns" % (particles, turns)}


def cpu_rate(workload, target_s=15.0, threads=None):
    """A bounded sample (about target_s of CPU work) of the workload."""
    threads = threads or os.cpu_count() or 1
    kind = "reference"
    fn = _ref_sample
    from oracle import ref_runner
    if not ref_runner.available():
        kind, fn = "port", _port_sample
    probe = fn(workload, max(64, 8 * threads), 1, threads)
    n = int(max(64, min(200_000, probe["rate"] * target_s)))
    res = fn(workload, n, 1, threads)
    res["kind"] = kind
    return res


def _atgpu_sample(workload, particles, turns, flat_r=False):
    """The reference's own GPU backend (atgpu, built by oracle/build_ref.py
    --atgpu) on the same workload, in a process of its own; None where it is
    not built or no GPU answers."""
    from oracle import ref_gpu_runner
    if not ref_gpu_runner.available():
        return None
    cmd = [sys.executable, os.path.join(REPO, "oracle", "ref_gpu_runner.py"), workload,
           "--particles", str(particles), "--turns", str(turns), "--steps", "2",
           "--check", "1024"] + (["--flat-r"] if flat_r else [])
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"unavailable": "timed out"}
    if out.returncode != 0:
        return {"unavailable": out.stderr.strip().splitlines()[-1][:200] if out.stderr else
                "exit %d" % out.returncode}
    return json.loads(out.stdout.strip().splitlines()[-1])


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ring_len = len(_ring(a.workload))
    threads = os.cpu_count() or 1
    kind = "reference"
    from oracle import ref_runner
    fn = _ref_sample
    if not ref_runner.available():
        kind, fn = "port", _port_sample
    probe = fn(a.workload, max(64, 8 * threads), 1, threads)
    # each step: about 10 s of CPU work by default, so K+W steps stay within minutes
    n = int(max(64, min(200_000, probe["rate"] * a.ref_step_seconds)))
    for _ in range(a.warmup):
        fn(a.workload, max(64, n // 10), 1, threads)
    rates, secs = [], []
    for _ in range(a.steps):
        res = fn(a.workload, n, 1, threads)
        rates.append(res["rate"])
        secs.append(res["seconds"])
    value = a.steps * n / sum(secs)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sum(secs) / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": dict(_config(a, range(ring_len)), sample="%d particles x 1 turn per step" % n),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": "%d particles x 1 turn per step, %d steps" % (n, a.steps)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # the reference's own GPU backend on the same workload, for comparison (its
    # stock path, and with R1/R2 in the one-dimensional form it reads)
    gpu_ref = {}
    for tag, flat in (("stock", False), ("r1_r2_as_1d", True)):
        if a.no_reference_gpu or (flat and a.workload != "large"):
            continue
        gpu_ref[tag] = _atgpu_sample(a.workload, a.particles, a.turns_per_step, flat)
    line["reference_gpu_backend"] = gpu_ref or None
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- #
# GPU arm                                                                      #
# --------------------------------------------------------------------------- #
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.th.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def run_b200(a):
    import torch
    import torch.distributed as dist

    from at_b200 import _lib, flops
    from at_b200.engine import Engine
    from at_b200.lattice import compile_lattice
    from at_b200 import tracking

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    ring = _ring(a.workload)
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    fpt, ntrans = flops.flops_per_particle_turn(cl)
    eng = Engine.get(local)
    if a.threads:
        eng.set_launch(threads=a.threads)
    lid = eng.upload(cl)
    mode = a.mode
    N, T = a.particles, a.turns_per_step

    # FP64 peak of this GPU, measured live
    import ctypes as C
    pk, pks = C.c_double(), C.c_double()
    _lib.check(_lib.lib().atb_fp64_peak(local, C.byref(pk), C.byref(pks)))
    fp64_peak = pk.value

    # particles resident in HBM: (6, N) Fortran order == torch (N, 6) row-major
    r0 = _bunch(a.workload, N, seed=rank)
    rd = torch.from_numpy(np.ascontiguousarray(r0.T)).to(dev)
    lost = torch.zeros(N, dtype=torch.uint8, device=dev)
    lturn = torch.zeros(N, dtype=torch.int32, device=dev)
    lelem = torch.zeros(N, dtype=torch.int32, device=dev)
    lcoord = torch.zeros((N, 6), dtype=torch.float64, device=dev)
    alive = torch.zeros(T, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # a dedicated stream: the engine launches on it and the events are
    # recorded on it (the legacy default stream's handle would read as NULL)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr != 0
    lp = (lost.data_ptr(), lturn.data_ptr(), lelem.data_ptr(), lcoord.data_ptr())

    def step(turn0, with_alive, arith=None):
        if with_alive:
            alive.zero_()
        eng.track_device(lid, rd.data_ptr(), N, T, turn0, losses=lp,
                         alive_ptr=alive.data_ptr() if with_alive else None,
                         mode=arith or mode, stream=sptr)

    turn = 0
    for _ in range(a.warmup):
        step(turn, False)
        turn += T
    torch.cuda.synchronize()
    eng.sync(sptr)

    clocks = Clocks(local) if rank == 0 else None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    times = []
    survivors = 0
    for _ in range(a.steps):
        flush.fill_(1.0)                      # evict the particle state from L2
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(turn, True)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
        survivors += int(alive.sum().item())
        turn += T
    torch.cuda.synchronize()
    eng.sync(sptr)
    if world > 1:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    tot = torch.tensor([sum(times)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    t_max = float(tot.item())
    value = world * N * T * a.steps / t_max
    # roofline of the tracking kernel: algorithmic flops of the particle-turns
    # actually tracked (survivors per turn) over its event-timed duration
    achieved = fpt * survivors / sum(times) / 1e12

    # the other arithmetic on the same resident bunch: with the exact
    # headline, the fast kernel (FMA contraction, reciprocal reuse; within
    # 2e-13 of each coordinate's scale after one turn of this ring, outside
    # the 1e-13 bound), and the other way round
    alt_line = None
    alt = "fast" if mode == "exact" else "exact"
    if world == 1 and not a.no_alt_line:
        xt = []
        step(turn, False, alt)                  # warm-up
        turn += T
        for _ in range(2):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(turn, False, alt)
            e1.record(stream)
            e1.synchronize()
            xt.append(e0.elapsed_time(e1) * 1e-3)
            turn += T
        eng.sync(sptr)
        # the same end to end through gpupass on pinned host arrays
        hb2 = torch.empty((N, 6), dtype=torch.float64).pin_memory()
        hb2.copy_(torch.from_numpy(np.ascontiguousarray(r0.T)))
        rh2 = hb2.numpy().T
        line2 = type(ring)(list(ring), energy=ring.energy, particle=ring.particle)
        tracking.gpupass(line2, rh2, 1, losses=True, mode=alt, gpu_pool=[local])
        et2 = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tracking.gpupass(line2, rh2, T, losses=True, reuse=True, keep_counter=True,
                             mode=alt, gpu_pool=[local])
            et2.append(time.perf_counter() - t0)
        alt_line = {"arithmetic": alt, "value": N * T * len(xt) / sum(xt), "unit": UNIT,
                    "e2e": {"value": N * T * len(et2) / sum(et2), "unit": UNIT,
                            "api": "at_b200.gpupass, pinned host arrays"},
                    "ms_per_step": 1e3 * sum(xt) / len(xt), "steps": len(xt),
                    "one_turn_deviation_from_oracle":
                        "exact: <= 1e-13 of each coordinate's scale on every ring (bit-identical "
                        "to the reference's C build away from sin/tan); fast: <= 1e-13 on the "
                        "FODO ring, <= 2e-13 on this ring (tests/test_gpu_parity.py)"}

    # end to end through the drop-in entry point on pinned host buffers
    e2e = None
    if not a.no_e2e:
        hb = torch.empty((N, 6), dtype=torch.float64).pin_memory()
        hb.copy_(torch.from_numpy(np.ascontiguousarray(r0.T)))
        rh = hb.numpy().T                      # (6, N) Fortran view, pinned
        assert rh.flags.f_contiguous
        line = list(ring)
        line_obj = type(ring)(line, energy=ring.energy, particle=ring.particle)
        tracking.gpupass(line_obj, rh, 1, losses=True, mode=mode, gpu_pool=[local])
        etimes = []
        if world > 1:
            dist.barrier()
        for k in range(a.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tracking.gpupass(line_obj, rh, T, losses=True, reuse=True, keep_counter=True,
                             mode=mode, gpu_pool=[local])
            etimes.append(time.perf_counter() - t0)
        et = torch.tensor([sum(etimes)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
        e2e = {"value": world * N * T * a.steps / float(et.item()), "unit": UNIT,
               "h2d_bytes_per_step": N * 48,
               "d2h_bytes_per_step": N * 48 + N * (1 + 4 + 4 + 48),
               "api": "at_b200.gpupass (reference gpupass/atpass signature), pinned host arrays"}

    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        try:
            c = cpu_rate(a.workload)
            cpu = {"value": c["rate"], "unit": UNIT, "cores": c["threads"], "kind": c["kind"],
                   "sample": c["sample"] + " of the same workload, OpenMP over all host cores"}
        except Exception as exc:  # noqa: BLE001
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": "failed: %s" % str(exc)[:200]}

    config0 = None
    if world == 1 and a.workload == "large" and not a.no_fodo_line:
        config0 = run_fodo_line(local, rank == 0 and not a.no_cpu_baseline)

    serve = None
    if world == 1 and not a.no_serve:
        serve = run_serving(a.serve_requests, mode, local, full=a.serve_full,
                            time_limit=a.serve_time_limit, chunk_flops=a.serve_chunk_flops,
                            forms_wanted=tuple(a.serve_forms.split(",")),
                            opts=json.loads(a.serve_opts))
    dif = None
    if world == 1 and not a.no_diff:
        dif = run_diff(local, a.diff_particles)
    bat = None
    if world == 1 and not a.no_batch:
        bat = run_batching(local, mode, a.batch_turn_scale, a.batch_sample)
    acc = None
    if world == 1 and not a.no_acceptance:
        acc = run_acceptance(mode, cpu)
    refl = None
    if world == 1 and a.refpts_line:
        refl = run_refpts_line(local, mode)

    traffic = None
    prof = os.path.join(REPO, "profiles", "traffic_%s.json" % a.workload)
    if os.path.exists(prof):
        with open(prof) as f:
            tp = json.load(f)
        traffic = tp.get("bytes_per_particle_launch", 0.0) * N
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * t_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded lattice and Gaussian bunch)",
            "config": _config(a, ring),
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic,
                         "peak_source": "measured live: atb_fp64_peak DFMA chains on this GPU",
                         "flops_per_particle_turn": fpt, "survivor_particle_turns": survivors,
                         # the exact arithmetic issues the reference's +,-,*,/ one by one
                         # (no FMA fusion), so its FP64-pipe ceiling in these flops is
                         # half the DFMA peak
                         "unfused_ceiling": fp64_peak / 2 if mode == "exact" else None,
                         "frac_of_unfused_ceiling":
                             achieved / (fp64_peak / 2) if mode == "exact" else None},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": a.steps, "clocks": clk,
            "config0_fodo": config0,
            "serving": serve, "differentiation": dif, "batching": bat, "acceptance": acc,
            "%s_arithmetic" % alt: alt_line,
        }
        if refl is not None:
            line["refpts_every_element"] = refl
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _fodo_rates(device, mode, ring, r0, n, nt):
    import torch

    from at_b200 import tracking
    from at_b200.engine import Engine
    from at_b200.lattice import compile_lattice

    dev = torch.device("cuda", device)
    eng = Engine.get(device)
    cl = compile_lattice(ring, ring.energy, ring.particle.rest_energy)
    lid = eng.upload(cl)
    st = torch.cuda.Stream(dev)
    times = []
    try:
        for k in range(3):
            rd = torch.from_numpy(np.ascontiguousarray(r0.T)).to(dev)
            lp = tuple(torch.zeros(s, dtype=d, device=dev).data_ptr() for s, d in
                       ((n, torch.uint8), (n, torch.int32), (n, torch.int32),
                        ((n, 6), torch.float64)))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            eng.track_device(lid, rd.data_ptr(), n, nt, 0, losses=lp, mode=mode,
                             stream=st.cuda_stream)
            e1.record(st)
            e1.synchronize()
            eng.sync(st.cuda_stream)
            if k:
                times.append(e0.elapsed_time(e1) * 1e-3)
    finally:
        eng.free(lid)
    hb = torch.empty((n, 6), dtype=torch.float64).pin_memory()
    e2e = []
    for _ in range(3):
        hb.copy_(torch.from_numpy(np.ascontiguousarray(r0.T)))
        rh = hb.numpy().T
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, ld = tracking.gpupass(ring, rh, nt, losses=True, mode=mode, gpu_pool=[device])
        e2e.append(time.perf_counter() - t0)
    return {"value": n * nt / min(times), "unit": UNIT, "device_s": min(times),
            "e2e": {"value": n * nt / min(e2e[1:]), "unit": UNIT, "wall_s": min(e2e[1:]),
                    "h2d_bytes": n * 48, "d2h_bytes": n * (48 + 57)},
            "lost": int(ld["islost"].sum()), "arithmetic": mode}


def run_fodo_line(device, with_cpu):
    """The FODO workload at its stated size: 10,000 particles (Gaussian,
    seed 0) for 1000 turns with the loss map, device-resident (CUDA events on
    the launching stream) and end to end through ``gpupass`` on pinned host
    arrays; beside it the reference's own CPU engine on a sample of the same
    ring.  On this ring the fast arithmetic meets the path's tolerances (1e-13
    of scale after one turn, the 1000-turn loss-map rule:
    tests/test_gpu_parity.py), so it gives the line's value, with the exact
    arithmetic as ``other_arithmetic``.  10,000 particles fill only part of
    the GPU (one particle's chain of instructions per turn bounds the time),
    so this line is latency-bound, not the roofline case."""
    mode = "fast"
    from at_b200 import rings

    ring = rings.fodo_ring()
    n, nt = 10_000, 1000
    r0 = rings.gaussian(n, seed=0)
    out = {"workload": "FODO ring (385 elements), 10000 particles, 1000 turns, losses on"}
    out.update(_fodo_rates(device, mode, ring, r0, n, nt))
    out["other_arithmetic"] = _fodo_rates(device, "fast" if mode == "exact" else "exact",
                                          ring, r0, n, nt)
    if with_cpu:
        c = cpu_rate("fodo")
        out["cpu_baseline"] = {"value": c["rate"], "unit": UNIT, "cores": c["threads"],
                               "kind": c["kind"], "sample": c["sample"]}
    return out


def run_refpts_line(device, mode, n=10_000, nt=20, reps=3):
    """Snapshots at every element: the FODO ring, ``n`` particles (Gaussian,
    seed 0), ``nt`` turns, refpts at each of the 385 elements and at the
    turn's end, end to end through ``gpupass`` on host arrays (the result
    array allocated by the call, as the reference's is), beside the same call
    without refpts.  The difference is the cost of writing the snapshots and
    returning them to the host, reported against the snapshot bytes."""
    from at_b200 import rings, tracking

    ring = rings.fodo_ring()
    refs = np.arange(len(ring) + 1, dtype=np.uint32)
    r0 = rings.gaussian(n, seed=0)
    out = {"workload": "FODO ring (385 elements), %d particles, %d turns, refpts at all %d "
                       "points, losses on" % (n, nt, refs.size),
           "arithmetic": mode, "rout_bytes": 48 * n * refs.size * nt}
    for name, rp in (("without_refpts", None), ("with_refpts", refs)):
        r = r0.copy(order="F")
        tracking.gpupass(ring, r, 1, rp, losses=True, mode=mode, gpu_pool=[device])
        times = []
        for _ in range(reps):
            r = r0.copy(order="F")
            t0 = time.perf_counter()
            res = tracking.gpupass(ring, r, nt, rp, losses=True, mode=mode, gpu_pool=[device])
            times.append(time.perf_counter() - t0)
            del res
        out[name] = {"wall_s": min(times), "particle_turns_per_s": n * nt / min(times)}
    extra = out["with_refpts"]["wall_s"] - out["without_refpts"]["wall_s"]
    out["snapshot_gb_per_s"] = out["rout_bytes"] / max(extra, 1e-9) / 1e9
    return out


def run_serving(nreq, mode, device, full=False, time_limit=None, chunk_flops=None,
                forms_wanted=("device", "rounds", "sequential"), opts=None):
    """A finite Poisson trace (200 requests/s) over the 16-lattice pool,
    served three ways on the same trace: the device-resident server (one
    persistent kernel fed by a queue the host appends to), the round server
    (one batched launch per round), and one blocking drop-in call per request
    in arrival order.  ``full``: the stated size ranges (N log-uniform in
    [1e3, 2e6] particles, T in [100, 1e4] turns), else a scaled-down trace (N up
    to 1e5, T up to 1000) that finishes in seconds.  The offered load exceeds
    the GPU's capacity either way, so latencies are queue-dominated; a
    ``time_limit`` ends the trace early and reports the completed requests."""
    from at_b200 import rings, serving

    lats, orbits = rings.serving_pool()
    n_range, t_range = ((1e3, 2e6), (100, 10_000)) if full else ((1e3, 1e5), (100, 1000))
    kw = dict(rate_hz=200.0, seed=7, n_range=n_range, t_range=t_range, centre_of=orbits.get)
    out = {"requests": nreq, "rate_hz": 200.0, "lattices": len(lats),
           "sizes": "N log-uniform [%g, %g], T log-uniform [%g, %g]" % (*n_range, *t_range),
           "arithmetic": mode}
    forms = [f for f in (("continuous_batching_device_resident", serving.TrackingServer, "device"),
                         ("continuous_batching_rounds", serving.RoundServer, "rounds"))
             if f[2] in forms_wanted]
    traces = {}
    for name, cls, _ in forms:
        trace = serving.make_trace(list(lats), nreq, **kw)
        extra_kw = {}
        if cls is serving.TrackingServer and chunk_flops:
            extra_kw["chunk_flops"] = float(chunk_flops)
            out["chunk_flops"] = float(chunk_flops)
        if cls is serving.TrackingServer and opts:
            extra_kw.update(opts)
            out["server_options"] = dict(opts)
        srv = cls(lats, hbm_budget_bytes=150e9, device=device, mode=mode, **extra_kw)
        extra = {}
        try:
            wall = srv.serve(trace, time_limit=time_limit)
            if hasattr(srv, "counters"):
                extra["tile_counters"] = srv.counters()
        finally:
            srv.close()
        st = serving.latency_stats(trace)
        pt = sum(r.n * r.nturns for r in trace if r.finished is not None)
        out[name] = dict(st, particle_turns_per_s=pt / wall, wall_s=wall, **extra)
        traces[name] = trace
    if "sequential" in forms_wanted:
        seq_trace = serving.make_trace(list(lats), nreq, **kw)
        wall_seq = serving.serve_sequential(lats, seq_trace, mode=mode, device=device,
                                            time_limit=time_limit)
        sq = serving.latency_stats(seq_trace)
        pt = sum(r.n * r.nturns for r in seq_trace if r.finished is not None)
        out["plain_drop_in_sequential"] = dict(sq, particle_turns_per_s=pt / wall_seq,
                                               wall_s=wall_seq)
        same = True
        for name, _, _ in forms:
            for a, b in zip(traces[name], seq_trace):
                if a.finished is not None and b.finished is not None:
                    same = same and bool(np.array_equal(a.result, b.result, equal_nan=True))
        out["results_identical"] = same
    return out


def _survivor_turns(ld, nturns):
    lost = ld["islost"]
    return float(np.where(lost, ld["turn"].astype(np.float64) + 1.0, float(nturns)).sum())


def run_batching(device, mode, turn_scale, sample=None):
    """The batched-variant workload: 256 error-seeded copies of the large
    ring (seeds 2-257), each with N_i in [1024, 16384] particles on an x-y
    dynamic-aperture grid at delta in {-3 %, 0, +3 %} and T_i in [500, 5000]
    turns scaled by ``turn_scale``, as ONE graph-captured persistent launch
    (launch shape from the autotuner), against the plain drop-in called once
    per variant on the same jobs (all of them, or a seeded sample of
    ``sample`` variants timed and reported as a rate)."""
    from at_b200 import rings, tracking
    from at_b200.batch import BatchTracker

    work = rings.batch_workload(256, first_seed=2, turn_scale=turn_scale, seed=0)
    lats = [rings.large_ring_variant(s) for s, _, _ in work]
    parts = [rings.da_grid(n, seed=s) for s, n, _ in work]
    turns = [t for _, _, t in work]
    t0 = time.perf_counter()
    bt = BatchTracker(lats, parts, turns, mode=mode, tune=True, graph=True, device=device)
    setup = time.perf_counter() - t0
    try:
        bt.run()
        bt.reset()
        dt = bt.run()
        w0 = time.perf_counter()
        bt.reset()
        bt.run()
        wall_batch = time.perf_counter() - w0
        res = bt.results()
        tuning = bt.tuning
    finally:
        bt.close()
    pt = sum(n * t for (_, n, t) in work)
    surv = sum(_survivor_turns(ld, t) for (_, ld), t in zip(res, turns))
    ks = list(range(len(work)))
    if sample is not None and sample < len(work):
        ks = sorted(np.random.default_rng(1).choice(len(work), sample, replace=False).tolist())
    t0 = time.perf_counter()
    same = True
    for k in ks:
        r = parts[k].copy(order="F")
        tracking.gpupass(lats[k], r, turns[k], losses=True, mode=mode, gpu_pool=[device])
        same = same and bool(np.array_equal(r, res[k][0], equal_nan=True))
    seq = time.perf_counter() - t0
    pt_seq = sum(work[k][1] * work[k][2] for k in ks)
    return {"variants": len(work), "particles": int(sum(n for _, n, _ in work)),
            "turns": "U{500..5000} x %g" % turn_scale, "particle_turns": pt,
            "survivor_particle_turns": surv,
            "one_launch": {"device_s": dt, "wall_s_incl_reset": wall_batch,
                           "particle_turns_per_s": pt / dt,
                           "survivor_particle_turns_per_s": surv / dt},
            "plain_drop_in_per_variant": {"variants_timed": len(ks), "wall_s": seq,
                                          "particle_turns_per_s": pt_seq / seq,
                                          "wall_s_all_variants_at_this_rate": pt / (pt_seq / seq)},
            "setup_s_compile_upload_tune_capture": setup,
            "autotune": tuning, "results_identical": same}


def run_acceptance(mode, cpu):
    """A dynamic-aperture scan as users run it (the reference's
    get_acceptance, radial grid of 41 x 21 points, 1024 turns, on the large
    ring): wall time through ``at_b200.acceptance`` (orbit search, grid,
    tracking with the loss map, boundary), against the time the reference's
    engine needs for the same particle-turns at the CPU rate measured in
    this run (tracking only)."""
    from at_b200 import acceptance, rings

    ring = rings.large_ring(seed=1)
    kw = dict(planes=["x", "y"], npoints=[41, 21], amplitudes=[6e-3, 3e-3], nturns=1024,
              grid_mode=acceptance.GridMode.RADIAL, mode=mode)
    acceptance.get_acceptance(ring, **dict(kw, nturns=2))
    t0 = time.perf_counter()
    b, s, g = acceptance.get_acceptance(ring, **kw)
    wall = time.perf_counter() - t0
    pt = g.shape[1] * (kw["nturns"] + 1)
    out = {"grid": "radial 41 x 21 (x up to 6 mm, y up to 3 mm), 1024 turns, large ring",
           "particles": int(g.shape[1]), "survivors": int(s.shape[1]), "wall_s": wall,
           "particle_turns_per_s": pt / wall}
    if cpu and cpu.get("value"):
        out["reference_engine_tracking_s_at_measured_cpu_rate"] = pt / cpu["value"]
    return out


def run_diff(device, n=65536):
    """Exact derivatives on the FODO ring (the differentiable-tracking
    workload): 65,536 particles, sigma 1e-6 around the closed orbit, with
    respect to the initial coordinates and the 64 quadrupole + 64 sextupole
    strengths, for 1 and 100 turns.  Device time of the tangent launch (CUDA
    events), of the autograd backward contraction, of the adjoint kernels'
    forward pass and backward sweep for the same vector-Jacobian product
    (with their agreement with the tangent's), and of the 2 x 128 + 12
    exact-mode tracking runs that central differences would need instead."""
    import torch

    from at_b200 import diff, physics, rings
    from at_b200.engine import Engine

    ring = rings.fodo_ring()
    orbit = physics.find_orbit6(ring, mode="exact")
    r0 = rings.gaussian(n, [1e-6] * 6, seed=11, centre=orbit)
    params = diff.multipole_strengths(ring)
    tr = diff.TangentTracker(ring, params, device=device)
    adj = diff.AdjointTracker(ring, params, device=device)
    dev = torch.device("cuda", device)
    x = torch.tensor(np.ascontiguousarray(r0.T), dtype=torch.float64, device=dev)
    out = {"workload": "FODO ring (385 elements), %d particles sigma 1e-6 around the closed "
                       "orbit, %d strengths (64 quadrupole + 64 sextupole)" % (n, len(params))}
    eng = Engine.get(device)
    lid = eng.upload(tr.cl)
    # the exact tracking runs on a stream of its own with its events (the
    # legacy default stream's handle would read as NULL: the engine's stream)
    trk = torch.cuda.Stream(dev)
    try:
        for nt in (1, 100):
            tr.track(x, None, nt)                     # warm-up
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r, jac, grad, lost = tr.track(x, None, nt)
            e1.record()
            e1.synchronize()
            t_tan = e0.elapsed_time(e1) * 1e-3
            # the adjoint (vector-Jacobian) products of the autograd backward
            g = torch.randn_like(r)
            e0.record()
            vjp_x = torch.einsum("ni,nij->nj", g, jac)
            vjp_k = torch.einsum("ni,pin->p", g, grad)
            e1.record()
            e1.synchronize()
            t_bwd = e0.elapsed_time(e1) * 1e-3
            # the same products from the adjoint kernels
            _, _, st = adj.forward(x, None, nt)       # warm-up
            adj.backward(st, g)
            e0.record()
            _, _, st = adj.forward(x, None, nt)
            e1.record()
            e1.synchronize()
            t_afwd = e0.elapsed_time(e1) * 1e-3
            e0.record()
            ax, ak = adj.backward(st, g)
            e1.record()
            e1.synchronize()
            t_abwd = e0.elapsed_time(e1) * 1e-3
            del st

            def rel(a, b):
                return float(((a - b).abs().max() / b.abs().max()).item())
            # one exact-mode tracking of the same particles (device resident)
            xr = x.clone()
            trk.wait_stream(torch.cuda.current_stream(dev))
            eng.track_device(lid, xr.data_ptr(), n, nt, mode="exact", stream=trk.cuda_stream)
            xr = x.clone()
            trk.wait_stream(torch.cuda.current_stream(dev))
            e0.record(trk)
            eng.track_device(lid, xr.data_ptr(), n, nt, mode="exact", stream=trk.cuda_stream)
            e1.record(trk)
            e1.synchronize()
            eng.sync(trk.cuda_stream)
            t_trk = e0.elapsed_time(e1) * 1e-3
            runs = 2 * len(params) + 12
            out["turns_%d" % nt] = {
                "tangent_ms": 1e3 * t_tan, "backward_ms": 1e3 * t_bwd,
                "particle_turns_per_s": n * nt / t_tan,
                "lost": int(lost.sum().item()),
                "exact_tracking_ms": 1e3 * t_trk,
                "central_differences_ms": 1e3 * t_trk * runs,
                "speedup_vs_central_differences": t_trk * runs / t_tan,
                "adjoint": {"forward_ms": 1e3 * t_afwd, "backward_ms": 1e3 * t_abwd,
                            "particle_turns_per_s": n * nt / (t_afwd + t_abwd),
                            "speedup_vs_tangent_vjp": (t_tan + t_bwd) / (t_afwd + t_abwd),
                            "rel_diff_vs_tangent": {"d_r0": rel(ax, vjp_x),
                                                    "d_strengths": rel(ak, vjp_k)}}}
        # the adjoint with every element's entry state stored by the forward
        # pass (N x 385 elements x turns x 48 B: 12 GB for 10 turns), so the
        # backward sweep tracks nothing again
        nt = 10
        g = torch.randn((n, 6), dtype=torch.float64, device=dev)
        ts = {}
        for store in (False, True):
            _, _, st = adj.forward(x, None, nt, store_elements=store)      # warm-up
            adj.backward(st, g)
            del st
            e0.record()
            _, _, st = adj.forward(x, None, nt, store_elements=store)
            e1.record()
            e1.synchronize()
            tf = e0.elapsed_time(e1) * 1e-3
            e0.record()
            adj.backward(st, g)
            e1.record()
            e1.synchronize()
            ts[store] = (tf, e0.elapsed_time(e1) * 1e-3)
            del st
        out["adjoint_10_turns"] = {
            mode: {"forward_ms": 1e3 * ts[s][0], "backward_ms": 1e3 * ts[s][1],
                   "particle_turns_per_s": n * nt / sum(ts[s])}
            for mode, s in (("tracked_again", False), ("element_states_stored", True))}
    finally:
        eng.free(lid)
        tr.close()
        adj.close()
    return out


def main():
    a = _defaults(_args())
    if a.impl == "reference":
        return run_reference(a)
    if a.diff_only:
        print(json.dumps({"differentiation": run_diff(0, a.diff_particles)}), flush=True)
        return 0
    if a.batch_only:
        print(json.dumps({"batching": run_batching(0, a.mode, a.batch_turn_scale,
                                                   a.batch_sample)}), flush=True)
        return 0
    if a.serve_only:
        print(json.dumps({"serving": run_serving(
            a.serve_requests, a.mode, 0, full=a.serve_full, time_limit=a.serve_time_limit,
            chunk_flops=a.serve_chunk_flops,
            forms_wanted=tuple(a.serve_forms.split(",")),
            opts=json.loads(a.serve_opts))}), flush=True)
        return 0
    return run_b200(a)


if __name__ == "__main__":
    sys.exit(main())
