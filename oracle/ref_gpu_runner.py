"""Run the reference's own GPU backend (atgpu) -- baseline infrastructure only.

``oracle/_ref/pyat_full`` is the reference's pyat built from its sources by
``oracle/build_ref.py --full --atgpu``, including its CUDA backend
``at.tracking.gpu`` (atgpu: the lattice becomes an element array in device
memory and a generated tracking kernel, compiled with NVRTC for the device at
the first call; one launch per turn, atgpu/CudaGPU.cpp:157-185).  This script
calls that backend's ``gpupass`` through its own Python entry, exactly as
pyat's ``_lattice_pass`` does with ``use_mp=MPMode.GPU``
(pyat/at/tracking/track.py:115-127), on pyat ``Element`` objects of the
benchmark lattices, and prints one JSON line.  It runs in a process of its
own so the reference's CUDA context and its ``at`` package stay apart from
the engine's.

    python oracle/ref_gpu_runner.py large --particles 1000000 --turns 10 --steps 3

The timing is wall clock around each ``gpupass`` call (host arrays in and
out, as the reference's API takes them), after a warm-up call that compiles
the kernel and uploads the lattice.  With ``--check`` it also tracks a sample
for one turn on the backend and on the reference's C engine and reports the
largest difference relative to each coordinate's scale.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
import warnings

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PYAT = os.path.join(HERE, "_ref", "pyat_full")


def available() -> bool:
    import sysconfig
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.exists(os.path.join(PYAT, "at", "tracking", "gpu" + ext))


def pyat_lattice(at, ring, flat_r=False):
    """The ring as pyat objects.  atgpu reads the beam energy from each
    cavity and radiating magnet (atgpu/CavityPass.cpp:20,
    StrMPoleSymplectic4RadPass.cpp:21), so those carry ``Energy``.

    pyat holds the misalignment rotations R1/R2 as (6, 6) matrices, and the
    reference's CPU engine reads them so.  atgpu reads them through
    get1DArray, which accepts 1-D arrays only (atgpu/AbstractInterface.cpp:
    51-64, IdentityPass.cpp:23-24), and getOptional1DArray discards the
    error: a (6, 6) R1/R2 is silently ignored.  With ``flat_r`` the same
    matrices are given as (36,) arrays of the same column-major memory,
    which atgpu then applies (transform66, IdentityPass.cpp:178-190)."""
    import numpy as np
    line = []
    for e in ring:
        d = dict(vars(e))
        name = d.pop("FamName", "E")
        if d.get("PassMethod") == "RFCavityPass":
            line.append(at.RFCavity(name, d["Length"], d["Voltage"], d["Frequency"],
                                    d["HarmNumber"], ring.energy, TimeLag=d.get("TimeLag", 0.0)))
            continue
        kw = {}
        for k, v in d.items():
            kw[k] = np.asfortranarray(np.asarray(v, dtype=np.float64)) if isinstance(
                v, (np.ndarray, list)) else v
        el = at.Element(name, **kw)
        for k in ("MaxOrder", "NumIntSteps", "FringeBendEntrance", "FringeBendExit",
                  "FringeQuadEntrance", "FringeQuadExit"):
            if hasattr(el, k):
                setattr(el, k, int(getattr(el, k)))
        if str(d.get("PassMethod", "")).endswith("RadPass"):
            el.Energy = float(ring.energy)
        if flat_r:
            for k in ("R1", "R2"):
                if hasattr(el, k):
                    m = np.asfortranarray(np.asarray(getattr(el, k), dtype=np.float64))
                    object.__setattr__(el, k, np.asfortranarray(m.reshape(-1, order="F")))
        line.append(el)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return at.Lattice(line, energy=ring.energy, particle=at.Particle("electron"),
                          periodicity=1)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["large", "fodo"])
    ap.add_argument("--particles", type=int, default=100_000)
    ap.add_argument("--turns", type=int, default=10)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--check", type=int, default=0, help="one-turn check sample size")
    ap.add_argument("--flat-r", action="store_true",
                    help="give R1/R2 as (36,) arrays, the form atgpu reads")
    a = ap.parse_args(argv)

    sys.path.insert(0, PYAT)
    sys.path.insert(1, REPO)
    import numpy as np
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        import at
        from at.tracking import gpu as atgpu            # the reference's CUDA backend
        from at.tracking.atpass import atpass as cpu_atpass
    from at_b200 import rings

    ring = rings.large_ring() if a.workload == "large" else rings.fodo_ring()
    lat = pyat_lattice(at, ring, flat_r=a.flat_r)
    line = list(lat)
    cpu_line = list(pyat_lattice(at, ring)) if a.flat_r else line
    kw = dict(energy=float(ring.energy), particle=lat.particle)
    n, t = a.particles, a.turns
    r0 = (rings.large_ring_bunch(n, seed=0) if a.workload == "large"
          else rings.gaussian(n, seed=0))
    info = atgpu.gpuinfo()
    r = r0.copy(order="F")
    t0 = time.perf_counter()
    atgpu.gpupass(line, r, 1, losses=True, **kw)          # compile + upload
    first = time.perf_counter() - t0
    times = []
    turn = 1
    for _ in range(a.steps):
        t0 = time.perf_counter()
        atgpu.gpupass(line, r, t, turn=turn, reuse=True, losses=True, **kw)
        times.append(time.perf_counter() - t0)
        turn += t
    out = {"impl": "reference atgpu (the reference's CUDA backend, NVRTC-compiled)",
           "r1_r2": "(36,) arrays (applied)" if a.flat_r else "(6, 6) matrices (ignored by atgpu)",
           "device": info, "workload": a.workload, "particles": n, "turns_per_step": t,
           "steps": a.steps, "seconds": times, "first_call_s": first,
           "value": n * t * a.steps / sum(times), "unit": "particle-turns/s",
           "lost": int(np.isnan(r[0]).sum())}
    if a.check:
        m = a.check
        rs = r0[:, :m].copy(order="F")
        rg, rc = rs.copy(order="F"), rs.copy(order="F")
        atgpu.gpupass(line, rg, 1, **kw)
        cpu_atpass(cpu_line, rc, 1, **kw)
        ok = np.all(np.isfinite(rg), axis=0) & np.all(np.isfinite(rc), axis=0)
        d = np.abs(rg[:, ok] - rc[:, ok]).max(axis=1) / np.maximum(
            np.abs(rc[:, ok]).max(axis=1), 1e-300)
        out["one_turn_vs_reference_cpu"] = {"particles": m, "scale_rel_max": float(d.max()),
                                            "per_coordinate": [float(x) for x in d]}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
