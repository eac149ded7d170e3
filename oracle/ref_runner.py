"""Run the reference's own compiled engine (oracle/_ref) -- test and
baseline infrastructure only.

``oracle/_ref/at`` holds ``pyat/at.c`` and the hot-path integrators compiled
from the reference sources by ``oracle/build_ref.py`` with a generated stub
package; this module imports that ``atpass`` and calls it exactly as pyat's
``_lattice_pass`` does (``pyat/at/tracking/track.py:129``).  It is used as
``python oracle/ref_runner.py <workload> ...`` (a separate process, so the
stub ``at`` package never meets another ``at``) by bench.py's reference arm
and CPU baseline, and by tests that compare the oracle with the reference.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = os.path.join(HERE, "_ref")


def available() -> bool:
    import sysconfig
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.exists(os.path.join(REF, "at", "tracking", "atpass" + ext))


def _import_ref():
    sys.path.insert(0, REF)
    from at.tracking.atpass import atpass  # the reference engine
    import at.lattice as shim
    return atpass, shim


def run(workload: str, nparticles: int, nturns: int, threads: int, seed: int = 0):
    sys.path.insert(0, REPO)
    import numpy as np
    from at_b200 import rings

    atpass, shim = _import_ref()
    if workload == "large":
        ring = rings.large_ring()
        r = rings.gaussian(nparticles, rings.LARGE_SIGMA, seed=seed,
                           centre=rings.LARGE_ORBIT)
    else:
        ring = rings.fodo_ring()
        r = rings.gaussian(nparticles, seed=seed)
    particle = shim.Particle("electron", rest_energy=ring.particle.rest_energy, charge=-1.0)
    kw = dict(energy=float(ring.energy), particle=particle, omp_num_threads=threads,
              losses=True)
    # warm-up call (builds the lattice cache), then the timed call
    w = r[:, : min(64, nparticles)].copy(order="F")
    atpass(list(ring), w, 1, **kw)
    t0 = time.perf_counter()
    atpass(list(ring), r, nturns, **kw)
    dt = time.perf_counter() - t0
    return {"particle_turns": nparticles * nturns, "seconds": dt,
            "rate": nparticles * nturns / dt, "threads": threads,
            "sample": "%d particles x %d turns" % (nparticles, nturns)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["large", "fodo"])
    ap.add_argument("--particles", type=int, default=1000)
    ap.add_argument("--turns", type=int, default=1)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    os.environ.setdefault("OMP_NUM_THREADS", str(args.threads))
    print(json.dumps(run(args.workload, args.particles, args.turns, args.threads)))


if __name__ == "__main__":
    main()
