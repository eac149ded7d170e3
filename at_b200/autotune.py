"""Launch-parameter autotuner for the tracking kernel.

The kernel's throughput depends on the threads per block (occupancy versus
per-block staging cost), on the shared-memory segment capacity (how many
blocks fit per SM versus how often a block re-stages the lattice) and on the
particles per thread (two interleaved particles share every parameter load
and hide each other's FP64 latency, at the cost of registers).  The
autotuner times each candidate on a short sample of the actual workload
(copies of the particles, a couple of turns) and keeps the fastest; results
are cached per device, table size and job count in a JSON file
(``$AT_B200_TUNE_CACHE``, default ``~/.cache/at_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
import time

THREADS = (128, 256, 384, 512)
SEG_CAPS = (3072, 4096, 6144)
PPT = (1, 2)


def cache_path() -> str:
    return os.environ.get("AT_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "at_b200",
                                       "autotune.json"))


def _load_cache() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(c: dict):
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p + ".tmp", "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(p + ".tmp", p)
    except OSError:
        pass


def cache_key(device_name: str, table_words: int, njobs: int, nparticles: int, mode) -> str:
    # buckets keep the cache small: table size and particle count to powers of 2
    tw = 1 << max(0, int(table_words).bit_length() - 1)
    npb = 1 << max(0, int(nparticles).bit_length() - 1)
    return "%s|words~%d|jobs=%d|np~%d|%s" % (device_name, tw, njobs, npb, mode)


def tune(engine, run_sample, key: str | None = None, candidates=None, use_cache: bool = True):
    """Pick (threads, seg_cap_words, particles_per_thread) for ``engine``.

    ``run_sample()`` must launch a short, representative sample of the work
    and return its device time in seconds (it is called once per candidate
    after one warm-up call).  Candidates are (threads, seg_cap_words, ppt)
    triples; pairs mean one particle per thread.  The winner is applied with
    ``engine.set_launch`` and returned with the per-candidate timings."""
    cache = _load_cache() if (use_cache and key) else {}
    if key and key in cache and "ppt" in cache[key]:
        best = cache[key]
        engine.set_launch(threads=best["threads"], seg_cap_words=best["seg_cap"],
                          particles_per_thread=best["ppt"])
        return best["threads"], best["seg_cap"], best["ppt"], {"cached": True}
    timings = {}
    last = None

    def measure(cands):
        nonlocal last
        for t, c, k in cands:
            if (t, c, k) in timings:
                continue
            try:
                engine.set_launch(threads=t, seg_cap_words=c, particles_per_thread=k)
                run_sample()
                timings[(t, c, k)] = run_sample()
            except Exception as exc:  # noqa: BLE001 - a candidate that cannot launch is skipped
                timings[(t, c, k)] = float("inf")
                last = exc

    if candidates:
        measure([tuple(c) + (1,) * (3 - len(c)) for c in candidates])
    else:
        # the block shape with one particle per thread first, then the other
        # particle counts at the winning shape (the shape and the particle
        # count interact only through occupancy, which the first pass fixes)
        measure([(t, c, 1) for t in THREADS for c in SEG_CAPS])
        t0, c0, _ = min(timings, key=timings.get)
        measure([(t0, c0, k) for k in PPT])
    best = min(timings, key=timings.get)
    if timings[best] == float("inf"):
        raise RuntimeError("no launch configuration could run: %s" % last)
    engine.set_launch(threads=best[0], seg_cap_words=best[1], particles_per_thread=best[2])
    if key:
        cache = _load_cache()
        cache[key] = {"threads": best[0], "seg_cap": best[1], "ppt": best[2],
                      "seconds": timings[best], "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
        _store_cache(cache)
    return best[0], best[1], best[2], {"%dx%dx%d" % k: v for k, v in timings.items()}
