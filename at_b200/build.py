"""Build the CUDA engine ``at_b200/libatb200.so`` in-tree for sm_100a.

The kernel translation units are compiled with different contraction flags
(``-fmad=false`` for the exact-order tracking kernel and the tangent kernel),
then linked with the host runtime into one shared library exporting the C ABI
of ``include/atb200.h``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libatb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC, "-I" + INCLUDE]

UNITS = [
    ("track_exact.cu", ["-fmad=false"]),
    ("track_fast.cu", ["-fmad=true"]),
    ("tangent.cu", ["-fmad=false"]),
    ("adjoint.cu", ["-fmad=false"]),
    ("atb200.cu", []),
    ("atb_noalloc.cu", []),
]
DEPS = ["atb_physics.cuh", "atb_dual.cuh", "track_kernel.cuh", "tangent_kernel.cuh",
        "adjoint_kernel.cuh",
        "atb_diffusion.cuh", "atb_integrators.h",
        "atb_kernel_api.h", "atb_table.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build the CUDA engine")


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(INCLUDE, "atb200.h"), __file__]
    objs, jobs = [], []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + deps):
            cmd = [nv, *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            jobs.append((src, cmd))
    # the units are independent: compile them side by side
    running = [(src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True)) for src, cmd in jobs]
    failed = []
    for src, proc in running:
        _, err = proc.communicate()
        if proc.returncode != 0:
            failed.append("nvcc failed for %s:\n%s" % (src, err))
        elif ptxas_info or verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("\n".join(failed))
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [nv, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd))
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n%s" % p.stderr)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
