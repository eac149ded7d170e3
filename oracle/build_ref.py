"""Build recipe for the reference's own C tracking engine (test infrastructure).

This script compiles the reference's C sources *where they lie* (the
``AT_REFERENCE`` directory, else a ``reference`` checkout beside this
repository) with plain ``gcc``, using
the flags of the reference's ``setup.py`` (``-std=c99 -O2 -fopenmp -DPYAT``; the
ISO C mode turns FMA contraction off, so this is the reference arithmetic).
Outputs go only to ``oracle/_ref/`` (git-ignored):

``oracle/_ref/at/``
    ``pyat/at.c`` as ``at/tracking/atpass<EXT>`` plus the hot-path integrators
    (``atintegrators/<PassMethod>.c``) as ``at/integrators/<PassMethod><EXT>``,
    with a tiny generated ``at`` package shim that supplies the two Python types
    ``at.c`` looks up at import (``at.lattice.Particle``/``Element``) and the
    ``at.integrators`` directory it dlopens pass methods from.  Only compiled
    reference code and these generated stubs; no reference Python source.  This
    travels with the repository snapshot and is what the timed reference arm and
    the oracle-validation tests run.

``oracle/_ref/pyat_full/`` (only with ``--full``; never leaves this machine)
    A complete importable pyat (Python package copied from the reference plus
    every extension built here).  Used only by ``tests/golden/make_golden.py`` to
    generate the committed golden fixtures and by CPU tests that cross-check the
    oracle against the reference when the reference tree is present.

``oracle/_ref/pyat_full/at/tracking/gpu<EXT>`` (only with ``--atgpu``)
    The reference's own GPU backend (``atgpu``, its CUDA flavour), built as
    the reference's ``setup.py`` builds it with ``CUDA`` set: ``genheader.py``
    run on a copy of ``atgpu/`` under ``oracle/_ref/atgpu_build/`` to generate
    the kernel header, then the ``*Pass.cpp`` and runtime sources compiled with
    ``-DPYAT -DCUDA`` and linked against ``libcuda`` (the toolkit's link stub
    here; the driver's library where it runs) and ``libnvrtc``.  It compiles
    its generated tracking kernel with NVRTC at run time, so it only loads on a
    machine with a CUDA driver; the full pyat copy does not import it by itself
    (its ``cconfig`` is built without CUDA), callers import
    ``at.tracking.gpu`` explicitly.

The reference's own build system is not run.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys
import sysconfig
from os.path import basename, join, splitext

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = join(HERE, "_ref")
EXT = sysconfig.get_config_var("EXT_SUFFIX") or ".so"

#: the pass methods on the accelerated path (plus IdentityPass for markers)
HOT_PASSES = (
    "DriftPass",
    "StrMPoleSymplectic4Pass",
    "BndMPoleSymplectic4Pass",
    "ThinMPolePass",
    "RFCavityPass",
    "CorrectorPass",
    "AperturePass",
    "IdentityPass",
    "StrMPoleSymplectic4RadPass",
    "BndMPoleSymplectic4RadPass",
)

SHIM_LATTICE = '''\
"""Generated stub: the two types the reference atpass extension looks up."""


class Particle:
    def __init__(self, name="relativistic", rest_energy=0.0, charge=-1.0):
        self.name = name
        self.rest_energy = float(rest_energy)
        self.charge = float(charge)


class Element:
    pass
'''


def _ref_root() -> str:
    """The reference checkout: ``AT_REFERENCE``, else the directory
    ``reference`` beside the repository root."""
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return os.environ.get("AT_REFERENCE", os.path.join(os.path.dirname(repo), "reference"))


def _cflags(ref: str, openmp: bool = True) -> list[str]:
    import numpy

    flags = [
        "-O2", "-g0", "-fPIC", "-shared", "-std=c99", "-DNDEBUG", "-DPYAT",
        "-fno-strict-overflow", "-Wno-unused-function", "-Wno-unknown-pragmas",
        "-w",
        "-I" + numpy.get_include(),
        "-I" + sysconfig.get_paths()["include"],
        "-I" + join(ref, "atintegrators"),
    ]
    if openmp:
        flags += ["-fopenmp", "-DOMP_PARTICLE_THRESHOLD=10"]
    return flags


def _compile(cmd: list[str]) -> tuple[list[str], int, str]:
    p = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, p.returncode, p.stderr


def _run_all(cmds: list[list[str]]) -> None:
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for cmd, rc, err in ex.map(_compile, cmds):
            if rc != 0:
                raise RuntimeError("reference build failed: %s\n%s" % (" ".join(cmd), err))


def _needs(out: str, src: str) -> bool:
    return not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src)


def build_minimal(ref: str, out_root: str = REF_OUT) -> str:
    """Compile at.c and the hot-path integrators into ``<out_root>/at``."""
    pkg = join(out_root, "at")
    for d in (pkg, join(pkg, "tracking"), join(pkg, "integrators")):
        os.makedirs(d, exist_ok=True)
    for d in (pkg, join(pkg, "tracking"), join(pkg, "integrators")):
        init = join(d, "__init__.py")
        if not os.path.exists(init):
            with open(init, "w") as f:
                f.write('"""Generated stub package."""\n')
    with open(join(pkg, "lattice.py"), "w") as f:
        f.write(SHIM_LATTICE)
    cmds = []
    src = join(ref, "pyat", "at.c")
    out = join(pkg, "tracking", "atpass" + EXT)
    if _needs(out, src):
        cmds.append(["gcc", *_cflags(ref), src, "-o", out, "-lm", "-lgomp"])
    for name in HOT_PASSES:
        src = join(ref, "atintegrators", name + ".c")
        out = join(pkg, "integrators", name + EXT)
        if _needs(out, src):
            cmds.append(["gcc", *_cflags(ref), src, "-o", out, "-lm", "-lgomp"])
    _run_all(cmds)
    return out_root


def build_full(ref: str, out_root: str = join(REF_OUT, "pyat_full")) -> str:
    """Complete importable pyat (Python copied from the reference, C built here)."""
    pkg = join(out_root, "at")
    if not os.path.isdir(pkg):
        shutil.copytree(join(ref, "pyat", "at"), pkg)
        shutil.copytree(join(ref, "pyat", "machine_data"), join(out_root, "machine_data"))
        with open(join(pkg, "_version.py"), "w") as f:
            f.write('__version__ = "0.0.0"\n__version_tuple__ = (0, 0, 0)\n')
        # h5py is only needed for v7.3 .mat files; an empty stand-in lets
        # at.load import.
        os.makedirs(join(out_root, "h5py"), exist_ok=True)
        with open(join(out_root, "h5py", "__init__.py"), "w") as f:
            f.write("")
    cmds = []
    integ = join(ref, "atintegrators")
    for src in sorted(glob.glob(join(integ, "*Pass.c"))):
        name = splitext(basename(src))[0]
        out = join(pkg, "integrators", name + EXT)
        if _needs(out, src):
            cmds.append(["gcc", *_cflags(ref), src, "-o", out, "-lm", "-lgomp"])
    for src in sorted(glob.glob(join(integ, "*Pass.cc"))):
        name = splitext(basename(src))[0]
        out = join(pkg, "integrators", name + EXT)
        fl = [f for f in _cflags(ref) if f != "-std=c99"]
        if _needs(out, src):
            cmds.append(["g++", *fl, src, "-o", out, "-lm", "-lgomp"])
    extras = [
        (join(ref, "pyat", "at.c"), join(pkg, "tracking", "atpass" + EXT)),
        (join(ref, "pyat", "at", "cconfig.c"), join(pkg, "cconfig" + EXT)),
        (join(ref, "atmat", "atphysics", "Radiation", "findmpoleraddiffmatrix.c"),
         join(pkg, "physics", "diffmatrix" + EXT)),
        (join(ref, "atmat", "atphysics", "Radiation", "FDW.c"),
         join(pkg, "physics", "wiggdiffmatrix" + EXT)),
    ]
    for src, out in extras:
        if _needs(out, src):
            cmds.append(["gcc", *_cflags(ref), src, "-o", out, "-lm", "-lgomp"])
    _run_all(cmds)
    return out_root


ATGPU_SOURCES = ("AbstractGPU.cpp", "AbstractInterface.cpp", "PyInterface.cpp", "Lattice.cpp",
                 "PassMethodFactory.cpp", "SymplecticIntegrator.cpp", "CudaGPU.cpp")


def build_atgpu(ref: str, out_root: str = join(REF_OUT, "pyat_full")) -> str:
    """The reference's CUDA backend as ``at/tracking/gpu<EXT>`` of the full
    pyat copy (the extension ``at.tracking.gpu`` of the reference's
    setup.py:237-253 with CUDA set)."""
    import numpy

    cuda = os.environ.get("CUDA_PATH", "/usr/local/cuda")
    work = join(REF_OUT, "atgpu_build")
    src = join(work, "atgpu")
    if os.path.isdir(src):
        shutil.rmtree(src)
    shutil.copytree(join(ref, "atgpu"), src)
    # the sources include ../atintegrators/atconstants.h
    link = join(work, "atintegrators")
    if not os.path.lexists(link):
        os.symlink(join(ref, "atintegrators"), link)
    # genheader.py reads atgpu/Element.h and writes atgpu/element.gpuh relative
    # to the working directory, as the reference's setup.py runs it
    subprocess.run([sys.executable, join("atgpu", "genheader.py")], cwd=work, check=True)
    sources = sorted(glob.glob(join(src, "*Pass.cpp"))) + [join(src, f) for f in ATGPU_SOURCES]
    out = join(out_root, "at", "tracking", "gpu" + EXT)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-DPYAT", "-DCUDA", "-Wno-unused-function",
           "-Wno-unknown-pragmas", "-I" + sysconfig.get_paths()["include"],
           "-I" + numpy.get_include(), "-I" + join(cuda, "include"), "-I" + src, *sources,
           "-o", out, "-L" + join(cuda, "lib64"), "-L" + join(cuda, "lib64", "stubs"),
           "-Wl,-rpath," + join(cuda, "lib64"), "-lcuda", "-lnvrtc"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    shutil.rmtree(work)          # build scratch (holds a link into the reference tree)
    if p.returncode != 0:
        raise RuntimeError("atgpu build failed:\n" + p.stderr[-4000:])
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--full", action="store_true", help="also build the full pyat copy")
    ap.add_argument("--atgpu", action="store_true",
                    help="also build the reference's CUDA backend into the full pyat copy")
    args = ap.parse_args(argv)
    ref = _ref_root()
    if not os.path.isdir(join(ref, "atintegrators")):
        print("reference tree not found at %s: nothing to build" % ref)
        return 0
    build_minimal(ref)
    if args.full or args.atgpu:
        build_full(ref)
    if args.atgpu:
        print("atgpu ->", build_atgpu(ref))
    print("reference build ->", REF_OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main())
