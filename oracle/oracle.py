"""ORACLE -- test infrastructure only.

Python front of the C restatement in ``oracle/oracle.c`` of the reference
tracking path (``pyat/at.c`` engine + the ``atintegrators`` pass methods on
the accelerated path).  It reads elements by attribute, as the reference's
integrators do (``atintegrators/atelem.c:219-352``), independently of the
product's lattice compiler, and calls the C engine through ctypes.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, and only as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sysconfig

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.c")
LIB = os.path.join(HERE, "liboracle.so")
SRC_Q = os.path.join(HERE, "oracle_q.c")
LIB_Q = os.path.join(HERE, "liboracle_q.so")
#: the same source with FMA contraction allowed: one rounding-level
#: perturbation of every operation, used to tell whether a particle's fate is
#: determined to rounding (tests only)
LIB_FMA = os.path.join(HERE, "liboracle_fma.so")

PASSES = {
    "IdentityPass": 0, "DriftPass": 1, "StrMPoleSymplectic4Pass": 2,
    "StrMPoleSymplectic4RadPass": 3, "BndMPoleSymplectic4Pass": 4,
    "BndMPoleSymplectic4RadPass": 5, "ThinMPolePass": 6, "RFCavityPass": 7,
    "CorrectorPass": 8, "AperturePass": 9, "QuantDiffPass": 10,
}
C0 = 2.99792458e8

_dp = C.POINTER(C.c_double)


class ORng(C.Structure):
    """The engine's random stream (atintegrators/atrandom.c pcg32 state)."""
    _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64), ("spare", C.c_double),
                ("has_spare", C.c_int)]


AT_RNG_STATE = 0x853c49e6748fea9b
# pyat/at.c:74 THREAD_PCG32_INITIALIZER: the stream before any reset_rng
_rng = ORng(AT_RNG_STATE, 1, 0.0, 0)


class OElem(C.Structure):
    _fields_ = [
        ("pass_", C.c_int32), ("MaxOrder", C.c_int32), ("NumIntSteps", C.c_int32),
        ("FringeBendEntrance", C.c_int32), ("FringeBendExit", C.c_int32),
        ("FringeQuadEntrance", C.c_int32), ("FringeQuadExit", C.c_int32), ("Integrator", C.c_int32),
        ("Length", C.c_double), ("BendingAngle", C.c_double), ("EntranceAngle", C.c_double),
        ("ExitAngle", C.c_double), ("FringeInt1", C.c_double), ("FringeInt2", C.c_double),
        ("FullGap", C.c_double), ("Scaling", C.c_double), ("Voltage", C.c_double),
        ("Frequency", C.c_double), ("TimeLag", C.c_double), ("PhaseLag", C.c_double),
        ("bax", C.c_double), ("bay", C.c_double),
        ("PolynomA", _dp), ("PolynomB", _dp), ("fringeIntM0", _dp), ("fringeIntP0", _dp),
        ("R1", _dp), ("R2", _dp), ("T1", _dp), ("T2", _dp), ("RApertures", _dp),
        ("EApertures", _dp), ("KickAngle", _dp), ("Limits", _dp), ("Lmatp", _dp),
    ]


def _stale(lib, srcs):
    return not os.path.exists(lib) or any(os.path.getmtime(lib) < os.path.getmtime(s)
                                          for s in srcs)


def build(force: bool = False) -> str:
    """Compile the C restatement (ISO C99, no FMA contraction, OpenMP), and
    its binary128 variant for high-precision finite differences."""
    if force or _stale(LIB, [SRC]):
        cmd = ["gcc", "-O2", "-std=c99", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
               "-fPIC", "-shared", SRC, "-o", LIB + ".tmp", "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    if has_fma() and (force or _stale(LIB_FMA, [SRC])):
        cmd = ["gcc", "-O2", "-std=gnu99", "-ffp-contract=fast", "-mfma", "-fno-fast-math",
               "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB_FMA + ".tmp", "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(LIB_FMA + ".tmp", LIB_FMA)
    if force or _stale(LIB_Q, [SRC, SRC_Q]):
        cmd = ["gcc", "-O2", "-std=gnu99", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
               "-fPIC", "-shared", SRC_Q, "-o", LIB_Q + ".tmp", "-lquadmath", "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(LIB_Q + ".tmp", LIB_Q)
    return LIB


_lib = None
_lib_q = None
_lib_fma = None


def has_fma() -> bool:
    """Whether this CPU has FMA instructions (the contracted build needs them)."""
    try:
        with open("/proc/cpuinfo") as f:
            return " fma " in f.read()
    except OSError:
        return False


def _load(variant: str = "reference"):
    global _lib, _lib_fma
    if variant == "fma":
        if _lib_fma is None:
            build()
            if not os.path.exists(LIB_FMA):
                raise RuntimeError("the FMA-contracted oracle needs a CPU with FMA")
            _lib_fma = _bind(C.CDLL(LIB_FMA))
        return _lib_fma
    if _lib is None:
        build()
        _lib = _bind(C.CDLL(LIB))
    return _lib


def _bind(L):
    f = L.oracle_track
    f.argtypes = [C.POINTER(OElem), C.c_int, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                  C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                  C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_int, C.POINTER(ORng)]
    f.restype = C.c_int
    L.oracle_rng_seed.argtypes = [C.POINTER(ORng), C.c_uint64, C.c_uint64]
    L.oracle_rng_seed.restype = None
    g = L.oracle_diffmatrix
    g.argtypes = [C.POINTER(OElem), C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    g.restype = C.c_int
    return L


def _load_q():
    global _lib_q
    if _lib_q is None:
        build()
        L = C.CDLL(LIB_Q)
        f = L.oracle_track_hilo
        f.argtypes = [C.POINTER(OElem), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                      C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]
        f.restype = C.c_int
        _lib_q = L
    return _lib_q


def _arr(el, name, keep):
    a = getattr(el, name, None)
    if a is None:
        return None
    a = np.asarray(a, dtype=np.float64).ravel(order="F").copy()
    keep.append(a)
    return a.ctypes.data_as(_dp)


def _elements(line, keep, integrator=4):
    arr = (OElem * max(len(line), 1))()
    for o, el in zip(arr, line):
        pm = el.PassMethod
        if pm not in PASSES:
            raise RuntimeError("PassMethod %s: library, module or trackFunction not found" % pm)
        o.pass_ = PASSES[pm]
        o.Length = float(getattr(el, "Length", 0.0))
        o.MaxOrder = int(getattr(el, "MaxOrder", 0))
        o.NumIntSteps = int(getattr(el, "NumIntSteps", 0))
        o.Integrator = int(integrator)
        o.BendingAngle = float(getattr(el, "BendingAngle", 0.0)) if pm.startswith("Bnd") else 0.0
        o.EntranceAngle = float(getattr(el, "EntranceAngle", 0.0))
        o.ExitAngle = float(getattr(el, "ExitAngle", 0.0))
        o.FringeBendEntrance = int(getattr(el, "FringeBendEntrance", 1))
        o.FringeBendExit = int(getattr(el, "FringeBendExit", 1))
        o.FringeInt1 = float(getattr(el, "FringeInt1", 0.0))
        o.FringeInt2 = float(getattr(el, "FringeInt2", 0.0))
        o.FullGap = float(getattr(el, "FullGap", 0.0))
        o.Scaling = float(getattr(el, "FieldScaling", 1.0))
        o.FringeQuadEntrance = int(getattr(el, "FringeQuadEntrance", 0))
        o.FringeQuadExit = int(getattr(el, "FringeQuadExit", 0))
        o.Voltage = float(getattr(el, "Voltage", 0.0))
        o.Frequency = float(getattr(el, "Frequency", 0.0))
        o.TimeLag = float(getattr(el, "TimeLag", 0.0))
        o.PhaseLag = float(getattr(el, "PhaseLag", 0.0))
        if pm == "ThinMPolePass" and getattr(el, "BendingAngle", None) is not None:
            # ThinMPolePass.c:219-224 with atelem.c:312-315: size dims[0]*dims[1],
            # where dims[1] counts as 0 for a 1-D array
            ba = np.asarray(el.BendingAngle, dtype=np.float64)
            sz = ba.shape[0] * ba.shape[1] if ba.ndim >= 2 else 0
            flat = ba.ravel(order="F")
            o.bax = float(flat[0]) if sz >= 1 else 0.0
            o.bay = float(flat[1]) if sz >= 2 else 0.0
        for name in ("PolynomA", "PolynomB", "fringeIntM0", "fringeIntP0", "R1", "R2", "T1",
                     "T2", "RApertures", "EApertures", "KickAngle", "Limits", "Lmatp"):
            setattr(o, name, _arr(el, name, keep))
    return arr


def integrator_table(k: int):
    """The oracle's (c, d) coefficient lists of integrator ``k``."""
    lib = _load()
    c = (C.c_double * 8)()
    d = (C.c_double * 8)()
    lib.oracle_integ.restype = C.c_int
    n = lib.oracle_integ(int(k), c, d)
    return list(c[:n]), list(d[:n])


def track(line, r, nturns, refpts=None, turn=0, energy=0.0, rest_energy=0.0, losses=False,
          start_elem=0, end_elem=None, nthreads=None, t0=None, element=False, integrator=4,
          arithmetic="reference"):
    """Track the (6, N) Fortran-ordered ``r`` in place with the C oracle.
    ``integrator`` (1-6) selects the thick multipoles' symplectic integrator
    as the reference GPU backend's gpupass does (4 is the CPU engine's).

    ``arithmetic="fma"`` runs the same source compiled with FMA contraction
    (a rounding-level perturbation of every operation; tests only).

    Returns ``(rout, lossdict or None)`` with the reference's layouts."""
    lib = _load(arithmetic)
    keep: list = []
    els = _elements(line, keep, integrator)
    nelem = len(line)
    # pyat/at.c:504 accumulates the lengths one by one; Python's sum() of
    # floats is compensated (3.12+) and can differ in the last bits
    ring_length = 0.0
    for e in line:
        ring_length += float(getattr(e, "Length", 0.0))
    T0 = ring_length / C0 if t0 is None else t0
    if end_elem is None or end_elem == 0:
        end_elem = nelem
    npart = r.size // 6
    refs = np.ascontiguousarray(refpts if refpts is not None else [], dtype=np.uint32)
    rout = np.zeros((6, npart, refs.size, nturns), dtype=np.float64, order="F")
    ld = None
    lost = lturn = lelem = lcoord = None
    if losses:
        lost = np.zeros(npart, dtype=np.uint8)
        lturn = np.zeros(npart, dtype=np.uint32)
        lelem = np.zeros(npart, dtype=np.uint32)
        lcoord = np.zeros((6, npart), dtype=np.float64, order="F")
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    rc = lib.oracle_track(els, nelem, r.ctypes.data, npart, nturns, turn, start_elem, end_elem,
                          refs.ctypes.data if refs.size else None, refs.size,
                          1 if losses else 0, 0 if element else 1, energy, rest_energy, T0,
                          rout.ctypes.data if refs.size else None,
                          None if lost is None else lost.ctypes.data,
                          None if lturn is None else lturn.ctypes.data,
                          None if lelem is None else lelem.ctypes.data,
                          None if lcoord is None else lcoord.ctypes.data, nthreads,
                          C.byref(_rng))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    if losses:
        ld = {"islost": lost.astype(bool), "turn": lturn, "elem": lelem, "coord": lcoord}
    return rout, ld


def reset_rng(*, rank=0, seed=None):
    """pyat/at.c:833-852 reset_rng: reseed the engine's random stream."""
    lib = _load()
    lib.oracle_rng_seed(C.byref(_rng), AT_RNG_STATE if seed is None else int(seed), int(rank))


def diffmatrix(element, orbit, energy=0.0, rest_energy=0.0):
    """The Ohmi diffusion matrix of one element for a particle at ``orbit``
    (the reference's ``diffusion_matrix``), as a (6, 6) array."""
    lib = _load()
    keep: list = []
    els = _elements([element], keep)
    orb = np.ascontiguousarray(np.asarray(orbit, dtype=np.float64).ravel())
    out = np.zeros(36, dtype=np.float64)
    lib.oracle_diffmatrix(els, orb.ctypes.data, energy, rest_energy, out.ctypes.data)
    return out.reshape(6, 6, order="F")


def track_quad(line, r, nturns, turn=0, energy=0.0, rest_energy=0.0, nthreads=None):
    """Track the (6, N) array ``r`` (not modified) for whole turns with the
    oracle's integrators in binary128; returns ``(hi, lo)``, two (6, N)
    double arrays whose sum is the binary128 result.  For finite differences
    of the map far below double's rounding floor."""
    lib = _load_q()
    keep: list = []
    els = _elements(line, keep)
    ring_length = 0.0
    for e in line:
        ring_length += float(getattr(e, "Length", 0.0))
    T0 = ring_length / C0
    rin = np.asfortranarray(r, dtype=np.float64)
    npart = rin.size // 6
    hi = np.empty((6, npart), dtype=np.float64, order="F")
    lo = np.empty((6, npart), dtype=np.float64, order="F")
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    rc = lib.oracle_track_hilo(els, len(line), rin.ctypes.data, hi.ctypes.data, lo.ctypes.data,
                               npart, nturns, turn, energy, rest_energy, T0, nthreads)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return hi, lo


def ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"
