"""ctypes binding of the C ABI in ``include/atb200.h``.

The shared library is built in-tree (``python -m at_b200.build``).  There is
no fallback: if the library is missing or a call fails, an exception is
raised.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libatb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "atb200.h")

ATB_OK = 0
ATB_ERR_ARG = -1
ATB_ERR_CUDA = -2
ATB_ERR_TIMEOUT = -3
ATB_ERR_NOMEM = -4
ATB_ERR_NOLAT = -5
MODE_EXACT = 0
MODE_FAST = 1
FLAG_ELEMENT = 1

_lock = threading.Lock()
_lib = None

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64


class AtbJobDesc(C.Structure):
    _fields_ = [
        ("lattice_id", C.c_int32), ("nturns", C.c_int32), ("turn0", C.c_int32),
        ("losses", C.c_int32), ("r", C.c_void_p), ("np", C.c_int64),
        ("islost", C.c_void_p), ("lturn", C.c_void_p), ("lelem", C.c_void_p),
        ("lcoord", C.c_void_p),
    ]


_SIGS = {
    "atb_version": ([], C.c_int),
    "atb_last_error": ([], C.c_char_p),
    "atb_device_count": ([C.POINTER(C.c_int)], C.c_int),
    "atb_device_info": ([C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                         C.POINTER(C.c_int), C.POINTER(C.c_uint64)], C.c_int),
    "atb_create": ([C.c_int, C.POINTER(_vp)], C.c_int),
    "atb_destroy": ([_vp], C.c_int),
    "atb_set_launch": ([_vp, C.c_int, C.c_int, C.c_int, _i64], C.c_int),
    "atb_set_particles_per_thread": ([_vp, _i32], C.c_int),
    "atb_set_refill_factor": ([_vp, _i32], C.c_int),
    "atb_lattice_upload": ([_vp, _vp, _i64, _vp, _i32, C.POINTER(_i32)], C.c_int),
    "atb_lattice_update": ([_vp, _i32, _vp, _i64], C.c_int),
    "atb_lattice_free": ([_vp, _i32], C.c_int),
    "atb_track": ([_vp, _i32, _vp, _i64, _i32, _i32, _i32, _i32, _vp, _i32, _vp, _i32, _vp, _vp,
                   _vp, _vp, _vp, _vp, _i32, _i32], C.c_int),
    "atb_track_device": ([_vp, _i32, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp,
                          _i32, _vp], C.c_int),
    "atb_track_batch": ([_vp, C.POINTER(AtbJobDesc), _i32, _i32, _vp], C.c_int),
    "atb_element_maps": ([_vp, _i32, _vp, _vp, _vp, C.c_double, _vp], C.c_int),
    "atb_element_pass": ([_vp, _i32, _vp, _vp, _vp, _vp], C.c_int),
    "atb_serve_open": ([_vp, _vp, _i32, _i32, _i32, _i32, C.POINTER(_vp)], C.c_int),
    "atb_serve_submit": ([_vp, C.POINTER(AtbJobDesc), _i32, C.c_double, _vp,
                          C.POINTER(_i32)], C.c_int),
    "atb_serve_poll": ([_vp, _i32, _i32, _vp, C.POINTER(_i32)], C.c_int),
    "atb_serve_counters": ([_vp, C.POINTER(_i32)], C.c_int),
    "atb_serve_reset": ([_vp], C.c_int),
    "atb_serve_close": ([_vp], C.c_int),
    "atb_tangent_device": ([_vp, _i32, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                            _vp], C.c_int),
    "atb_adjoint_forward": ([_vp, _i32, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _i32, _vp, _i32,
                             _vp, _vp, _vp], C.c_int),
    "atb_adjoint_backward": ([_vp, _i32, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp,
                              _i32, _vp, _vp, _vp], C.c_int),
    "atb_sync": ([_vp, _vp], C.c_int),
    "atb_set_rng": ([_vp, C.c_uint64], C.c_int),
    "atb_batch_prepare": ([_vp, C.POINTER(AtbJobDesc), _i32, _i32, C.POINTER(_i32)], C.c_int),
    "atb_batch_capture": ([_vp, _i32], C.c_int),
    "atb_batch_launch": ([_vp, _i32, _vp], C.c_int),
    "atb_batch_free": ([_vp, _i32], C.c_int),
    "atb_fp64_peak": ([C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "atb_track_noalloc": ([_i32, _vp, _i64, _vp, _vp, _i32, _vp, _i64, _i32, _i32, _i32, _vp,
                           _vp, _vp, _vp, _i32, _vp], C.c_int),
}


class EngineError(RuntimeError):
    """A failing call of the CUDA engine (the message is the engine's)."""

    def __init__(self, code: int, msg: str):
        super().__init__("atb200 error %d: %s" % (code, msg))
        self.code = code


def header_functions() -> list[str]:
    """Names of the functions declared in include/atb200.h."""
    with open(HEADER) as f:
        text = f.read()
    return re.findall(r"^\s*(?:int|const char\*)\s+(atb_\w+)\s*\(", text, flags=re.M)


def lib():
    """The loaded engine; raises if the in-tree library was not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    "the at_b200 CUDA engine is not built (%s missing): run "
                    "`python -m at_b200.build`" % LIB_PATH)
            L = C.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _lib = L
    return _lib


def check(rc: int):
    if rc != ATB_OK:
        msg = lib().atb_last_error()
        raise EngineError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    """Address of a numpy array's data (or None)."""
    if a is None:
        return None
    return a.ctypes.data
