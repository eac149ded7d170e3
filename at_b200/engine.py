"""Per-device engine objects over the C ABI (include/atb200.h)."""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .lattice import CompiledLattice

_engines: dict[int, "Engine"] = {}
_elock = threading.Lock()


def default_mode() -> int:
    """The arithmetic of calls that do not choose one: "exact" (the
    reference's operation order, within 1e-13 of the reference after one
    turn on every tested ring), or AT_B200_MODE."""
    m = os.environ.get("AT_B200_MODE", "exact").lower()
    if m not in ("fast", "exact"):
        raise ValueError("AT_B200_MODE must be 'fast' or 'exact'")
    return _lib.MODE_FAST if m == "fast" else _lib.MODE_EXACT


def mode_code(mode) -> int:
    if mode is None:
        return default_mode()
    if isinstance(mode, str):
        if mode not in ("fast", "exact"):
            raise ValueError("mode must be 'fast' or 'exact'")
        return _lib.MODE_FAST if mode == "fast" else _lib.MODE_EXACT
    return int(mode)


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().atb_device_count(C.byref(n))
    return n.value if rc == 0 else 0


def device_info(dev: int):
    name = C.create_string_buffer(256)
    ma, mi, sm = C.c_int(), C.c_int(), C.c_int()
    mem = C.c_uint64()
    check(lib().atb_device_info(dev, name, 256, C.byref(ma), C.byref(mi), C.byref(sm), C.byref(mem)))
    return name.value.decode(), ma.value, mi.value, sm.value, mem.value


class Engine:
    """One CUDA engine (handle, stream, buffers) bound to a device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().atb_create(int(device), C.byref(h)))
        self.h = h
        self.device = int(device)
        self.lock = threading.Lock()
        self.nelem = {}            # lattice id -> number of elements

    @classmethod
    def get(cls, device: int = 0) -> "Engine":
        with _elock:
            e = _engines.get(device)
            if e is None:
                e = cls(device)
                _engines[device] = e
            return e

    def close(self):
        if self.h:
            lib().atb_destroy(self.h)
            self.h = None

    # -- launch tuning ------------------------------------------------------
    def set_launch(self, threads: int = 0, seg_cap_words: int = 0, resident_max_words: int = 0,
                   rout_budget_bytes: int = 0, particles_per_thread: int = 0,
                   refill_factor: int = 0):
        """Launch shape of the tracking kernel (0 keeps a setting): threads
        per block, shared-memory segment and resident-table sizes in 64-bit
        words, the refpts snapshot budget, particles per thread (1 or 2) and
        the refill factor of prepared batches (1-64).  Refused while prepared
        batches exist."""
        check(lib().atb_set_launch(self.h, int(threads), int(seg_cap_words),
                                   int(resident_max_words), int(rout_budget_bytes)))
        if particles_per_thread:
            check(lib().atb_set_particles_per_thread(self.h, int(particles_per_thread)))
        if refill_factor:
            check(lib().atb_set_refill_factor(self.h, int(refill_factor)))

    # -- lattices -----------------------------------------------------------
    def upload(self, cl: CompiledLattice) -> int:
        lid = C.c_int32(-1)
        words = np.ascontiguousarray(cl.words, dtype=np.float64)
        off = np.ascontiguousarray(cl.offsets, dtype=np.uint32)
        check(lib().atb_lattice_upload(self.h, ptr(words) if words.size else None,
                                       int(words.size), ptr(off), int(cl.nelem), C.byref(lid)))
        self.nelem[lid.value] = int(cl.nelem)
        return lid.value

    def update(self, lid: int, cl: CompiledLattice):
        words = np.ascontiguousarray(cl.words, dtype=np.float64)
        check(lib().atb_lattice_update(self.h, int(lid), ptr(words) if words.size else None,
                                       int(words.size)))

    def free(self, lid: int):
        check(lib().atb_lattice_free(self.h, int(lid)))
        self.nelem.pop(int(lid), None)

    # -- tracking -----------------------------------------------------------
    def track(self, lid: int, r: np.ndarray, nturns: int, turn0: int = 0, start_elem: int = 0,
              end_elem: int | None = None, refpts: np.ndarray | None = None, losses: bool = False,
              stats: bool = False, mode=None, element: bool = False):
        """Track the (6, N) Fortran-ordered array ``r`` in place through
        elements [start_elem, end_elem) of the first turn and [0, end_elem) of
        the others (``end_elem`` None: every element of the lattice; 0 stops
        before the first element, as in the C interface).

        Returns ``(rout, loss_dict or None, (alive, moments) or None)``."""
        if end_elem is None:
            end_elem = self.nelem[int(lid)]
        npart = r.size // 6
        nref = 0 if refpts is None else int(refpts.size)
        rout = np.empty((6, npart, nref, nturns), dtype=np.float64, order="F")
        ld = None
        islost = lturn = lelem = lcoord = None
        if losses:
            islost = np.zeros(npart, dtype=np.bool_)
            lturn = np.zeros(npart, dtype=np.uint32)
            lelem = np.zeros(npart, dtype=np.uint32)
            lcoord = np.zeros((6, npart), dtype=np.float64, order="F")
        alive = moments = None
        if stats:
            alive = np.zeros(nturns, dtype=np.uint32)
            moments = np.zeros((nturns, 12), dtype=np.float64)
        refs = None if refpts is None else np.ascontiguousarray(refpts, dtype=np.uint32)
        with self.lock:
            check(lib().atb_track(
                self.h, int(lid), ptr(r), npart, int(nturns), int(turn0), int(start_elem),
                int(end_elem), ptr(refs) if nref else None, nref,
                ptr(rout) if (nref and npart) else None, 1 if losses else 0, ptr(islost),
                ptr(lturn), ptr(lelem), ptr(lcoord), ptr(alive), ptr(moments), mode_code(mode),
                _lib.FLAG_ELEMENT if element else 0))
        if losses:
            ld = {"islost": islost, "turn": lturn, "elem": lelem, "coord": lcoord}
        return rout, ld, ((alive, moments) if stats else None)

    def track_device(self, lid: int, r_ptr: int, npart: int, nturns: int, turn0: int = 0,
                     losses=None, alive_ptr: int | None = None, moments_ptr: int | None = None,
                     mode=None, stream: int | None = None):
        """Enqueue tracking of a device-resident (6, N) array (no host copies).

        ``losses`` is ``None`` or a tuple of device pointers
        (islost, lturn, lelem, lcoord)."""
        lp = losses if losses is not None else (None, None, None, None)
        check(lib().atb_track_device(self.h, int(lid), r_ptr, int(npart), int(nturns), int(turn0),
                                     1 if losses is not None else 0, lp[0], lp[1], lp[2], lp[3],
                                     alive_ptr, moments_ptr, mode_code(mode), stream))

    def tangent_device(self, lid: int, r_ptr: int, npart: int, nturns: int, turn0: int,
                       param_elem: np.ndarray, param_order: np.ndarray, value_ptr: int | None,
                       jac_ptr: int, grad_ptr: int | None, lost_ptr: int | None = None,
                       stream: int | None = None):
        """Enqueue tangent tracking of a device-resident (6, N) array: exact
        derivatives d r / d r0 into ``jac_ptr`` (N, 6, 6) and d r / d K into
        ``grad_ptr`` (P, 6, N) for the strengths PolynomB[param_order[q]] of
        elements param_elem[q], whose values are read from ``value_ptr``."""
        pe = np.ascontiguousarray(param_elem, dtype=np.int32)
        po = np.ascontiguousarray(param_order, dtype=np.int32)
        check(lib().atb_tangent_device(self.h, int(lid), r_ptr, int(npart), int(nturns),
                                       int(turn0), ptr(pe) if pe.size else None,
                                       ptr(po) if po.size else None, value_ptr, int(pe.size),
                                       jac_ptr, grad_ptr, lost_ptr, stream))

    def adjoint_forward(self, lid: int, r_ptr: int, npart: int, nturns: int, turn0: int,
                        param_elem: np.ndarray, param_order: np.ndarray, value_ptr: int | None,
                        ckpt_ptr: int | None, stride: int, lost_ptr: int | None = None,
                        stream: int | None = None, estates_ptr: int | None = None):
        """Enqueue the adjoint's forward pass: track the device (6, N) array in
        place with the strengths at ``value_ptr`` substituted, storing the
        state entering every ``stride``-th turn at ``ckpt_ptr`` (and, with
        ``estates_ptr``, every element's entry state of every turn)."""
        pe = np.ascontiguousarray(param_elem, dtype=np.int32)
        po = np.ascontiguousarray(param_order, dtype=np.int32)
        check(lib().atb_adjoint_forward(self.h, int(lid), r_ptr, int(npart), int(nturns),
                                        int(turn0), ptr(pe) if pe.size else None,
                                        ptr(po) if po.size else None, value_ptr, int(pe.size),
                                        ckpt_ptr, int(stride), estates_ptr, lost_ptr, stream))

    def adjoint_backward(self, lid: int, ckpt_ptr: int, npart: int, nturns: int, turn0: int,
                         stride: int, param_elem: np.ndarray, param_order: np.ndarray,
                         value_ptr: int | None, lam_ptr: int, gparam_ptr: int | None,
                         stream: int | None = None, estates_ptr: int | None = None,
                         rfinal_ptr: int | None = None):
        """Enqueue the backward sweep: ``lam_ptr`` ((6, N) device) goes from
        dL/d r_final to dL/d r_initial, ``gparam_ptr`` receives dL/dK (with
        the forward pass's element states and final states, nothing is
        tracked again)."""
        pe = np.ascontiguousarray(param_elem, dtype=np.int32)
        po = np.ascontiguousarray(param_order, dtype=np.int32)
        check(lib().atb_adjoint_backward(self.h, int(lid), ckpt_ptr, int(npart), int(nturns),
                                         int(turn0), int(stride), estates_ptr, rfinal_ptr,
                                         ptr(pe) if pe.size else None,
                                         ptr(po) if po.size else None, value_ptr, int(pe.size),
                                         lam_ptr, gparam_ptr, stream))

    def element_maps(self, lid: int, orbits_ptr: int, m_ptr: int, b_ptr: int,
                     diff_const: float, stream: int | None = None):
        """Enqueue the per-element transfer and diffusion matrices for the
        entrance orbits at ``orbits_ptr`` ((nelem, 6) device array)."""
        check(lib().atb_element_maps(self.h, int(lid), orbits_ptr, m_ptr, b_ptr,
                                     float(diff_const), stream))

    def element_pass(self, lid: int, rin_ptr: int, rout_ptr: int, m_ptr: int | None = None,
                     stream: int | None = None):
        """Enqueue every element alone on its own particle: element i tracks
        row i of the (nelem, 6) device array at ``rin_ptr`` into ``rout_ptr``
        (and its transfer matrix into ``m_ptr`` when given)."""
        check(lib().atb_element_pass(self.h, int(lid), rin_ptr, rout_ptr, m_ptr, stream))

    def track_batch(self, jobs: list[dict], mode=None, stream: int | None = None):
        """One persistent launch over many jobs (dicts with lattice_id, r, np,
        nturns, optional turn0 and losses=(islost, lturn, lelem, lcoord)
        device pointers)."""
        check(lib().atb_track_batch(self.h, self._descs(jobs), len(jobs), mode_code(mode),
                                    stream))

    @staticmethod
    def _descs(jobs: list[dict]):
        arr = (_lib.AtbJobDesc * max(1, len(jobs)))()
        for a, j in zip(arr, jobs):
            a.lattice_id = j["lattice_id"]
            a.nturns = j["nturns"]
            a.turn0 = j.get("turn0", 0)
            lp = j.get("losses")
            a.losses = 1 if lp is not None else 0
            a.r = j["r"]
            a.np = j["np"]
            if lp is not None:
                a.islost, a.lturn, a.lelem, a.lcoord = lp
        return arr

    def batch_prepare(self, jobs: list[dict], mode=None) -> int:
        bid = C.c_int32(-1)
        check(lib().atb_batch_prepare(self.h, self._descs(jobs), len(jobs), mode_code(mode),
                                      C.byref(bid)))
        return bid.value

    def batch_capture(self, bid: int):
        check(lib().atb_batch_capture(self.h, int(bid)))

    def batch_launch(self, bid: int, stream: int | None = None):
        check(lib().atb_batch_launch(self.h, int(bid), stream))

    def batch_free(self, bid: int):
        check(lib().atb_batch_free(self.h, int(bid)))

    def set_rng(self, key: int):
        """Key of the quantum-diffusion random kicks of the launches that
        follow."""
        check(lib().atb_set_rng(self.h, int(key) & 0xFFFFFFFFFFFFFFFF))

    def sync(self, stream: int | None = None):
        check(lib().atb_sync(self.h, stream))
