"""Drop-in tracking entry points with the reference's Python signatures.

``gpupass`` / ``atpass`` replace ``at.tracking.gpu.gpupass``
(``pyat/at/tracking/gpu.pyi:10-28``, ``atgpu/PyInterface.cpp:132-402``) and
``at.tracking.atpass.atpass`` (``pyat/at/tracking/atpass.pyi:11-27``,
``pyat/at.c:340-681``); ``elempass`` replaces ``atpass.elempass``
(``pyat/at.c:683-753``) and ``gpuinfo`` replaces ``gpu.gpuinfo``.  Argument
checks, their order and the exception types follow ``pyat/at.c``; the
tracking itself runs in the CUDA engine (no CPU fallback).
"""
from __future__ import annotations

import math
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import engine as _eng
from .lattice import C0, CompiledLattice, check_integrator, compile_lattice

__all__ = ["gpupass", "atpass", "elempass", "gpuinfo", "reset_cache"]

_defref = np.array([], dtype=np.uint32)


class _State:
    """The reference's static engine state (pyat/at.c:62-75, 346-348)."""

    def __init__(self):
        self.lattice = None            # the list last tracked successfully
        self.compiled: CompiledLattice | None = None
        self.integrator = 4                # integrator the cached table was compiled for
        self.lids: dict[int, int] = {}  # device -> uploaded lattice id
        self.last_turn = 0
        self.lock = threading.RLock()


_state = _State()


def reset_cache():
    """Forget the cached lattice (as a non-reuse call would)."""
    with _state.lock:
        _drop_uploads()
        _state.lattice = None
        _state.compiled = None


def _drop_uploads():
    for dev, lid in list(_state.lids.items()):
        try:
            _eng.Engine.get(dev).free(lid)
        except Exception:  # noqa: BLE001 - best effort
            pass
    _state.lids.clear()


def gpuinfo():
    """[name, 'sm_XY' version, SM count, 'CUDA'] per device
    (atgpu/PyInterface.cpp:95-129)."""
    out = []
    for d in range(_eng.device_count()):
        name, ma, mi, sm, _ = _eng.device_info(d)
        out.append([name, "%d.%d" % (ma, mi), sm, "CUDA"])
    return out


def _check_rin(r_in):
    if not isinstance(r_in, np.ndarray):
        raise TypeError("argument 2 must be numpy.ndarray, not %s" % type(r_in).__name__)
    if r_in.ndim == 0 or r_in.shape[0] != 6:
        raise ValueError("rin is not 6D")
    if r_in.dtype != np.float64:
        raise ValueError("rin is not a double array")
    if not (r_in.flags.f_contiguous and r_in.flags.aligned):
        raise ValueError("rin is not Fortran-aligned")


def _as_int(v, name):
    if isinstance(v, (bool, np.bool_)):
        return int(v)
    if isinstance(v, (int, np.integer)):
        return int(v)
    raise TypeError("%s must be an integer, not %s" % (name, type(v).__name__))


# -- quantum-diffusion random kicks ---------------------------------------------
# The reference keeps one PCG32 stream per process, reset by reset_rng
# (pyat/at.c:833-852); here each call gets a fresh 64-bit key derived from
# (seed, rank, call number), and the kernels derive every kick from the key.
_AT_RNG_STATE = 0x853c49e6748fea9b
_rng = {"seed": _AT_RNG_STATE, "rank": 0, "calls": 0}
_M64 = 0xFFFFFFFFFFFFFFFF


def _mix64(z: int) -> int:
    """The splitmix64 finaliser (Steele, Lea and Flood 2014)."""
    z &= _M64
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & _M64
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & _M64
    return z ^ (z >> 31)


def reset_rng(*, rank: int = 0, seed: int | None = None):
    """Restart the random kicks of QuantDiffPass elements from ``seed``
    (the reference's ``reset_rng(*, rank=0, seed=None)``): the calls that
    follow draw the same kicks after every reset with the same arguments."""
    _rng["seed"] = _AT_RNG_STATE if seed is None else int(seed) & _M64
    _rng["rank"] = int(rank) & _M64
    _rng["calls"] = 0


def _next_rng_key(device: int) -> int:
    k = _mix64(_mix64(_rng["seed"] ^ _mix64(_rng["rank"] + 1)) + _rng["calls"])
    return _mix64(k + 0x9e3779b97f4a7c15 * (device + 1))


def _energy_particle(line, energy, particle):
    """pyat/at.c:275-306 set_energy_particle."""
    e = 0.0
    rest, charge = 0.0, -1.0
    if energy is None and line is not None:
        energy = getattr(line, "energy", None)
    if energy is not None:
        try:
            e = float(energy)
        except (TypeError, ValueError):
            e = 0.0
        if particle is None and line is not None:
            particle = getattr(line, "particle", None)
        if particle is not None:
            try:
                rest = float(getattr(particle, "rest_energy"))
            except (AttributeError, TypeError, ValueError):
                pass
            try:
                charge = float(getattr(particle, "charge"))
            except (AttributeError, TypeError, ValueError):
                pass
    return e, rest, charge


def _devices(gpu_pool):
    if gpu_pool is None:
        return [0]
    if not isinstance(gpu_pool, list):
        raise TypeError("gpu_pool must be a list")
    if len(gpu_pool) == 0:
        raise RuntimeError("at_gpupass() gpu_pool is empty")
    n = _eng.device_count()
    devs = []
    for g in gpu_pool:
        g = _as_int(g, "gpu_pool entry")
        if g < 0 or g >= n:
            raise RuntimeError("Invalid GPU id %d, must be in [0..%d]" % (g, n - 1))
        devs.append(g)
    return devs


def gpupass(line, r_in, nturns, refpts=_defref, *, turn=0, energy=None, particle=None,
            keep_counter=False, reuse=False, losses=False, bunch_spos=None,
            bunch_currents=None, gpu_pool=None, integrator=4, verbose=False, start_elem=0,
            end_elem=None, omp_num_threads=0, harmonic_number=None, fillpattern=None,
            mode=None, stats=False):
    """Track ``r_in`` (6, N) through ``line`` for ``nturns`` turns on the GPU.

    Same arguments and results as the reference ``atpass``/``gpupass``:
    ``r_in`` is updated in place to the final coordinates (lost particles
    become ``(NaN, 0, 0, 0, 0, 0)``); the result is ``rout`` (6, N, R, T)
    with the coordinates at the ``refpts`` elements of every turn, or
    ``(rout, {"islost", "turn", "elem", "coord"})`` when ``losses`` is true.
    ``gpu_pool`` may list several devices: the particles are then split into
    contiguous shards, one per device (the reference accepts one).
    ``integrator`` selects the thick multipoles' symplectic integrator as in
    the reference GPU backend: 1 Euler, 2 McLachlan-Atela 2nd order, 3 Ruth 3rd
    order, 4 Forest-Ruth 4th order (the default, the CPU engine's), 5
    McLachlan-Atela 4th order, 6 Yoshida 6th order; changing it recompiles the
    lattice even with ``reuse``.
    ``mode`` selects "exact" (default: the reference's operation order,
    bit-identical to the reference's C build on the +,-,*,/ path) or "fast"
    arithmetic (FMA contraction and reciprocal reuse: about 2.5x the
    throughput, and up to 2e-13 of each coordinate's scale from the
    reference after one turn of a 2,000-element radiating ring); ``stats=True``
    adds per-turn survivor counts and coordinate sums as a third result.
    ``omp_num_threads``, ``bunch_spos``, ``bunch_currents``,
    ``harmonic_number`` and ``fillpattern`` are accepted for compatibility;
    they only concern collective pass methods, which are not on this path.
    """
    # -- argument parsing (pyat/at.c:399-418) ---------------------------------
    if not isinstance(line, list):
        raise TypeError("argument 1 must be list, not %s" % type(line).__name__)
    if not isinstance(r_in, np.ndarray):
        raise TypeError("argument 2 must be numpy.ndarray, not %s" % type(r_in).__name__)
    nturns = _as_int(nturns, "nturns")
    if refpts is not None and not isinstance(refpts, np.ndarray):
        raise TypeError("refpts must be numpy.ndarray")
    turn = _as_int(turn if turn is not None else 0, "turn")
    if energy is not None and not isinstance(energy, float):
        raise TypeError("energy must be float, not %s" % type(energy).__name__)
    start_elem = _as_int(start_elem if start_elem is not None else 0, "start_elem")
    end_elem = _as_int(end_elem if end_elem is not None else 0, "end_elem")
    integrator = check_integrator(integrator)
    _check_rin(r_in)
    npart = r_in.size // 6
    devs = _devices(gpu_pool)

    with _state.lock:
        # -- lattice cache (pyat/at.c:445-512) --------------------------------
        if not (reuse and _state.lattice is line and _state.compiled is not None and
                _state.integrator == integrator):
            _drop_uploads()
            _state.lattice = None
            _state.compiled = None
            e, rest, charge = _energy_particle(line, energy, particle)
            _state.compiled = compile_lattice(line, e, rest, charge, integrator=integrator)
            _state.integrator = integrator
        cl = _state.compiled
        nelem = cl.nelem
        # -- partial turns (pyat/at.c:514-536) ---------------------------------
        if end_elem == 0:
            end_elem = nelem
        if nelem != 0:
            if start_elem < 0 or start_elem >= nelem:
                raise ValueError("start_elem out of range, %d not in [0..%d]" % (start_elem, nelem - 1))
            if end_elem < 0 or end_elem > nelem:
                raise ValueError("end_elem out of range, %d not in [0..%d]" % (start_elem, nelem))
            if start_elem > end_elem:
                raise ValueError("end_elem must be greater that start_elem")
            if end_elem != nelem and nturns != 1:
                raise ValueError("partial turn tracking not ending at the end of the ring "
                                 "requires nturns=1")
        else:
            start_elem = end_elem = 0
        # -- energy (pyat/at.c:538-551) -----------------------------------------
        e, rest, charge = _energy_particle(line, energy, particle)
        old_version = (cl.energy, cl.rest_energy)
        cl.set_energy(e, rest)
        if refpts is not None and refpts.size and refpts.dtype != np.uint32:
            raise ValueError("refpts is not a uint32 array")
        if refpts is not None and refpts.size == 0:
            refpts = None
        nturn0 = _state.last_turn if keep_counter else turn
        err = cl.first_error(start_elem, end_elem, nturns)
        if err is not None and npart > 0:
            raise err
        # -- upload / refresh on every device of the pool ---------------------
        for d in devs:
            eng = _eng.Engine.get(d)
            if d not in _state.lids:
                _state.lids[d] = eng.upload(cl)
            elif (cl.energy, cl.rest_energy) != old_version:
                eng.update(_state.lids[d], cl)
            eng.set_rng(_next_rng_key(d))
        _rng["calls"] += 1
        # -- track --------------------------------------------------------------
        if len(devs) == 1 or npart < 2 * len(devs):
            eng = _eng.Engine.get(devs[0])
            rout, ld, st = eng.track(_state.lids[devs[0]], r_in, nturns, nturn0, start_elem,
                                     end_elem, refpts, bool(losses), bool(stats), mode)
        else:
            rout, ld, st = _track_sharded(devs, r_in, nturns, nturn0, start_elem, end_elem,
                                          refpts, bool(losses), bool(stats), mode)
        _state.lattice = line
        _state.last_turn = nturn0 + nturns
    out = rout if not losses else (rout, ld)
    if stats:
        return (out, st) if not losses else (rout, ld, st)
    return out


def _track_sharded(devs, r_in, nturns, nturn0, start_elem, end_elem, refpts, losses, stats,
                   mode):
    """Split the particles into one contiguous shard per device; no exchange
    is needed (particles are independent), results are concatenated as
    pyat's format_results does (pyat/at/tracking/utils.py:118-130)."""
    npart = r_in.size // 6
    bounds = np.linspace(0, npart, len(devs) + 1).astype(np.int64)
    shards = [np.asfortranarray(r_in.reshape(6, -1, order="F")[:, a:b]) for a, b in
              zip(bounds[:-1], bounds[1:])]

    def run(k):
        eng = _eng.Engine.get(devs[k])
        return eng.track(_state.lids[devs[k]], shards[k], nturns, nturn0, start_elem, end_elem,
                         refpts, losses, stats, mode)

    with ThreadPoolExecutor(len(devs)) as ex:
        res = list(ex.map(run, range(len(devs))))
    r2 = r_in.reshape(6, -1, order="F")
    for (a, b), s in zip(zip(bounds[:-1], bounds[1:]), shards):
        r2[:, a:b] = s
    rout = np.concatenate([x[0] for x in res], axis=1)
    ld = None
    if losses:
        ld = {k: np.concatenate([x[1][k] for x in res], axis=-1) for k in res[0][1]}
        ld["coord"] = np.asfortranarray(ld["coord"])
    st = None
    if stats:
        st = (sum(x[2][0] for x in res), sum(x[2][1] for x in res))
    return np.asfortranarray(rout), ld, st


def atpass(line, rin, nturns, refpts=_defref, *, turn=0, energy=None, particle=None,
           keep_counter=False, reuse=False, omp_num_threads=0, losses=False, bunch_spos=None,
           bunch_currents=None, start_elem=0, end_elem=None, harmonic_number=None,
           fillpattern=None, mode=None):
    """``at.tracking.atpass.atpass`` signature (pyat/at/tracking/atpass.pyi:11-27),
    tracked on the GPU."""
    return gpupass(line, rin, nturns, refpts, turn=turn, energy=energy, particle=particle,
                   keep_counter=keep_counter, reuse=reuse, losses=losses, start_elem=start_elem,
                   end_elem=end_elem, mode=mode)


def elempass(element, rin, *, energy=None, particle=None, mode=None):
    """Track through one element (pyat/at.c:683-753): turn 0, T0 = 0, no loss
    marking; ``rin`` is updated in place and returned."""
    if element is None or isinstance(element, (list, tuple, np.ndarray)):
        raise TypeError("argument 1 must be an Element")
    if energy is not None and not isinstance(energy, float):
        raise TypeError("energy must be float, not %s" % type(energy).__name__)
    _check_rin(rin)
    e, rest, charge = _energy_particle(None, energy, particle)
    cl = compile_lattice([element], e, rest, charge, t0=0.0)
    err = cl.first_error(0, 1, 1)
    if err is not None:
        raise err
    if rin.size == 0:
        return rin
    eng = _eng.Engine.get(0)
    lid = eng.upload(cl)
    try:
        eng.track(lid, rin, 1, 0, 0, 1, None, False, False, mode, element=True)
    finally:
        eng.free(lid)
    return rin


def revolution_time(line) -> float:
    ring_length = 0.0
    for el in line:
        try:
            ring_length += float(getattr(el, "Length"))
        except (AttributeError, TypeError, ValueError):
            pass
    return ring_length / C0


def _unused(*_):  # pragma: no cover - keeps math imported for type checkers
    return math.pi
