"""Callers of the tracking path: closed orbit and one-turn matrix.

Restates, on the GPU engine, pyat's ``find_orbit6`` Newton iteration on the
one-turn map (``pyat/at/physics/orbit.py``; step sizes and convergence from
``pyat/at/lattice/options.py:78-81``) and ``find_m66``'s central differences
(``pyat/at/physics/matrix.py:105-169``).  Each iteration tracks 7 (orbit) or
13 (matrix) particles for one turn through ``gpupass``.
"""
from __future__ import annotations

import math

import numpy as np

from .tracking import gpupass

XYSTEP = 3.0e-8
DPSTEP = 3.0e-6
ORB_CONVERGENCE = 1.0e-12
ORB_MAXITER = 20


def _one_turn(ring, r, mode):
    r = np.asfortranarray(r)
    gpupass(ring, r, 1, mode=mode)
    return r


def _rf_theta(ring) -> np.ndarray:
    """The one-turn path-length slip of the reference particle,
    theta[5] = beta c h / f_rf - L0 with h = round(f_rf L0 / (beta c))
    (pyat/at/physics/orbit.py:319-334); zero for a ring without cavity."""
    from .lattice import C0, element_length

    theta = np.zeros(6)
    freqs = [float(e.Frequency) for e in ring
             if getattr(e, "PassMethod", None) == "RFCavityPass" and hasattr(e, "Frequency")]
    if not freqs:
        return theta
    l0 = 0.0
    for e in ring:
        l0 += element_length(e)
    energy = float(getattr(ring, "energy", 0.0))
    rest = float(getattr(getattr(ring, "particle", None), "rest_energy", 0.0))
    if rest == 0.0 or energy == 0.0:
        beta = 1.0
    else:
        gamma = energy / rest
        beta = math.sqrt(1.0 - 1.0 / gamma / gamma)
    f_rf = freqs[0]
    harm = round(f_rf * l0 / beta / C0)
    theta[5] = beta * C0 * harm / f_rf - l0
    return theta


def energy_loss(ring, elem_track) -> float:
    """Energy lost per turn [eV] by tracking a particle at zero through each
    radiating element alone (pyat/at/physics/energy_loss.py:80-89, method
    TRACKING); ``elem_track(element, r)`` tracks the (6, 1) array ``r``
    through one element in place."""
    delta = 0.0
    for e in ring:
        if str(getattr(e, "PassMethod", "")).endswith("RadPass"):
            r = np.zeros((6, 1), order="F")
            elem_track(e, r)
            delta += r[4, 0]
    return -delta * float(ring.energy)


def _ct_guess(ring, elem_track, u0: float | None = None) -> float:
    """Initial ct of the orbit search: minus the synchronous time shift
    ts = c/(2 pi f) asin(U0 / V) - TimeLag of cavities sharing one frequency
    (pyat/at/physics/energy_loss.py:156-205 and orbit.py:323-330); 0 when
    the ring does not radiate or the cavities differ in frequency or lag."""
    from .lattice import C0

    cavs = [e for e in ring if getattr(e, "PassMethod", None) == "RFCavityPass"]
    if not cavs or (elem_track is None and u0 is None):
        return 0.0
    if u0 is None:
        u0 = energy_loss(ring, elem_track)
    freqs = {float(c.Frequency) for c in cavs}
    lags = {float(getattr(c, "TimeLag", 0.0)) for c in cavs}
    if len(freqs) != 1 or len(lags) != 1:
        return 0.0
    vrf = sum(float(c.Voltage) for c in cavs)
    if u0 > vrf:
        raise RuntimeError("the RF voltage (%.3e eV) is lower than the radiation losses "
                           "(%.3e eV)" % (vrf, u0))
    frf = freqs.pop()
    timelag = C0 / (2 * np.pi * frf) * np.arcsin(u0 / vrf)
    return -(timelag - lags.pop())


def _orbit6(ring, one_turn, guess=None, convergence: float = ORB_CONVERGENCE,
            max_iterations: int = ORB_MAXITER, xy_step: float = XYSTEP,
            dp_step: float = DPSTEP, elem_track=None) -> np.ndarray:
    """Newton iteration of pyat/at/physics/orbit.py:307-368 (_orbit6) with
    ``one_turn(r)`` tracking a (6, 7) array one turn: forward differences
    for the Jacobian, x <- x - (J - 1)^-1 (M(x) - x - theta), until the step
    norm is below ``convergence``.  Without a guess the search starts at the
    synchronous ct of the radiation loss (``elem_track`` tracks single
    elements for it)."""
    if guess is None:
        x = np.zeros(6)
        x[5] = _ct_guess(ring, elem_track)
    else:
        x = np.asarray(guess, dtype=np.float64).copy()
    theta = _rf_theta(ring)
    scaling = np.array([xy_step] * 4 + [dp_step] * 2)
    delta = np.concatenate((np.diag(scaling), np.zeros((6, 1))), axis=1)
    ident = np.identity(6)
    for _ in range(max_iterations):
        r = np.asfortranarray(x.reshape(6, 1) + delta)
        r = one_turn(r)
        if not np.all(np.isfinite(r)):
            raise RuntimeError("find_orbit6: particles lost while searching the orbit")
        ref_out = r[:, 6]
        j6 = (r[:, :6] - r[:, 6:]) / scaling
        b_over_a = np.linalg.solve(j6 - ident, ref_out - x - theta)
        x_next = x - b_over_a
        change = np.linalg.norm(x_next - x)
        x = x_next
        if change <= convergence:
            break
    return x


def find_orbit6(ring, guess=None, convergence: float = ORB_CONVERGENCE,
                max_iterations: int = ORB_MAXITER, xy_step: float = XYSTEP,
                dp_step: float = DPSTEP, mode=None) -> np.ndarray:
    """6-D closed orbit at the ring entrance, as the reference defines it:
    M(x) = x + theta, theta the RF path-length slip of a particle with
    beta < 1 (Newton on the one-turn map tracked by the engine).  The
    synchronous-phase guess takes the radiation energy loss from one launch
    over all elements (optics.energy_loss), equal to one elempass per
    radiating element."""
    from . import optics

    x0 = None
    if guess is None:
        x0 = np.zeros(6)
        x0[5] = _ct_guess(ring, None, u0=optics.energy_loss(ring))
    return _orbit6(ring, lambda r: _one_turn(ring, r, mode), guess if guess is not None else x0,
                   convergence, max_iterations, xy_step, dp_step)


def find_m66(ring, orbit=None, xy_step: float = XYSTEP, dp_step: float = DPSTEP,
             mode=None) -> tuple[np.ndarray, np.ndarray]:
    """One-turn 6x6 matrix around ``orbit`` by central differences
    (pyat/at/physics/matrix.py:147-161)."""
    if orbit is None:
        orbit = find_orbit6(ring, mode=mode)
    steps = np.array([xy_step] * 4 + [dp_step] * 2)
    d = np.diag(0.5 * steps)
    r = np.concatenate((orbit[:, None] + d, orbit[:, None] - d), axis=1)
    r = _one_turn(ring, r, mode)
    m = (r[:, :6] - r[:, 6:]) / steps[None, :]
    return m, orbit
