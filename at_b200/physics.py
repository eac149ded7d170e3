"""Callers of the tracking path: closed orbit and one-turn matrix.

Restates, on the GPU engine, pyat's ``find_orbit6`` Newton iteration on the
one-turn map (``pyat/at/physics/orbit.py``; step sizes and convergence from
``pyat/at/lattice/options.py:78-81``) and ``find_m66``'s central differences
(``pyat/at/physics/matrix.py:105-169``).  Each iteration tracks 7 (orbit) or
13 (matrix) particles for one turn through ``gpupass``.
"""
from __future__ import annotations

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


def find_orbit6(ring, guess=None, convergence: float = ORB_CONVERGENCE,
                max_iterations: int = ORB_MAXITER, xy_step: float = XYSTEP,
                dp_step: float = DPSTEP, mode=None) -> np.ndarray:
    """6-D closed orbit at the ring entrance (Newton on the one-turn map)."""
    x = np.zeros(6) if guess is None else np.asarray(guess, dtype=np.float64).copy()
    steps = np.array([xy_step] * 4 + [dp_step] * 2)
    for _ in range(max_iterations):
        r = np.tile(x[:, None], (1, 7))
        r[np.arange(6), np.arange(6)] += steps
        r = _one_turn(ring, r, mode)
        if not np.all(np.isfinite(r)):
            raise RuntimeError("find_orbit6: particles lost while searching the orbit")
        m = (r[:, :6] - r[:, 6:7]) / steps[None, :]
        dx = np.linalg.solve(np.eye(6) - m, r[:, 6] - x)
        x = x + dx
        if np.max(np.abs(dx)) < convergence:
            break
    return x


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
