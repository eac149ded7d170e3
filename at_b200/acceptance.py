"""Acceptance scans (dynamic aperture, momentum acceptance) on the GPU engine.

Restates the grid modes of the reference's acceptance tools
(pyat/at/acceptance/acceptance.py:29-519 and boundary.py:33-407): a 1-D or
2-D grid of particles around the closed orbit (cartesian, or radial in
(r, theta)) is projected from the observation point to the end of the ring,
tracked for ``nturns`` with the loss map, and the boundary of the surviving
region is extracted.  Every grid point is tracked in ONE engine call, which
is what a GPU is for; the reference's recursive search (a sequence of small
dependent trackings) and flood fill are not provided, and ``use_mp`` /
``gpu_pool`` / ``start_method`` are accepted for signature compatibility
only (the engine decides the parallelism).
"""
from __future__ import annotations

from collections import namedtuple
from enum import Enum

import numpy as np
from scipy.ndimage import binary_dilation, binary_opening

from .tracking import gpupass

__all__ = ["GridMode", "get_acceptance", "get_1d_acceptance", "get_horizontal_acceptance",
           "get_vertical_acceptance", "get_momentum_acceptance"]

_AXES = {"x": 0, "px": 1, "xp": 1, "y": 2, "py": 3, "yp": 3, "dp": 4, "delta": 4, "ct": 5}


class GridMode(Enum):
    """Grid of the 2-D boundary search (boundary.py:20-27)."""
    RADIAL = 0
    CARTESIAN = 1
    RECURSIVE = 2
    FLOODFILL = 3


def _plane_index(planes):
    return np.array([_AXES[p] for p in np.atleast_1d(planes)], dtype=int)


def grid_configuration(planes, npoints, amplitudes, grid_mode, bounds=None, shift_zero=1.0e-6):
    """Grid definition (boundary.py:76-108): ordering (x, y) for CARTESIAN,
    (r, theta) for RADIAL; a 1-D scan is always cartesian."""
    ndims = len(np.atleast_1d(planes))
    if ndims > 2 or ndims == 0:
        raise ValueError("planes can have 1 or 2 element (1D or 2D aperture)")
    if ndims == 1 and grid_mode is GridMode.RADIAL:
        grid_mode = GridMode.CARTESIAN
    if np.shape(np.atleast_1d(npoints)) != (ndims,):
        raise ValueError("npoints shape should be (len(planes),)")
    if np.shape(np.atleast_1d(amplitudes)) != (ndims,):
        raise ValueError("amplitudes shape should be (len(planes),)")
    if bounds is not None and np.shape(np.atleast_2d(bounds)) != (ndims, 2):
        raise ValueError("bounds shape should be (len(planes),2)")
    if grid_mode is GridMode.RADIAL:
        if bounds is None:
            bounds = np.array([[0, 1], [np.pi, 0]])
        bounds = np.array(bounds, dtype=float)
        bounds[0][bounds[0] == 0] = 1.0e-6
    elif grid_mode is GridMode.CARTESIAN:
        if bounds is None:
            bounds = np.array([[p - 1, 1] for p in range(ndims)])
    else:
        raise NotImplementedError("grid mode %s: the engine evaluates full grids "
                                  "(RADIAL or CARTESIAN)" % grid_mode)
    bounds = tuple(map(tuple, np.atleast_2d(bounds)))
    cfg = namedtuple("config", ["planes", "planesi", "amplitudes", "shape", "bounds", "mode",
                                "shift_zero"])
    return cfg(np.atleast_1d(planes), _plane_index(planes), np.atleast_1d(amplitudes),
               np.atleast_1d(np.array(npoints, dtype=np.int32)), bounds, grid_mode, shift_zero)


_Grid = namedtuple("grid", ["grid", "offset"])


def get_parts(config, offset):
    """(6, n) particles of the grid around ``offset`` (+ shift_zero on every
    coordinate) and the grid itself (boundary.py:111-147)."""
    amp, npt, bnd = config.amplitudes, config.shape, config.bounds
    if config.mode is GridMode.CARTESIAN:
        axes = [np.linspace(*b, int(n)) * a for a, b, n in zip(amp, bnd, npt)]
        try:
            g1, g2 = np.meshgrid(*axes)
        except ValueError:
            g1, g2 = np.meshgrid(axes, 0.0)
        g = np.array([g1.flatten(), g2.flatten()])
    else:
        axes = [np.linspace(*b, int(n)) for b, n in zip(bnd, npt)]
        rr, th = np.meshgrid(*axes)
        g = np.array([(amp[0] * np.cos(th) * rr).flatten(), (amp[1] * np.sin(th) * rr).flatten()])
    pind = config.planesi
    parts = np.zeros((6, int(np.prod(npt))))
    parts[pind, :] = [g[i] for i in range(len(pind))]
    off = np.array(offset, dtype=float) + config.shift_zero
    parts = (parts.T + off).T
    return np.asfortranarray(parts), _Grid(np.atleast_2d(g), np.atleast_1d(off[pind]))


def _search_bnd(ma, sa):
    bnd = np.zeros((2, 1))
    for j, m in enumerate(ma):
        bnd = sa[:, j]
        if not m and j > 0:
            bnd = sa[:, j - 1]
            break
    return bnd


def _nearest_order(grid):
    """Boundary points ordered around the origin: the outermost point per
    angle, then a nearest-neighbour walk on the normalised grid
    (boundary.py:171-214)."""
    angle = np.arctan2(*grid)
    norm = np.linalg.norm(grid.T, axis=1)
    val, inv = np.unique(angle, return_inverse=True)
    gf = np.zeros((2, len(val)))
    for i in range(len(val)):
        inds = np.where(inv == i)[0]
        ni = norm[inds]
        gf[:, i] = grid[:, inds[np.where(ni == np.amax(ni))[0]][0]]
    gf = gf[:, np.argsort(np.arctan2(*gf))]
    x, y = gf[0].copy(), gf[1].copy()
    dx = min(np.diff(np.unique(x)))
    dy = min(np.diff(np.unique(y)))
    order = [0]
    for i in range(1, len(x)):
        dd = np.sqrt(((x - x[order[-1]]) / dx) ** 2 + ((y - y[order[-1]]) / dy) ** 2)
        if i <= 3:
            cand = [j for j in np.argsort(dd) if j not in order]
        else:
            sgn = np.sign(order[-1] - order[-2])
            cand = [j for j in np.argsort(dd)
                    if j not in order and np.sign(j - order[-1]) == sgn]
        if cand:
            order.append(cand[0])
    dd = np.sqrt(((x[order[0]] - x[order[-1]]) / dx) ** 2 +
                 ((y[order[0]] - y[order[-1]]) / dy) ** 2)
    if dd < 1.5:
        order.append(order[0])
    return gf[:, order]


def get_grid_boundary(mask, grid, config):
    """Boundary of the surviving region (boundary.py:166-277): the last
    survivor along each ray (RADIAL), the cleaned edge of the surviving set
    (CARTESIAN 2-D), or the last survivor on each side (1-D)."""
    if not np.any(mask):
        return np.zeros(2) if len(config.shape) == 1 else np.zeros((2, 1))
    if config.mode is GridMode.RADIAL:
        angles = np.round(np.arctan2(*grid.grid), decimals=8)
        angles, invi = np.unique(angles, return_inverse=True)
        bnd = np.zeros((2, len(angles)))
        for i in range(len(angles)):
            bnd[:, i] = _search_bnd(mask[invi == i], grid.grid[:, invi == i])
        return bnd
    cnt = np.flip(config.shape)
    if len(cnt) == 1:
        g = grid.grid
        xp, xn = g[0] >= 0, g[0] <= 0
        bp = _search_bnd(mask[xp], g[:, xp])
        bn = _search_bnd(np.flip(mask[xn]), np.flip(g[:, xn], axis=1))
        return np.squeeze([bn[0], bp[0]])
    mask2d = np.reshape(mask.copy(), cnt)
    b1 = binary_opening(mask2d, np.ones((2, 1)))
    b2 = binary_opening(mask2d, np.ones((1, 2)))
    bnd = np.logical_and(b1, b2)
    bnd = np.logical_and(binary_dilation(bnd == 0, border_value=1), bnd)
    return _nearest_order(grid.grid[:, bnd.reshape(mask.shape)])


def _orbit_at(ring, obs, orbit, mode):
    from . import physics

    if orbit is None:
        orbit = physics.find_orbit6(ring, mode=mode)
        if obs:
            r = np.asfortranarray(np.asarray(orbit, dtype=float).reshape(6, 1).copy())
            gpupass(ring, r, 1, end_elem=int(obs), mode=mode)
            orbit = r[:, 0].copy()
    return np.asarray(orbit, dtype=float)


def get_acceptance(ring, planes, npoints, amplitudes, nturns: int = 1024, refpts=None,
                   dp=None, offset=None, bounds=None, grid_mode=GridMode.RADIAL, use_mp=False,
                   gpu_pool=None, verbose: bool = False, divider: int = 2,
                   shift_zero: float = 1.0e-6, start_method=None, mode=None, **kwargs):
    """Acceptance at the observation points ``refpts`` (the reference's
    ``get_acceptance``): returns (boundary, survived, grid), lists of them
    for several points.  Particles of every point are first tracked from it
    to the end of the ring, then all together for ``nturns``.  ``mode``
    selects the engine arithmetic ("fast" or "exact")."""
    if grid_mode in (GridMode.RECURSIVE, GridMode.FLOODFILL):
        raise NotImplementedError("the engine tracks full grids: use GridMode.RADIAL or "
                                  "GridMode.CARTESIAN")
    if dp not in (None, 0.0):
        raise NotImplementedError("dp: the closed orbit is the 6-D one of the ring")
    config = grid_configuration(planes, npoints, amplitudes, grid_mode, bounds=bounds,
                                shift_zero=shift_zero)
    obspt = [None] if refpts is None else [int(k) for k in np.atleast_1d(refpts)]
    offsets = [None] * len(obspt) if offset is None else list(
        np.broadcast_to(np.asarray(offset, dtype=float), (len(obspt), 6)))
    allparts, grids = [], []
    for obs, orb in zip(obspt, offsets):
        orbit = _orbit_at(ring, obs, orb, mode)
        parts, grd = get_parts(config, orbit)
        gpupass(ring, parts, 1, start_elem=0 if obs is None else obs, mode=mode)
        allparts.append(parts)
        grids.append(grd)
    parts = np.asfortranarray(np.concatenate(allparts, axis=1))
    _, ld = gpupass(ring, parts, int(nturns), losses=True, mode=mode)
    masks = np.split(~ld["islost"], len(grids))
    survived = [g.grid[:, m] for g, m in zip(grids, masks)]
    boundary = [get_grid_boundary(m, g, config) for g, m in zip(grids, masks)]
    grids = [g.grid for g in grids]
    if len(obspt) == 1:
        return boundary[0], survived[0], grids[0]
    return boundary, survived, grids


def get_1d_acceptance(ring, plane, resolution, amplitude, nturns: int = 1024, refpts=None,
                      dp=None, offset=None, grid_mode=GridMode.RADIAL, use_mp=False,
                      gpu_pool=None, verbose=False, divider=2, shift_zero=1.0e-6,
                      start_method=None, mode=None, **kwargs):
    """1-D acceptance (acceptance.py:207-317) on a grid of
    ceil(amplitude / resolution) points per side."""
    if len(np.atleast_1d(plane)) != 1:
        raise ValueError("1D acceptance: single plane required")
    if not (np.isscalar(resolution) and np.isscalar(amplitude)):
        raise ValueError("1D acceptance: scalar args required")
    npoint = np.ceil(amplitude / resolution)
    if npoint <= 1:
        raise ValueError("Grid has only one point: increase amplitude or reduce resolution")
    b, s, g = get_acceptance(ring, plane, npoint, amplitude, nturns=nturns, refpts=refpts,
                             dp=dp, offset=offset, grid_mode=grid_mode, shift_zero=shift_zero,
                             mode=mode)
    return np.squeeze(b), s, g


def get_horizontal_acceptance(ring, resolution, amplitude, *args, **kwargs):
    """Horizontal 1-D acceptance (acceptance.py:320-384)."""
    return get_1d_acceptance(ring, "x", resolution, amplitude, *args, **kwargs)


def get_vertical_acceptance(ring, resolution, amplitude, *args, **kwargs):
    """Vertical 1-D acceptance (acceptance.py:387-451)."""
    return get_1d_acceptance(ring, "y", resolution, amplitude, *args, **kwargs)


def get_momentum_acceptance(ring, resolution, amplitude, *args, **kwargs):
    """Momentum acceptance (acceptance.py:454-518)."""
    return get_1d_acceptance(ring, "dp", resolution, amplitude, *args, **kwargs)
