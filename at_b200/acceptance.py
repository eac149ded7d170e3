"""Dynamic-aperture and momentum-acceptance scans on the GPU engine.

API: the reference's ``get_acceptance``, ``get_1d_acceptance`` and the
horizontal, vertical and momentum wrappers (pyat/at/acceptance/acceptance.py:
29-519), with its four ``GridMode`` searches (boundary.py:20-27) and the same
returned (boundary, survived, tracked) arrays.  The searches are designed for
a GPU, where one launch of a few thousand particles costs about as much as
one of a single particle:

* RADIAL / CARTESIAN grids: every point of every observation point is a
  particle of ONE engine call (after one partial turn that carries each
  observation point's particles to the end of the ring, as the reference
  does, boundary.py:313-341).
* FLOODFILL: the reference walks the grid from its border inwards, tracking
  one particle at a time and queueing the neighbours of every lost one
  (floodfill_acceptance.py:22-238).  Which points that walk reaches depends
  only on which grid points are lost, and particles are independent, so here
  ONE launch tracks the whole grid and the walk is replayed on the host from
  the loss map: same tracked set, survivors and loss turns.
* RECURSIVE: the reference's per-ray search (boundary.py:409-500) advances
  every ray by one step per tracking call and halves the step after a loss.
  Here each launch is speculative: for every ray still searching it also
  tracks the points of its next few steps under either outcome, so the
  replayed search finds most of its points already tracked and needs several
  times fewer launches.  The replay keeps the reference's step arithmetic and
  its rule that a point within numpy ``allclose(rtol=1e-9)`` of an earlier one
  reuses that point's result, so boundaries, survivors and tracked points are
  the reference's.

``use_mp``, ``gpu_pool`` and ``start_method`` are accepted for signature
compatibility (the engine is the GPU); as with the reference's GPU mode, the
1-D scans keep the requested grid mode.  ``mode`` selects the engine
arithmetic ("exact", the default, or "fast").
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum

import numpy as np

from .tracking import gpupass

__all__ = ["GridMode", "Scan", "make_scan", "scan_grid", "scan_particles", "grid_boundary",
           "floodfill_walk", "get_acceptance", "get_1d_acceptance",
           "get_horizontal_acceptance", "get_vertical_acceptance", "get_momentum_acceptance"]

_COORD = {"x": 0, "px": 1, "xp": 1, "y": 2, "py": 3, "yp": 3, "dp": 4, "delta": 4, "ct": 5}


class GridMode(Enum):
    """How the 2-D boundary is searched (values as the reference's)."""
    RADIAL = 0        #: full (r, theta) grid
    CARTESIAN = 1     #: full (x, y) grid
    RECURSIVE = 2     #: per-ray step-halving search
    FLOODFILL = 3     #: from the grid's border inwards through lost points


@dataclass(frozen=True)
class Scan:
    """One acceptance scan: the scanned coordinates, their ranges and the
    search mode.  ``bounds[k]`` scales ``amplitudes[k]`` (cartesian and flood
    fill), or gives the radius and angle ranges (radial and recursive)."""
    planes: tuple
    coords: tuple
    amplitudes: np.ndarray
    counts: np.ndarray
    bounds: np.ndarray
    mode: GridMode
    shift_zero: float

    @property
    def ndim(self) -> int:
        return len(self.coords)


def make_scan(planes, npoints, amplitudes, grid_mode=GridMode.RADIAL, bounds=None,
              shift_zero=1.0e-6) -> Scan:
    """Validate and complete a scan definition.  A 1-D radial scan is a
    cartesian one.  Default ranges: radius (0, 1] (a zero radius becomes
    1e-6, where the ray still has a direction) over angles pi -> 0;
    cartesian and flood fill [-1, 1] on the first axis and [0, 1] on the
    second."""
    names = tuple(np.atleast_1d(planes).tolist())
    nd = len(names)
    if nd not in (1, 2):
        raise ValueError("an acceptance scan has one or two planes, got %d" % nd)
    try:
        coords = tuple(_COORD[p] for p in names)
    except KeyError as exc:
        raise ValueError("unknown plane %s" % exc) from None
    counts = np.atleast_1d(np.asarray(npoints)).astype(np.int32)
    amps = np.atleast_1d(np.asarray(amplitudes, dtype=np.float64))
    if counts.shape != (nd,) or amps.shape != (nd,):
        raise ValueError("npoints and amplitudes need one entry per plane (%d)" % nd)
    mode = grid_mode
    if nd == 1 and mode is GridMode.RADIAL:
        mode = GridMode.CARTESIAN
    if mode in (GridMode.RADIAL, GridMode.RECURSIVE):
        b = np.array([[0.0, 1.0], [np.pi, 0.0]]) if bounds is None else np.array(
            bounds, dtype=np.float64, ndmin=2)
        b[0][b[0] == 0] = 1.0e-6
    elif mode in (GridMode.CARTESIAN, GridMode.FLOODFILL):
        b = (np.array([[-1.0, 1.0], [0.0, 1.0]])[:nd] if bounds is None
             else np.array(bounds, dtype=np.float64, ndmin=2))
    else:
        raise ValueError("unknown grid mode %r" % (grid_mode,))
    if bounds is not None and b.shape != (nd, 2):
        raise ValueError("bounds need a (low, high) pair per plane")
    return Scan(names, coords, amps, counts, b, mode, float(shift_zero))


def scan_grid(scan: Scan) -> np.ndarray:
    """The (2, n) grid of a RADIAL or CARTESIAN scan in the reference's point
    order: the second axis outermost (rays of increasing radius, one angle
    after the other, for RADIAL); a 1-D grid has a zero second row."""
    if scan.mode is GridMode.RADIAL:
        radius = np.linspace(*scan.bounds[0], scan.counts[0])
        angle = np.linspace(*scan.bounds[1], scan.counts[1])
        rr = np.tile(radius, angle.size)
        th = np.repeat(angle, radius.size)
        return np.array([scan.amplitudes[0] * np.cos(th) * rr,
                         scan.amplitudes[1] * np.sin(th) * rr])
    axes = [np.linspace(*scan.bounds[k], scan.counts[k]) * scan.amplitudes[k]
            for k in range(scan.ndim)]
    if scan.ndim == 1:
        return np.array([axes[0], np.zeros_like(axes[0])])
    return np.array([np.tile(axes[0], axes[1].size), np.repeat(axes[1], axes[0].size)])


def scan_particles(scan: Scan, centre) -> tuple[np.ndarray, np.ndarray]:
    """(6, n) particles of a grid scan: the grid on the scanned coordinates,
    plus ``centre + shift_zero`` on every coordinate.  Returns the particles
    and the grid."""
    g = scan_grid(scan)
    base = np.asarray(centre, dtype=np.float64) + scan.shift_zero
    parts = np.zeros((6, g.shape[1]))
    for k, c in enumerate(scan.coords):
        parts[c] = g[k]
    parts += base[:, None]
    return np.asfortranarray(parts), g


# -- boundaries -------------------------------------------------------------------

def _edge_index(alive: np.ndarray) -> int:
    """Along a ray (points in order of increasing amplitude): the point just
    before the first loss after the ray's first point, or the last point if
    none is lost.  The ray's first point counts as reached whatever its
    fate (the reference's rule)."""
    dead = np.flatnonzero(~alive[1:])
    return int(dead[0]) if dead.size else alive.size - 1


def _radial_edges(alive, grid):
    """One boundary point per ray; rays are told apart by their direction
    (the angle of atan2(first, second) coordinate, to 8 decimals) and come
    in increasing order of it."""
    key = np.round(np.arctan2(grid[0], grid[1]), 8)
    rays, member = np.unique(key, return_inverse=True)
    out = np.empty((2, rays.size))
    for k in range(rays.size):
        idx = np.flatnonzero(member == k)
        out[:, k] = grid[:, idx[_edge_index(alive[idx])]]
    return out


def _line_edges(alive, grid):
    """1-D scan: the edge on the negative side (walking down from zero) and
    on the positive side (walking up), first coordinate only."""
    up = np.flatnonzero(grid[0] >= 0)
    down = np.flatnonzero(grid[0] <= 0)[::-1]
    return np.array([grid[0, down[_edge_index(alive[down])]],
                     grid[0, up[_edge_index(alive[up])]]])


def _with_partner(m: np.ndarray, axis: int) -> np.ndarray:
    """Points of ``m`` that have a neighbour in ``m`` along ``axis``
    (morphological opening by a two-point segment; outside the grid is
    empty)."""
    lo = np.zeros_like(m)
    hi = np.zeros_like(m)
    if axis == 0:
        lo[1:] = m[:-1]
        hi[:-1] = m[1:]
    else:
        lo[:, 1:] = m[:, :-1]
        hi[:, :-1] = m[:, 1:]
    return m & (lo | hi)


def _cartesian_edges(alive, grid, counts):
    """The edge of the cleaned surviving region of a 2-D cartesian grid.

    Cleaning keeps a survivor only if it has a surviving neighbour both
    along x and along y (isolated points and one-point-wide spikes go).  The
    edge is the set of cleaned points with a 4-neighbour outside the cleaned
    set or on the grid's border.  As a contour it is listed by direction:
    for each direction from the origin the outermost edge point, in
    increasing angle atan2(x, y), closed by repeating the first point when
    the two ends are neighbours on the grid."""
    m = alive.reshape(counts[1], counts[0])
    clean = _with_partner(m, 0) & _with_partner(m, 1)
    inner = np.zeros_like(clean)
    inner[1:-1, 1:-1] = (clean[1:-1, 1:-1] & clean[:-2, 1:-1] & clean[2:, 1:-1] &
                         clean[1:-1, :-2] & clean[1:-1, 2:])
    pts = grid[:, (clean & ~inner).ravel()]
    if pts.shape[1] == 0:
        return np.zeros((2, 1))
    direction = np.arctan2(pts[0], pts[1])
    radius = np.hypot(pts[0], pts[1])
    order = np.lexsort((-radius, direction))
    keep = np.ones(order.size, dtype=bool)
    keep[1:] = direction[order[1:]] != direction[order[:-1]]
    contour = pts[:, order[keep]]
    steps = [np.diff(np.unique(grid[k])).min() for k in range(2)]
    gap = np.hypot(*[(contour[k, 0] - contour[k, -1]) / steps[k] for k in range(2)])
    if contour.shape[1] > 1 and gap < 1.5:
        contour = np.concatenate([contour, contour[:, :1]], axis=1)
    return contour


def grid_boundary(alive: np.ndarray, grid: np.ndarray, scan: Scan) -> np.ndarray:
    """Boundary of the surviving part of a RADIAL or CARTESIAN grid: per
    ray for RADIAL, the two edges of a 1-D scan, the contour of a 2-D
    cartesian grid.  With no survivor it is zero, as in the reference."""
    alive = np.asarray(alive, dtype=bool)
    if not alive.any():
        return np.zeros(2) if scan.ndim == 1 else np.zeros((2, 1))
    if scan.mode is GridMode.RADIAL:
        return _radial_edges(alive, grid)
    if scan.ndim == 1:
        return _line_edges(alive, grid)
    return _cartesian_edges(alive, grid, scan.counts)


# -- engine calls -----------------------------------------------------------------

def _rotated(ring, start: int):
    """The ring starting at element ``start`` (the reference's Lattice.rotate)."""
    if not start:
        return ring
    elems = list(ring[start:]) + list(ring[:start])
    try:
        return type(ring)(elems, energy=ring.energy, particle=ring.particle)
    except TypeError:
        out = type(ring)(elems)
        for attr in ("energy", "particle"):
            if hasattr(ring, attr):
                setattr(out, attr, getattr(ring, attr))
        return out


def _orbit_at(ring, obs, orbit, mode):
    """The 6-D closed orbit at element ``obs`` (element 0 if None), or the
    given ``orbit``."""
    from . import physics

    if orbit is not None:
        return np.asarray(orbit, dtype=np.float64)
    orb = np.asarray(physics.find_orbit6(ring, mode=mode), dtype=np.float64)
    if obs:
        r = np.asfortranarray(orb.reshape(6, 1).copy())
        gpupass(ring, r, 1, end_elem=int(obs), mode=mode)
        orb = r[:, 0].copy()
    return orb


def _lost(ring, parts, nturns, mode):
    """Track (6, n) particles for ``nturns`` turns: loss flags and loss
    turns."""
    if parts.shape[1] == 0:
        return np.zeros(0, dtype=bool), np.zeros(0, dtype=np.uint32)
    r = np.asfortranarray(parts)
    _, ld = gpupass(ring, r, int(nturns), losses=True, mode=mode)
    return ld["islost"].copy(), ld["turn"].copy()


def _to_ring_end(ring, parts, start, mode):
    """Carry (6, n) particles, in place, from element ``start`` to the end
    of the ring (a whole turn from element 0)."""
    gpupass(ring, parts, 1, start_elem=int(start), mode=mode)


# -- flood fill ---------------------------------------------------------------------

def floodfill_walk(lost: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """The points a border-inwards flood fill reaches on an (nx, ny) grid
    indexed i = ix * ny + iy: every border point, and every 4-neighbour of a
    reached point that is lost (breadth first over the lost region)."""
    lost = np.asarray(lost, dtype=bool).reshape(nx, ny)
    reached = np.zeros((nx, ny), dtype=bool)
    reached[[0, -1], :] = True
    reached[:, [0, -1]] = True
    while True:
        src = reached & lost
        grow = np.zeros_like(reached)
        grow[1:, :] |= src[:-1, :]
        grow[:-1, :] |= src[1:, :]
        grow[:, 1:] |= src[:, :-1]
        grow[:, :-1] |= src[:, 1:]
        new = grow & ~reached
        if not new.any():
            return reached.ravel()
        reached |= new


def _floodfill(ring, scan: Scan, nturns, centre, mode):
    """One observation point of a FLOODFILL scan (the ring already starts
    there): returns the (4, n) table of the reference's flood fill (grid
    coordinates of the reached points in grid order, turns survived, lost
    flag)."""
    lo_hi = scan.bounds * scan.amplitudes[:, None]
    if lo_hi[0, 0] == lo_hi[0, 1] or lo_hi[1, 0] == lo_hi[1, 1]:
        return np.zeros((4, 0))
    nx, ny = (int(v) for v in scan.counts)
    xs = np.linspace(lo_hi[0].min(), lo_hi[0].max(), nx)
    ys = np.linspace(lo_hi[1].min(), lo_hi[1].max(), ny)
    pts = np.array([np.repeat(xs, ny), np.tile(ys, nx)])
    parts = np.zeros((6, nx * ny)) + np.asarray(centre, dtype=np.float64)[:, None]
    parts[scan.coords[0]] += pts[0]
    parts[scan.coords[1]] += pts[1]
    lost, lturn = _lost(ring, parts, nturns, mode)
    reached = floodfill_walk(lost, nx, ny)
    turns = np.where(lost, lturn, nturns).astype(np.float64)
    return np.vstack([pts[:, reached], turns[reached], lost[reached].astype(np.float64)])


# -- recursive search ---------------------------------------------------------------

def _seen(p: np.ndarray, pool: np.ndarray) -> np.ndarray:
    """For each row of ``p``: is it within numpy allclose(rtol=1e-9,
    atol=1e-8) of some row of ``pool``?"""
    if pool.shape[0] == 0 or p.shape[0] == 0:
        return np.zeros(p.shape[0], dtype=bool)
    tol = 1e-8 + 1e-9 * np.abs(pool)[None, :, :]
    return np.all(np.abs(p[:, None, :] - pool[None, :, :]) <= tol, axis=2).any(axis=1)


class _Ray:
    """One ray's search state and its step rule: advance by step * f while
    the particles survive; after a loss step back by step * min(1, 2 f)
    (to zero if that would cross it) and scale f by 1/divider, until f is at
    the resolution."""

    def __init__(self, direction, steps, divider, ftol):
        self.d = direction            # (nplanes,) rounded cos/sin
        self.steps = steps            # (nplanes,) initial step per plane
        self.shrink = 1.0 / divider
        self.ftol = ftol

    def advance(self, pos, f):
        return pos + self.d * self.steps * f

    def retreat(self, pos, f):
        back = self.d * self.steps * min(1.0, 2.0 * f)
        if np.any(np.abs(back) > np.abs(pos)):
            return np.zeros_like(pos), f * self.shrink
        return pos - back, f * self.shrink

    def after(self, pos, f, depth):
        """The points the ray may track in its next ``depth`` steps once the
        point ``pos`` (reached with factor f) is known, whichever way each
        step ends."""
        out = []
        frontier = [(pos, f)]
        for _ in range(depth):
            nxt = []
            for p, g in frontier:
                nxt.append((self.advance(p, g), g))                    # p survived
                if g > self.ftol:                                      # p lost
                    q, h = self.retreat(p, g)
                    nxt.append((self.advance(q, h), h))
            out.extend(p for p, _ in nxt)
            frontier = nxt
        return out


def _recursive(ring, scan: Scan, nturns, centre, divider, mode, depth=3):
    """RECURSIVE search at one observation point (the ring starts there).
    Returns (boundary, survived, tracked) as the reference does.  The search
    itself is the reference's, replayed step by step; only its tracking
    calls change: a point it needs that is not known yet triggers one launch
    of that step's new points together with every such ray's possible
    points of the next ``depth`` steps."""
    nd = scan.ndim
    rtol = float(np.min(scan.amplitudes / scan.counts))
    steps = scan.amplitudes.astype(np.float64)
    ftol = float(np.min(rtol / steps))
    angles = np.atleast_1d(np.linspace(*scan.bounds[1], scan.counts[1] if nd == 2 else 2))
    cs = np.around(np.squeeze([np.cos(angles), np.sin(angles)]), decimals=9)
    rays = [_Ray(cs[:nd, i], steps, divider, ftol) for i in range(angles.size)]
    n = len(rays)
    pos = np.zeros((n, nd))
    fact = np.ones(n)
    alive = np.ones(n, dtype=bool)
    tracked = np.zeros((0, nd))            # every point tracked, in order
    kept = np.zeros((0, nd))               # the tracked survivors
    known: dict[bytes, bool] = {}          # engine results by exact position
    centre = np.asarray(centre, dtype=np.float64)
    launches = 0

    def run(points):
        parts = np.zeros((6, len(points))) + centre[:, None]
        for k, c in enumerate(scan.coords):
            parts[c] = np.array([p[k] for p in points]) + centre[c]
        lost, _ = _lost(ring, parts, nturns, mode)
        for p, lo in zip(points, lost):
            known[p.tobytes()] = not lo

    while alive.any():
        for i in np.flatnonzero(alive):
            pos[i] = rays[i].advance(pos[i], fact[i])
        idx = np.flatnonzero(~_seen(pos, tracked))
        alive = _seen(pos, kept)
        if idx.size:
            if any(pos[i].tobytes() not in known for i in idx):
                batch = {}
                for i in idx:
                    for p in [pos[i].copy()] + rays[i].after(pos[i], fact[i], depth):
                        if p.tobytes() not in known:
                            batch.setdefault(p.tobytes(), p)
                run(list(batch.values()))
                launches += 1
            got = np.array([known[pos[i].tobytes()] for i in idx])
            alive[idx] = got
            tracked = np.vstack([tracked, pos[idx]])
            kept = np.vstack([kept, pos[idx][got]])
        for i in range(n):
            if not alive[i] and fact[i] > ftol:
                pos[i], fact[i] = rays[i].retreat(pos[i], fact[i])
                alive[i] = True
    for i in range(n):
        pos[i] = pos[i] - rays[i].d * rays[i].steps * fact[i]
    _recursive.launches = launches
    return np.squeeze(pos.T), kept.T, tracked.T


# -- public scans -----------------------------------------------------------------

def get_acceptance(ring, planes, npoints, amplitudes, nturns: int = 1024, refpts=None,
                   dp=None, offset=None, bounds=None, grid_mode=GridMode.RADIAL, use_mp=False,
                   gpu_pool=None, verbose: bool = False, divider: int = 2,
                   shift_zero: float = 1.0e-6, start_method=None, mode="exact", **kwargs):
    """Acceptance at the observation points ``refpts`` (element 0 by
    default), as the reference's ``get_acceptance``: returns (boundary,
    survived, tracked), each a list with one entry per point when several
    are given.  ``offset`` replaces the closed orbit as the scan's centre."""
    if dp not in (None, 0.0):
        raise NotImplementedError("dp: scans are centred on the ring's 6-D closed orbit")
    scan = make_scan(planes, npoints, amplitudes, grid_mode, bounds, shift_zero)
    obs = [0] if refpts is None else [int(k) for k in np.atleast_1d(refpts)]
    centres = ([None] * len(obs) if offset is None else
               list(np.broadcast_to(np.asarray(offset, dtype=np.float64), (len(obs), 6))))
    if scan.mode is GridMode.RECURSIVE:
        out = [_recursive(_rotated(ring, o), scan, nturns, _orbit_at(ring, o, c, mode),
                          divider, mode) for o, c in zip(obs, centres)]
    elif scan.mode is GridMode.FLOODFILL:
        if scan.ndim != 2:
            raise ValueError("a flood fill needs two planes")
        out = []
        for o, c in zip(obs, centres):
            data = _floodfill(_rotated(ring, o), scan, nturns, _orbit_at(ring, o, c, mode), mode)
            surv = data[0:2, data[3] == 0]
            order = np.argsort(np.arctan2(surv[1, :], surv[0, :]))
            out.append((surv[:, order], surv, data[0:2]))
    else:
        allparts, grids = [], []
        for o, c in zip(obs, centres):
            parts, g = scan_particles(scan, _orbit_at(ring, o, c, mode))
            _to_ring_end(ring, parts, o, mode)
            allparts.append(parts)
            grids.append(g)
        lost, _ = _lost(ring, np.concatenate(allparts, axis=1), nturns, mode)
        out = []
        for g, lo in zip(grids, np.split(lost, len(grids))):
            out.append((grid_boundary(~lo, g, scan), g[:, ~lo], g))
    if len(out) == 1:
        return out[0]
    return tuple(list(x) for x in zip(*out))


def get_1d_acceptance(ring, plane, resolution, amplitude, nturns: int = 1024, refpts=None,
                      dp=None, offset=None, grid_mode=GridMode.RADIAL, use_mp=False,
                      gpu_pool=None, verbose=False, divider=2, shift_zero=1.0e-6,
                      start_method=None, mode="exact", **kwargs):
    """1-D acceptance on ceil(amplitude / resolution) points per side
    (acceptance.py:207-317); returns ([negative edge, positive edge],
    survived, tracked)."""
    if len(np.atleast_1d(plane)) != 1:
        raise ValueError("a 1-D acceptance scans one plane")
    if not (np.isscalar(resolution) and np.isscalar(amplitude)):
        raise ValueError("resolution and amplitude of a 1-D acceptance are scalars")
    npoint = np.ceil(amplitude / resolution)
    if grid_mode is not GridMode.RECURSIVE and npoint <= 1:
        raise ValueError("a grid of one point: raise the amplitude or lower the resolution")
    b, s, g = get_acceptance(ring, plane, npoint, amplitude, nturns=nturns, refpts=refpts,
                             dp=dp, offset=offset, grid_mode=grid_mode, divider=divider,
                             shift_zero=shift_zero, mode=mode)
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
