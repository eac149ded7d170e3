"""Closed orbits, one-turn matrices and linear optics, batched across rings.

The reference's optics functions call its tracking engine many times with a
handful of particles: a 6-D closed orbit is a Newton iteration of 7-particle
one-turn trackings (pyat/at/physics/orbit.py:307-368), a 4-D one at fixed
momentum 5 particles (orbit.py:16-73), a one-turn matrix 12 particles
(matrix.py:105-169), and ``linopt6`` with chromaticity repeats these on two
frequency-shifted copies of the ring (linear.py:323-611, 846-971).  On a GPU
such calls are latency-bound: a few particles cannot fill it, and each call
costs a launch and its copies.

Here every search takes a LIST of rings and advances all of them together:
each Newton step of every ring is one job of ONE batched launch
(``atb_track_batch``), so K error-seeded variants -- or the nominal and the two
frequency-shifted rings of a chromaticity measurement -- cost one launch per
step instead of K calls.  The steps themselves are the reference's (same
finite-difference steps, Newton update and convergence test), and each ring's
particles are tracked exactly as alone, so a batched result equals the
single-ring one.  The radiation energy loss that seeds the 6-D search is one
launch over all elements (``atb_element_pass``) instead of one ``elempass``
call per radiating element.

``linopt6`` returns the reference's three record arrays (elemdata0, beamdata,
elemdata): the normalising matrix A of the one-turn matrix (Forest's
eigenvector normalisation), put in standard form by rotating each mode's
column pair to zero phase, and at every observation point the Wolski mode
matrices R_k of M_s A, the betatron functions and dispersion read from them,
the phase advances, the closed orbit and M_s.
"""
from __future__ import annotations

import copy as _copy
import math

import numpy as np

from . import physics
from .engine import Engine
from .lattice import C0, compile_lattice, element_length
from .radiation import a_matrix, mode_matrices
from .tracking import _energy_particle, gpupass

__all__ = ["energy_loss", "element_exits", "find_orbit6_batch", "find_orbit4_batch",
           "find_m66", "find_m66_batch", "disable_6d", "slip_factor", "linopt6",
           "get_tune", "chromaticity"]

XYSTEP = physics.XYSTEP
DPSTEP = physics.DPSTEP

#: linopt6's per-point record (the reference's field names and shapes)
OPTICS6_DTYPE = [("alpha", np.float64, (2,)), ("beta", np.float64, (2,)),
                 ("mu", np.float64, (3,)), ("R", np.float64, (3, 6, 6)),
                 ("A", np.float64, (6, 6)), ("dispersion", np.float64, (4,)),
                 ("closed_orbit", np.float64, (6,)), ("M", np.float64, (6, 6)),
                 ("s_pos", np.float64)]
BEAM6_DTYPE = [("tune", np.float64, (3,)), ("chromaticity", np.float64, (3,)),
               ("damping_time", np.float64, (3,))]


def _compiled(ring):
    e, rest, charge = _energy_particle(ring, None, None)
    return compile_lattice(ring, e, rest, charge)


class _Rings:
    """Rings compiled and uploaded once; ``one_turn`` tracks each ring's own
    particles for one turn, all rings in one batched launch (exact
    arithmetic)."""

    def __init__(self, rings, device: int = 0):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.eng = Engine.get(device)
        self.lids = [self.eng.upload(_compiled(r)) for r in rings]
        self.stream = torch.cuda.Stream(self.dev)
        self.launches = 0

    def one_turn(self, which: list[int], parts: list[np.ndarray]) -> list[np.ndarray]:
        """Track parts[j] ((6, n_j)) of ring which[j] for one turn."""
        torch = self.torch
        sizes = [p.shape[1] for p in parts]
        offs = np.concatenate(([0], np.cumsum(sizes)))
        host = np.concatenate([np.asarray(p, dtype=np.float64).T for p in parts], axis=0)
        buf = torch.from_numpy(np.ascontiguousarray(host)).to(self.dev)
        base = buf.data_ptr()
        jobs = [{"lattice_id": self.lids[k], "nturns": 1, "r": base + 48 * int(o), "np": int(n)}
                for k, o, n in zip(which, offs[:-1], sizes)]
        with torch.cuda.stream(self.stream):
            self.eng.track_batch(jobs, "exact", stream=self.stream.cuda_stream)
        self.stream.synchronize()
        self.eng.sync(self.stream.cuda_stream)
        self.launches += 1
        out = buf.cpu().numpy()
        return [np.asfortranarray(out[a:b].T) for a, b in zip(offs[:-1], offs[1:])]

    def close(self):
        for lid in self.lids:
            self.eng.free(lid)
        self.lids = []


# -- single elements -----------------------------------------------------------------

def element_exits(ring, r_in: np.ndarray, device: int = 0) -> np.ndarray:
    """Every element alone on its own particle: row i of the (nelem, 6)
    ``r_in`` enters element i; returns the exit coordinates (nelem, 6),
    from one launch (the exact arithmetic, turn 0)."""
    import torch

    cl = _compiled(ring)
    rin = np.ascontiguousarray(np.asarray(r_in, dtype=np.float64).reshape(cl.nelem, 6))
    eng = Engine.get(device)
    lid = eng.upload(cl)
    dev = torch.device("cuda", device)
    try:
        a = torch.from_numpy(rin).to(dev)
        b = torch.empty_like(a)
        st = torch.cuda.Stream(dev)
        st.wait_stream(torch.cuda.current_stream(dev))
        eng.element_pass(lid, a.data_ptr(), b.data_ptr(), None, st.cuda_stream)
        st.synchronize()
        eng.sync(st.cuda_stream)
        return b.cpu().numpy()
    finally:
        eng.free(lid)


def energy_loss(ring, device: int = 0) -> float:
    """Energy lost per turn [eV], the reference's TRACKING method
    (pyat/at/physics/energy_loss.py:80-89): each radiating element entered
    at zero alone, the momentum changes summed in element order."""
    rad = [i for i, e in enumerate(ring) if str(getattr(e, "PassMethod", "")).endswith("RadPass")]
    if not rad:
        return 0.0
    out = element_exits(ring, np.zeros((len(ring), 6)), device)
    delta = 0.0
    for i in rad:
        delta += out[i, 4]
    return -delta * float(ring.energy)


def _ct_guess(ring, device: int = 0) -> float:
    """physics._ct_guess with the energy loss from one launch."""
    return physics._ct_guess(ring, None, u0=energy_loss(ring, device))


# -- closed orbits -------------------------------------------------------------------

def find_orbit6_batch(rings, guesses=None, convergence: float = physics.ORB_CONVERGENCE,
                      max_iterations: int = physics.ORB_MAXITER, xy_step: float = XYSTEP,
                      dp_step: float = DPSTEP, device: int = 0, stats: dict | None = None):
    """6-D closed orbits of several rings (the reference's find_orbit6 of each,
    orbit.py:307-368): per Newton step, every unconverged ring's 7 particles
    (the point and its forward-difference neighbours) are one job of one
    batched one-turn launch."""
    rings = list(rings)
    n = len(rings)
    if guesses is None:
        xs = []
        for r in rings:
            x = np.zeros(6)
            x[5] = _ct_guess(r, device)
            xs.append(x)
    else:
        xs = [np.asarray(g, dtype=np.float64).copy() for g in guesses]
    thetas = [physics._rf_theta(r) for r in rings]
    scaling = np.array([xy_step] * 4 + [dp_step] * 2)
    delta = np.concatenate((np.diag(scaling), np.zeros((6, 1))), axis=1)
    ident = np.identity(6)
    active = list(range(n))
    batch = _Rings(rings, device)
    try:
        for _ in range(max_iterations):
            if not active:
                break
            outs = batch.one_turn(active, [xs[k].reshape(6, 1) + delta for k in active])
            still = []
            for k, r in zip(active, outs):
                if not np.all(np.isfinite(r)):
                    raise RuntimeError("find_orbit6: particles lost while searching the orbit "
                                       "of ring %d" % k)
                j6 = (r[:, :6] - r[:, 6:]) / scaling
                step = np.linalg.solve(j6 - ident, r[:, 6] - xs[k] - thetas[k])
                x_next = xs[k] - step
                change = np.linalg.norm(x_next - xs[k])
                xs[k] = x_next
                if change > convergence:
                    still.append(k)
            active = still
    finally:
        if stats is not None:
            stats["launches"] = batch.launches
        batch.close()
    return xs


def find_orbit4_batch(rings, dps, guesses=None, convergence: float = physics.ORB_CONVERGENCE,
                      max_iterations: int = physics.ORB_MAXITER, xy_step: float = XYSTEP,
                      device: int = 0):
    """4-D closed orbits at fixed momentum deviations ``dps`` (one per ring;
    the reference's _orbit_dp, orbit.py:16-73): Newton on (x, px, y, py)
    with forward differences, each step of every ring one job of one
    batched launch.  The rings must not radiate or accelerate."""
    rings = list(rings)
    xs = []
    for k in range(len(rings)):
        x = np.zeros(6) if guesses is None else np.asarray(guesses[k], dtype=np.float64).copy()
        x[4] = 0.0 if dps[k] is None else float(dps[k])
        xs.append(x)
    delta = np.zeros((6, 5), order="F")
    for i in range(4):
        delta[i, i] = xy_step
    scaling = np.full(4, xy_step)
    ident = np.identity(4)
    active = list(range(len(rings)))
    batch = _Rings(rings, device)
    try:
        for _ in range(max_iterations):
            if not active:
                break
            outs = batch.one_turn(active, [xs[k].reshape(6, 1) + delta for k in active])
            still = []
            for k, r in zip(active, outs):
                j4 = (r[:4, :4] - r[:4, 4:]) / scaling
                step = np.linalg.solve(j4 - ident, r[:4, 4] - xs[k][:4])
                x_next = xs[k] - np.append(step, np.zeros(2))
                change = np.linalg.norm(x_next - xs[k])
                xs[k] = x_next
                if change > convergence:
                    still.append(k)
            active = still
    finally:
        batch.close()
    return xs


# -- one-turn matrices ---------------------------------------------------------------

def _cd_particles(orbit, xy_step, dp_step):
    steps = np.array([xy_step] * 4 + [dp_step] * 2)
    half = 0.5 * np.diag(steps)
    return np.asfortranarray(np.asarray(orbit, dtype=np.float64).reshape(6, 1) +
                             np.concatenate((half, -half), axis=1)), steps


def find_m66(ring, refpts=None, orbit=None, xy_step: float = XYSTEP, dp_step: float = DPSTEP,
             device: int = 0):
    """One-turn matrix and the matrices from the ring entrance to each of
    ``refpts`` (the reference's find_m66, matrix.py:105-169): central
    differences of 12 particles around the orbit, tracked once with refpts
    snapshots.  Returns (m66, ms (nrefs, 6, 6))."""
    if orbit is None:
        orbit = find_orbit6_batch([ring], device=device)[0]
    r, steps = _cd_particles(orbit, xy_step, dp_step)
    refs = None if refpts is None else np.asarray(refpts, dtype=np.uint32).reshape(-1)
    if refs is not None and refs.size:
        rout = gpupass(ring, r, 1, refpts=refs, mode="exact", gpu_pool=[device])
        snaps = np.moveaxis(rout[:, :, :, 0], 2, 0)          # (nrefs, 6, 12)
        ms = (snaps[:, :, :6] - snaps[:, :, 6:]) / steps
    else:
        gpupass(ring, r, 1, mode="exact", gpu_pool=[device])
        ms = np.empty((0, 6, 6))
    return (r[:, :6] - r[:, 6:]) / steps, ms


def find_m66_batch(rings, orbits, xy_step: float = XYSTEP, dp_step: float = DPSTEP,
                   device: int = 0) -> list[np.ndarray]:
    """One-turn matrices of several rings around their orbits, all 12 x K
    particles in one batched launch."""
    batch = _Rings(rings, device)
    try:
        parts = [_cd_particles(o, xy_step, dp_step)[0] for o in orbits]
        outs = batch.one_turn(list(range(len(parts))), parts)
    finally:
        batch.close()
    steps = np.array([xy_step] * 4 + [dp_step] * 2)
    return [(r[:, :6] - r[:, 6:]) / steps for r in outs]


# -- frequency, slip factor, tunes, chromaticity ------------------------------------

_RAD_TO_PLAIN = {"StrMPoleSymplectic4RadPass": "StrMPoleSymplectic4Pass",
                 "BndMPoleSymplectic4RadPass": "BndMPoleSymplectic4Pass"}


def _relist(ring, elems):
    out = _copy.copy(ring)
    out[:] = elems
    return out


def disable_6d(ring):
    """A copy of the ring without longitudinal motion (the reference's
    Lattice.disable_6d defaults): radiating magnets get their plain pass
    methods, cavities become identities (drifts when they have a length),
    quantum-diffusion elements identities.  Changed elements are copies; the
    others are shared.  The reference decides by element class; here the
    pass method decides, so generic elements are switched too."""
    elems = []
    for e in ring:
        pm = str(getattr(e, "PassMethod", ""))
        new = _RAD_TO_PLAIN.get(pm)
        if pm == "RFCavityPass":
            new = "DriftPass" if element_length(e) != 0.0 else "IdentityPass"
        elif pm == "QuantDiffPass":
            new = "IdentityPass"
        if new is None:
            elems.append(e)
        else:
            c = _copy.copy(e)
            c.PassMethod = new
            elems.append(c)
    return _relist(ring, elems)


def _cavities(ring):
    return [i for i, e in enumerate(ring) if getattr(e, "PassMethod", None) == "RFCavityPass"]


def _with_frequency_scale(ring, factor: float):
    """A copy whose cavities run at Frequency * factor."""
    elems = list(ring)
    for i in _cavities(ring):
        c = _copy.copy(elems[i])
        c.Frequency = float(c.Frequency) * factor
        elems[i] = c
    return _relist(ring, elems)


def _gamma(ring) -> float:
    e, rest, _ = _energy_particle(ring, None, None)
    return e / rest if rest > 0 else math.inf


def _s_pos(ring) -> np.ndarray:
    """Longitudinal position of every element entrance and of the end."""
    return np.concatenate(([0.0], np.cumsum([element_length(e) for e in ring])))


def slip_factor(ring, dp_step: float = DPSTEP, device: int = 0) -> float:
    """eta = 1/gamma^2 - alpha_c of a ring without longitudinal motion, with
    the momentum compaction alpha_c the slope of the one-turn path
    lengthening over momentum between the 4-D orbits at -dp_step/2 and
    +dp_step/2 (the reference's get_mcf / get_slip_factor,
    pyat/at/physics/revolution.py:15-80)."""
    dps = np.linspace(-dp_step / 2, dp_step / 2, 2)
    orbs = find_orbit4_batch([ring, ring], list(dps), device=device)
    batch = _Rings([ring], device)
    try:
        out = batch.one_turn([0], [np.stack(orbs, axis=1)])[0]
    finally:
        batch.close()
    fit = np.polynomial.Polynomial.fit(out[4], out[5], deg=1).convert().coef
    return 1.0 / _gamma(ring) ** 2 - fit[1] / _s_pos(ring)[-1]


def _tunes_of(m66: np.ndarray) -> np.ndarray:
    _, lam = a_matrix(m66)
    return np.mod(np.angle(lam) / 2.0 / np.pi, 1.0)


def get_tune(ring, orbit=None, device: int = 0) -> np.ndarray:
    """The three tunes of a 6-D ring from its one-turn matrix."""
    return _tunes_of(find_m66(ring, orbit=orbit, device=device)[0])


def chromaticity(ring, orbit=None, dp_step: float = DPSTEP, device: int = 0,
                 stats: dict | None = None) -> np.ndarray:
    """Chromaticities of a 6-D ring as the reference's linopt6 measures them
    (linear.py:519-534, 590-596): the RF frequency moved by -/+ dp_step * eta / 2,
    the closed orbits and tunes of both copies, dQ / d(delta).  Both orbit
    searches run as one batch, then both one-turn matrices in one launch."""
    if orbit is None:
        orbit = find_orbit6_batch([ring], device=device)[0]
    dff = dp_step * slip_factor(disable_6d(ring), dp_step, device)
    up = _with_frequency_scale(ring, 1.0 + 0.5 * dff)
    dn = _with_frequency_scale(ring, 1.0 - 0.5 * dff)
    o_up, o_dn = find_orbit6_batch([up, dn], guesses=[orbit, orbit], device=device, stats=stats)
    m_up, m_dn = find_m66_batch([up, dn], [o_up, o_dn], device=device)
    return (_tunes_of(m_up) - _tunes_of(m_dn)) / (o_up[4] - o_dn[4])


# -- linear optics -------------------------------------------------------------------

def _phase(a: np.ndarray, k: int) -> float:
    """Phase carried by mode k of a normalising matrix: the angle of its
    first row in the mode's own 2x2 block."""
    return math.atan2(a[2 * k, 2 * k + 1], a[2 * k, 2 * k])


def _standard(a: np.ndarray) -> np.ndarray:
    """A with each mode's column pair rotated to zero phase."""
    out = a.copy()
    for k in range(a.shape[0] // 2):
        th = -_phase(a, k)
        c, s = math.cos(th), math.sin(th)
        rot = np.array([[c, s], [-s, c]])
        out[:, 2 * k:2 * k + 2] = a[:, 2 * k:2 * k + 2] @ rot
    return out


def _point(a: np.ndarray):
    """Optics carried by a normalising matrix a at one point: (alpha, beta,
    mu, R, A, dispersion)."""
    r = mode_matrices(a)
    mu = np.array([_phase(a, k) for k in range(3)])
    beta = np.array([r[0, 0, 0], r[1, 2, 2]])
    alpha = -np.array([r[0, 1, 0], r[1, 3, 2]])
    disp = r[2, :4, 4] / r[2, 4, 4]
    return alpha, beta, mu, r, a, disp


def _unwrap_phases(mu: np.ndarray):
    """Make phase advances grow along the ring: a drop of more than 1e-3 from
    one point to the next (the first against zero) is a wrap of 2 pi."""
    prev = np.vstack((np.zeros((1, mu.shape[1])), mu))
    wraps = np.diff(prev, axis=0) < -1.0e-3
    mu += np.cumsum(wraps, axis=0) * 2.0 * np.pi


def linopt6(ring, refpts=None, orbit=None, get_chrom: bool = False, xy_step: float = XYSTEP,
            dp_step: float = DPSTEP, device: int = 0):
    """Linear optics of a 6-D ring at ``refpts`` (the reference's linopt6,
    pyat/at/physics/linear.py:846-971): returns (elemdata0, beamdata,
    elemdata) with the reference's fields -- alpha, beta, mu, R, A,
    dispersion, closed_orbit, M, s_pos per point; tune, chromaticity
    (NaN unless ``get_chrom``) and damping_time for the beam."""
    if orbit is None:
        orbit = find_orbit6_batch([ring], xy_step=xy_step, dp_step=dp_step, device=device)[0]
    orbit = np.asarray(orbit, dtype=np.float64)
    refs = np.zeros(0, dtype=np.uint32) if refpts is None else np.asarray(
        refpts, dtype=np.uint32).reshape(-1)
    mt, ms = find_m66(ring, refs, orbit, xy_step, dp_step, device)
    a0, lam = a_matrix(mt)
    astd = _standard(a0)
    el0 = _point(astd)
    pts = [_point(m @ astd) for m in ms]
    # closed orbit at the points: the orbit tracked one turn with snapshots
    if refs.size:
        r = np.asfortranarray(orbit.reshape(6, 1).copy())
        rout = gpupass(ring, r, 1, refpts=refs, mode="exact", gpu_pool=[device])
        orbs = rout[:, 0, :, 0].T
    else:
        orbs = np.zeros((0, 6))
    spos = _s_pos(ring)
    length = spos[-1]
    tunes = np.mod(np.angle(lam) / 2.0 / np.pi, 1.0)
    damping_times = length / C0 / -np.log(np.abs(lam))
    chrom = chromaticity(ring, orbit, dp_step, device) if get_chrom else np.full(3, np.nan)
    beamdata = np.array((tunes, chrom, damping_times), dtype=BEAM6_DTYPE).view(np.recarray)
    elemdata0 = np.array(el0 + (orbit, np.identity(6), 0.0),
                         dtype=OPTICS6_DTYPE).view(np.recarray)
    elemdata = np.recarray((refs.size,), dtype=OPTICS6_DTYPE)
    if refs.size:
        cols = list(zip(*pts))
        for name, val in zip(("alpha", "beta", "mu", "R", "A", "dispersion"), cols):
            elemdata[name] = np.array(val)
        elemdata["closed_orbit"] = orbs
        elemdata["M"] = ms
        elemdata["s_pos"] = spos[refs]
        _unwrap_phases(elemdata.mu)
    return elemdata0, beamdata, elemdata
