"""Ohmi's equilibrium beam envelope on the GPU engine.

The reference (pyat/at/physics/radiation.py:76-148 ``_dmatr`` and :151-276
``ohmi_envelope``) walks the ring element by element in Python: it tracks the
closed orbit to every element entrance, then asks each element for its
transfer matrix (``find_elem_m66``: 12 tracked particles, central
differences) and its diffusion matrix (pyat/at.c:755-831 ``diffusion_matrix``:
the bdiff branch of the radiating multipole passes), and accumulates
B_cum <- M B_cum M^T + B.  Here one kernel launch (``atb_element_maps``)
computes every element's exact transfer matrix (forward-mode derivatives of
the integrator) and its diffusion matrix at once, one thread per element; the
6x6 accumulation, the Lyapunov/Sylvester solve for the envelope
R = M R M^T + B_cum and the normal-mode analysis run on the host.

The normal-mode analysis (``a_matrix``, ``get_tunes_damp``) restates the
reference's pyat/at/physics/amat.py:41-247 (Forest's eigenvector
normalisation with the swapped longitudinal plane; Wolski's mode matrices).
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import block_diag, eig, inv, solve, solve_sylvester

from .engine import Engine
from .lattice import compile_lattice, diffusion_constant
from .tracking import _energy_particle, gpupass

ENVELOPE_DTYPE = [
    ("r66", np.float64, (6, 6)),
    ("r44", np.float64, (4, 4)),
    ("m66", np.float64, (6, 6)),
    ("orbit6", np.float64, (6,)),
    ("emitXY", np.float64, (2,)),
    ("emitXYZ", np.float64, (3,)),
]

_J2 = np.array([[0.0, 1.0], [-1.0, 0.0]])
_I2 = np.array([[-1.0j, -1.0], [1.0, 1.0j]])


def _jmat(dms: int) -> np.ndarray:
    return block_diag(*([_J2] * dms))


def _jmatswap(dms: int) -> np.ndarray:
    """The symplectic form with the longitudinal pair swapped (ct, delta)."""
    blocks = [_J2] * dms
    if dms == 3:
        blocks = [_J2, _J2, _J2.T]
    return block_diag(*blocks)


# -- element maps on the GPU ---------------------------------------------------

def element_maps(ring, orbits, energy=None, particle=None, device: int = 0):
    """Transfer and diffusion matrices of every element of ``ring`` for a
    particle entering it at ``orbits[i]`` ((nelem, 6)), from one kernel
    launch.  Returns ``(m, b)``, each (nelem, 6, 6): m[i] = d out / d in of
    element i (exact derivatives), b[i] its Ohmi diffusion matrix (zero for
    non-radiating pass methods).  The diffusion constant uses gamma from the
    energy alone, as the reference's ``diffusion_matrix`` does when called
    without a particle."""
    import torch

    e, rest, charge = _energy_particle(ring, energy, particle)
    cl = compile_lattice(ring, e, rest, charge, t0=0.0)
    orbits = np.ascontiguousarray(np.asarray(orbits, dtype=np.float64).reshape(-1, 6))
    if orbits.shape[0] != cl.nelem:
        raise ValueError("orbits must be (%d, 6)" % cl.nelem)
    eng = Engine.get(device)
    lid = eng.upload(cl)
    dev = torch.device("cuda", device)
    try:
        o = torch.from_numpy(orbits).to(dev)
        m = torch.empty((cl.nelem, 6, 6), dtype=torch.float64, device=dev)
        b = torch.empty((cl.nelem, 6, 6), dtype=torch.float64, device=dev)
        # run on a stream of our own, ordered after the caller's (which may be
        # the legacy default stream, whose handle 0 the engine reads as its
        # own stream) and before the copies back
        cur = torch.cuda.current_stream(dev)
        st = torch.cuda.Stream(dev)
        st.wait_stream(cur)
        eng.element_maps(lid, o.data_ptr(), m.data_ptr(), b.data_ptr(),
                         diffusion_constant(e, 0.0), st.cuda_stream)
        cur.wait_stream(st)
        out = m.cpu().numpy(), b.cpu().numpy()
    finally:
        eng.free(lid)
    return out


# -- normal modes (pyat/at/physics/amat.py) --------------------------------------

def a_matrix(m: np.ndarray):
    """A such that M = A R A^-1 with R block-diagonal (damped) rotations, the
    blocks ordered to follow x, y, z (amat.py:41-119).  Returns (A, eigvals)
    with one eigenvalue per mode."""
    nv = m.shape[0]
    dms = nv // 2
    s = _jmatswap(dms)
    lam, vv = eig(m)
    # symplectic norm of each eigenvector: -i/2 v^H S v
    norm = -0.5j * np.einsum("ik,ij,jk->k", vv.conj(), s, vv)
    if np.any(np.abs(norm) < 1.0e-12):
        raise RuntimeError("Unstable ring")
    pairs = np.repeat(np.arange(0, nv, 2), 2)
    order = pairs + (norm.real < 0)
    vv, norm, lam = vv[:, order], norm[order], lam[order]
    vn = vv / np.sqrt(np.abs(norm))[None, :]
    # projection of each mode on the x, y, z planes, to order them
    proj = 0.5 * np.abs(np.sqrt(-1.0j * vn.conj().T @ s @ block_diag(*([_I2] * dms))))
    rows = list(range(0, nv, 2))
    chosen = []
    for plane in range(0, nv, 2):
        k = int(np.argmax(proj[rows, plane]))
        chosen.append(rows.pop(k))
    v = vn[:, chosen]
    a = np.empty((nv, nv))
    a[:, 0::2] = v.real
    a[:, 1::2] = v.imag
    return a, lam[chosen]


def mode_matrices(a: np.ndarray) -> np.ndarray:
    """Wolski's R-matrices of the normal modes (amat.py:151-177)."""
    dms = a.shape[0] // 2
    ss = _jmat(dms)
    tt = _jmatswap(dms)
    slcs = [slice(2 * k, 2 * k + 2) for k in range(dms)]
    a_s = np.concatenate([a[:, sl] @ tt[sl, sl] for sl in slcs], axis=1)
    inva = solve(a, ss.T)
    return np.stack([a_s[:, sl] @ inva[sl, :] for sl in slcs], axis=0)


def get_tunes_damp(m: np.ndarray, r: np.ndarray | None = None):
    """Tunes, damping rates, mode matrices and (with the beam matrix ``r``)
    mode emittances of the one-turn matrix ``m`` (amat.py:198-247)."""
    nv = m.shape[0]
    dms = nv // 2
    a, lam = a_matrix(m)
    tunes = np.mod(np.angle(lam) / 2.0 / np.pi, 1.0)
    damping = -np.log(np.abs(lam))
    fields = [("tunes", np.float64, (dms,)), ("damping_rates", np.float64, (dms,)),
              ("mode_matrices", np.float64, (dms, nv, nv))]
    arrays = [tunes, damping, mode_matrices(a)]
    if r is not None:
        j = _jmat(dms)
        d = np.diag(a.T @ j @ r @ j @ a)
        fields.append(("mode_emittances", np.float64, (dms,)))
        arrays.append(-0.5 * (d[0::2] + d[1::2]))
    return np.rec.fromarrays([np.array(x) for x in arrays], dtype=fields)


# -- the envelope -----------------------------------------------------------------

#: the three planes' coordinate pairs: (x, px), (y, py), (delta, ct)
_PLANES = ((0, 1), (2, 3), (4, 5))
#: a projected emittance below this is taken as zero (no equilibrium beam
#: in that plane), as the reference's envelope code does
_EMIT_FLOOR = 1.0e-13


def _plane_emittances(sigma, planes):
    """sqrt(det) of each plane's 2x2 block of a beam matrix: the projected
    emittance (a negative determinant from rounding counts as zero)."""
    out = np.empty(len(planes))
    for k, (i, j) in enumerate(planes):
        det = sigma[i, i] * sigma[j, j] - sigma[i, j] * sigma[j, i]
        out[k] = np.sqrt(max(det, 0.0))
    return out


def _conditional(sigma, keep, given):
    """Covariance of the coordinates ``keep`` when the coordinates ``given``
    are held at zero: the Schur complement S_kk - S_kg S_gg^-1 S_gk of the
    Gaussian beam matrix."""
    s_kk = sigma[np.ix_(keep, keep)]
    s_kg = sigma[np.ix_(keep, given)]
    s_gg = sigma[np.ix_(given, given)]
    return s_kk - s_kg @ solve(s_gg, s_kg.T)


def _project(r66):
    """The envelope record's projections of a 6x6 beam matrix (the
    reference's emitXYZ, emitXY and r44, radiation.py:206-225): the three
    planes' projected emittances, and the betatron beam matrix at zero
    momentum deviation, i.e. the transverse covariance conditional on
    (delta, ct) = 0.  Without a horizontal equilibrium it is undefined (NaN);
    without a vertical one (an uncoupled ring) only its horizontal block is
    filled."""
    e3 = _plane_emittances(r66, _PLANES)
    r44 = np.zeros((4, 4))
    if e3[0] < _EMIT_FLOOR:
        r44[:] = np.nan
    elif e3[1] < _EMIT_FLOOR:
        r44[:2, :2] = _conditional(r66, [0, 1], [4, 5])
    else:
        r44[:] = _conditional(r66, [0, 1, 2, 3], [4, 5])
    e2 = _plane_emittances(r44, _PLANES[:2])
    return r44, e2, e3


def envelope_from_matrices(m66: np.ndarray, bcum: np.ndarray) -> dict:
    """The equilibrium beam matrix R = M R M^T + B_cum, solved as the
    Sylvester equation inv(M) R - R (-M^T) ... (radiation.py:245-258), with
    its projections and normal modes."""
    aa = inv(m66)
    rr = solve_sylvester(aa, -m66.T, aa @ bcum)
    rr = 0.5 * (rr + rr.T)
    r44, e2, e3 = _project(rr)
    modes = get_tunes_damp(m66, rr)
    return {"r66": rr, "r44": r44, "emitXY": e2, "emitXYZ": e3, "tunes": modes.tunes,
            "damping_rates": modes.damping_rates, "mode_matrices": modes.mode_matrices,
            "mode_emittances": modes.mode_emittances}


def cumulative_diffusion(ring, orbit, device: int = 0):
    """The orbit at every element entrance and the end (n + 1, 6), the
    cumulative diffusion matrices B_cum (n + 1, 6, 6) (radiation.py:76-148,
    ``_dmatr``) and the transfer matrices from the ring entrance to every
    element entrance (n + 1, 6, 6), chained from the exact element maps."""
    orbit = np.asarray(orbit, dtype=np.float64)
    n = len(ring)
    r = np.asfortranarray(orbit.reshape(6, 1).copy())
    rout = gpupass(ring, r, 1, refpts=np.arange(n + 1, dtype=np.uint32), mode="exact")
    orbs = np.asarray(rout).reshape(6, n + 1).T.copy()
    m, b = element_maps(ring, orbs[:n], device=device)
    bcum = np.empty((n + 1, 6, 6))
    mcum = np.empty((n + 1, 6, 6))
    bcum[0] = 0.0
    mcum[0] = np.eye(6)
    for k in range(n):
        bcum[k + 1] = m[k] @ bcum[k] @ m[k].T + b[k]
        mcum[k + 1] = m[k] @ mcum[k]
    return orbs, bcum, mcum


def quantdiffmat(ring, orbit=None, device: int = 0) -> np.ndarray:
    """Diffusion matrix of the whole ring, the symmetrised B_cum at its end
    (radiation.py:469-482)."""
    from . import physics

    if orbit is None:
        orbit = physics.find_orbit6(ring, mode="exact")
    _, bcum, _ = cumulative_diffusion(ring, orbit, device)
    return 0.5 * (bcum[-1] + bcum[-1].T)


def lmat(dmat: np.ndarray) -> np.ndarray:
    """Lower-triangular L with L L^T = dmat, the factor a QuantumDiffusion
    element applies to six standard normals (the reference's Lmatp,
    radiation.py:125-146).

    A diffusion matrix is symmetric positive semi-definite, and singular in
    a ring without vertical diffusion (zero rows and columns).  L comes from
    the column-by-column Cholesky recursion with semi-definite pivoting: a
    column whose pivot is at or below eps times the largest diagonal entry
    is left at zero, which still gives L L^T = dmat.  The reference lifts
    such eigenvalues to eps * max|eigenvalue| before a plain Cholesky, so
    its factor holds entries of about sqrt(eps) of the scale in that
    subspace where this one holds zeros; on a non-singular matrix the two
    agree to rounding."""
    d = 0.5 * (np.asarray(dmat, dtype=np.float64) + np.asarray(dmat, dtype=np.float64).T)
    n = d.shape[0]
    out = np.zeros((n, n))
    floor = np.finfo(float).eps * float(np.abs(np.diag(d)).max(initial=0.0))
    for j in range(n):
        piv = d[j, j] - out[j, :j] @ out[j, :j]
        if piv <= floor:
            continue
        out[j, j] = np.sqrt(piv)
        out[j + 1:, j] = (d[j + 1:, j] - out[j + 1:, :j] @ out[j, :j]) / out[j, j]
    return out


def gen_quantdiff_elem(ring, orbit=None, device: int = 0):
    """A QuantumDiffusion element reproducing the ring's quantum excitation
    at one point (radiation.py:485-500)."""
    from .elements import QuantumDiffusion

    return QuantumDiffusion("Diffusion", np.asfortranarray(lmat(quantdiffmat(ring, orbit,
                                                                            device))))


def ohmi_envelope(ring, refpts=None, orbit=None, device: int = 0):
    """Equilibrium beam envelope of a radiating ring (the reference's
    ``ohmi_envelope``, same three returned record arrays: ``emit0`` at the
    ring entrance, ``beamdata`` (tunes, damping_rates, mode_matrices,
    mode_emittances) and ``emit`` at ``refpts``).  The closed orbit, the
    element maps and the one-turn matrix come from the GPU engine (exact
    arithmetic, exact derivatives)."""
    from . import physics

    if orbit is None:
        orbit = physics.find_orbit6(ring, mode="exact")
    orbs, bcum, mcum = cumulative_diffusion(ring, orbit, device)
    mring = mcum[-1]
    env = envelope_from_matrices(mring, bcum[-1])
    rr = env["r66"]
    emit0 = np.rec.fromarrays((rr, env["r44"], mring, orbs[0], env["emitXY"], env["emitXYZ"]),
                              dtype=ENVELOPE_DTYPE)
    beamdata = np.rec.fromarrays(
        (env["tunes"], env["damping_rates"], env["mode_matrices"], env["mode_emittances"]),
        dtype=[("tunes", np.float64, (3,)), ("damping_rates", np.float64, (3,)),
               ("mode_matrices", np.float64, (3, 6, 6)), ("mode_emittances", np.float64, (3,))])
    refs = [] if refpts is None else [int(k) for k in np.atleast_1d(refpts)]
    recs = []
    for k in refs:
        sig = mcum[k] @ rr @ mcum[k].T + bcum[k]
        r44, e2, e3 = _project(sig)
        recs.append((sig, r44, mcum[k], orbs[k], e2, e3))
    emit = (np.rec.fromrecords(recs, dtype=ENVELOPE_DTYPE) if recs
            else np.recarray((0,), dtype=ENVELOPE_DTYPE))
    return emit0, beamdata, emit
