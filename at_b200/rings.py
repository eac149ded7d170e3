"""Seeded synthetic workloads (lattices and particle distributions).

``fodo_ring``     the 32-cell FODO ring, radiation off, 3 GeV electrons
                  (385 elements; 10,000 particles x 1000 turns is the plain
                  tracking workload).
``large_ring``    the radiating large ring: 32 cells of 7 combined-function
                  dipoles, 10 quadrupoles, 6 sextupoles, 2 octupoles, an
                  aperture per cell and 2 RF cavities, with seeded T1/T2 and
                  R1/R2 misalignments on every magnet.
``gaussian``      a seeded 6-D Gaussian bunch, Fortran-ordered (6, N).

No public dataset or lattice file is involved; every number is generated
here from fixed seeds.
"""
from __future__ import annotations

import math

import numpy as np

from . import elements as E
from .lattice import C0

FODO_SIGMA = (1e-4, 1e-5, 1e-5, 1e-6, 1e-3, 1e-3)


def gaussian(n: int, sigma=FODO_SIGMA, seed: int = 0, centre=None) -> np.ndarray:
    """``default_rng(seed).standard_normal((6, n)) * sigma`` (+ centre), F-order."""
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((6, n)) * np.asarray(sigma, dtype=np.float64)[:, None]
    if centre is not None:
        r += np.asarray(centre, dtype=np.float64)[:, None]
    return np.asfortranarray(r)


def fodo_ring(energy: float = 3e9, harmonic: int = 320, voltage: float = 3e6,
              ncells: int = 32, copy_cells: bool = True) -> E.Lattice:
    """32 x [QF, D0.3, SF, D0.3, B, D0.7, QD, D0.3, SD, D0.3, B, D0.7] + RF.

    QF/QD: StrMPoleSymplectic4Pass, L=0.5 m, PolynomB[1]=+/-1.0 m^-2,
    NumIntSteps=10; SF/SD: L=0.2 m, PolynomB[2]=+15/-25 m^-3; B:
    BndMPoleSymplectic4Pass, L=1.0 m, angle 2pi/64, entrance/exit pi/64.
    Cell length 6 m, circumference 192 m; one RFCavityPass (3 MV, h=320,
    TimeLag 0) at the end, frequency h*c/C."""
    cells = []
    for _ in range(ncells if copy_cells else 1):
        cells.append([
            E.Quadrupole("QF", 0.5, 1.0),
            E.Drift("D1", 0.3),
            E.Sextupole("SF", 0.2, 15.0),
            E.Drift("D2", 0.3),
            E.Dipole("B", 1.0, 2 * math.pi / 64, EntranceAngle=math.pi / 64,
                     ExitAngle=math.pi / 64),
            E.Drift("D3", 0.7),
            E.Quadrupole("QD", 0.5, -1.0),
            E.Drift("D4", 0.3),
            E.Sextupole("SD", 0.2, -25.0),
            E.Drift("D5", 0.3),
            E.Dipole("B", 1.0, 2 * math.pi / 64, EntranceAngle=math.pi / 64,
                     ExitAngle=math.pi / 64),
            E.Drift("D6", 0.7),
        ])
    if not copy_cells:
        cells = cells * ncells
    elems = [e for c in cells for e in c]
    circ = sum(e.Length for e in elems)
    freq = harmonic * C0 / circ
    elems.append(E.RFCavity("RF", 0.0, voltage, freq, harmonic, energy))
    return E.Lattice(elems, energy=energy, particle="electron", name="fodo32")


def radiating(line: E.Lattice) -> E.Lattice:
    """The same ring with the classical-radiation pass methods."""
    out = []
    for e in line:
        c = e.copy()
        if c.PassMethod == "StrMPoleSymplectic4Pass":
            c.PassMethod = "StrMPoleSymplectic4RadPass"
        elif c.PassMethod == "BndMPoleSymplectic4Pass":
            c.PassMethod = "BndMPoleSymplectic4RadPass"
        out.append(c)
    return E.Lattice(out, energy=line.energy, particle=line.particle, name=line.name + "_rad")


# ---------------------------------------------------------------------------
# large radiating ring
# ---------------------------------------------------------------------------
#: design constants of the large ring (chosen for this workload):
#: 3 GeV electrons; a 17.5 m cell of 10 half-periods alternating QF/QD
#: (L=0.4 m, K=+1.50/-2.05 m^-2), 7 of them with a 0.6 m combined-function
#: dipole of angle 2pi/224 (edge angles half that) whose gradient is drawn from
#: U[-0.5, 0.5] m^-2 (default_rng(seed), the same 7 values in every cell);
#: SF/SD sextupoles (L=0.2 m, K2=+26.65/-86.58 m^-3, which set the chromaticity
#: to about +1 in both planes) next to the quads of 6 half-periods and
#: octupoles (L=0.2 m, K3=100 m^-4) in 2; one aperture per cell; two RF
#: cavities (1 MV each, h=658).  Periodic tunes of the unperturbed cell:
#: 0.770 / 0.194 (ring 24.65 / 6.22), beta functions below 10.4 m.
LARGE_ENERGY = 3e9
LARGE_KF, LARGE_KD = 1.50, -2.05
LARGE_KSF, LARGE_KSD = 26.64966836, -86.57975448
LARGE_KOCT = 100.0
LARGE_DIPOLE_L = 0.6
LARGE_HARMONIC = 658
LARGE_VOLTAGE = 1.0e6
LARGE_SIGMA_T = 30e-6
LARGE_SIGMA_TILT = 100e-6
LARGE_APERTURE = (-0.02, 0.02, -0.01, 0.01)


def _rot(theta: float) -> np.ndarray:
    c, s = math.cos(theta), math.sin(theta)
    r = np.eye(6)
    r[0, 0] = r[1, 1] = r[2, 2] = r[3, 3] = c
    r[0, 2] = r[1, 3] = s
    r[2, 0] = r[3, 1] = -s
    return r


def large_ring(seed: int = 1, ncells: int = 32, misalign: bool = True,
               radiation: bool = True, design_seed: int | None = None) -> E.Lattice:
    """The radiating large ring: 32 cells x 61 elements + 2 RF = 1954 elements.

    The 7 dipole gradients are the first draws of ``default_rng(seed)``
    (of ``default_rng(design_seed)`` when given: error-seeded copies keep the
    design of seed 1 and redraw only the errors).  Each magnet gets
    T1 = -(dx, 0, dy, 0, 0, 0), T2 = -T1 and R1/R2 = x-y rotations by +/-theta
    with dx, dy ~ N(0, 30 um) and theta ~ N(0, 100 urad), drawn from
    ``default_rng(seed)`` after those 7 draws."""
    rng = np.random.default_rng(seed)
    kdip = rng.uniform(-0.5, 0.5, 7)
    if design_seed is not None:
        kdip = np.random.default_rng(design_seed).uniform(-0.5, 0.5, 7)
    angle = 2 * math.pi / (ncells * 7)
    spm = "StrMPoleSymplectic4RadPass" if radiation else "StrMPoleSymplectic4Pass"
    bpm = "BndMPoleSymplectic4RadPass" if radiation else "BndMPoleSymplectic4Pass"
    has_b = [1, 1, 1, 0, 1, 1, 1, 0, 1, 0]
    elems = []
    magnets = []
    for icell in range(ncells):
        ib = 0
        for h in range(10):
            f = (h % 2 == 0)
            q = E.Quadrupole("QF" if f else "QD", 0.4, LARGE_KF if f else LARGE_KD,
                             PassMethod=spm)
            elems.append(q)
            magnets.append(q)
            elems.append(E.Drift("D", 0.15))
            if h in (0, 1, 2, 4, 5, 6):
                s = E.Sextupole("SF" if f else "SD", 0.2, LARGE_KSF if f else LARGE_KSD,
                                PassMethod=spm)
                elems.append(s)
                magnets.append(s)
            elif h in (3, 8):
                o = E.Octupole("OC", 0.2, [], [0.0, 0.0, 0.0, LARGE_KOCT], PassMethod=spm)
                elems.append(o)
                magnets.append(o)
            else:
                elems.append(E.Drift("D", 0.2))
            elems.append(E.Drift("D", 0.15))
            if has_b[h]:
                b = E.Dipole("B", LARGE_DIPOLE_L, angle, float(kdip[ib]), EntranceAngle=angle / 2,
                             ExitAngle=angle / 2, PassMethod=bpm)
                elems.append(b)
                magnets.append(b)
                ib += 1
            else:
                elems.append(E.Drift("D", LARGE_DIPOLE_L))
            elems.append(E.Drift("D", 0.25))
        elems.append(E.Aperture("AP", list(LARGE_APERTURE)))
    if misalign:
        for m in magnets:
            dx, dy, th = rng.normal(0.0, [LARGE_SIGMA_T, LARGE_SIGMA_T, LARGE_SIGMA_TILT])
            m.T1 = [-dx, 0.0, -dy, 0.0, 0.0, 0.0]
            m.T2 = [dx, 0.0, dy, 0.0, 0.0, 0.0]
            m.R1 = _rot(th)
            m.R2 = _rot(-th)
    circ = sum(e.Length for e in elems)
    freq = LARGE_HARMONIC * C0 / circ
    cell_len = len(elems) // ncells
    out = []
    for i, e in enumerate(elems):
        out.append(e)
        if i in (0, (ncells // 2) * cell_len):
            out.append(E.RFCavity("RF", 0.0, LARGE_VOLTAGE, freq, LARGE_HARMONIC, LARGE_ENERGY))
    return E.Lattice(out, energy=LARGE_ENERGY, particle="electron", name="large_ring")


LARGE_SIGMA = (1e-4, 1e-5, 1e-5, 1e-6, 1e-3, 1e-3)

#: 6-D closed orbit of ``large_ring()`` (seed 1) at its entrance as the
#: reference's find_orbit6 defines it (M(x) = x + theta, theta the RF
#: path-length slip), found by Newton iteration on the one-turn map.
LARGE_ORBIT = (-0.0005151025164660066, -3.068590557039712e-05, -0.0009101295900902443,
               0.00032698077877960427, 2.839234239542605e-05, -0.022852877509548702)


def large_ring_bunch(n: int, seed: int = 0) -> np.ndarray:
    """The large-ring bunch: a 6-D Gaussian (sigma = 100 um, 10 urad, 10 um,
    1 urad, 1e-3, 1 mm) around the closed orbit, Fortran-ordered (6, n)."""
    return gaussian(n, LARGE_SIGMA, seed=seed, centre=LARGE_ORBIT)


# ---------------------------------------------------------------------------
# batched variants of the large ring (dynamic-aperture scans)
# ---------------------------------------------------------------------------
def large_ring_variant(seed: int, strength_rel: float = 1e-3) -> E.Lattice:
    """An error-seeded copy of the large ring: the design of seed 1 (its
    dipole gradients), misalignments drawn from ``default_rng(seed)`` as in
    ``large_ring``, and 0.1 % Gaussian errors on every magnet's main strength
    (dipole and quadrupole gradients, sextupole and octupole coefficients)
    from ``default_rng(seed + 100000)``."""
    ring = large_ring(seed=seed, design_seed=1)
    rng = np.random.default_rng(seed + 100_000)
    for e in ring:
        if e.PassMethod in ("StrMPoleSymplectic4RadPass", "BndMPoleSymplectic4RadPass",
                            "StrMPoleSymplectic4Pass", "BndMPoleSymplectic4Pass"):
            b = np.array(e.PolynomB, dtype=np.float64)
            k = int(np.flatnonzero(b)[-1]) if np.any(b) else 1
            b[k] *= 1.0 + strength_rel * rng.standard_normal()
            e.PolynomB = b
    return ring


def da_grid(n: int, seed: int, xmax: float = 4e-3, ymax: float = 2e-3,
            deltas=(-0.03, 0.0, 0.03), centre=LARGE_ORBIT) -> np.ndarray:
    """``n`` particles on an x-y dynamic-aperture grid around ``centre``, split
    over the momentum offsets ``deltas`` (Fortran-ordered (6, n)).  The grid
    for each delta has ceil(n/len(deltas)) points, row-major over x in
    [-xmax, xmax] and y in (0, ymax]; ``seed`` jitters it by a tenth of a step
    so variants do not share identical start points."""
    rng = np.random.default_rng(seed)
    per = -(-n // len(deltas))
    ny = max(1, int(round(np.sqrt(per / 2.0))))
    nx = -(-per // ny)
    xs = np.linspace(-xmax, xmax, nx)
    ys = np.linspace(ymax / ny, ymax, ny)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel()])[:, :per]
    out = np.zeros((6, n))
    c = np.asarray(centre, dtype=np.float64)
    k = 0
    for d in deltas:
        m = min(per, n - k)
        jit = 0.1 * rng.standard_normal((2, m)) * np.array([[2 * xmax / max(nx - 1, 1)],
                                                            [ymax / ny]])
        out[:, k:k + m] = c[:, None]
        out[0, k:k + m] += pts[0, :m] + jit[0]
        out[2, k:k + m] += pts[1, :m] + jit[1]
        out[4, k:k + m] += d
        k += m
    return np.asfortranarray(out)


def batch_workload(nvariants: int = 256, first_seed: int = 2, turn_scale: float = 1.0,
                   seed: int = 0):
    """The batched-variant workload: for variant i (lattice seed first_seed+i)
    N_i = round(exp(U[ln 1024, ln 16384])) particles on a DA grid and
    T_i ~ U{500..5000} turns (times ``turn_scale``, at least 1), all drawn from
    ``default_rng(seed)``.  Returns a list of (seed, N_i, T_i)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nvariants):
        n = int(round(np.exp(rng.uniform(np.log(1024), np.log(16384)))))
        t = int(rng.integers(500, 5001))
        out.append((first_seed + i, n, max(1, int(round(t * turn_scale)))))
    return out


def fodo_variant(seed: int, strength_rel: float = 1e-3) -> E.Lattice:
    """The FODO ring with 0.1 % Gaussian errors (``default_rng(seed)``) on every
    quadrupole and sextupole strength; each magnet is its own object."""
    ring = fodo_ring()
    rng = np.random.default_rng(seed)
    for e in ring:
        if e.PassMethod == "StrMPoleSymplectic4Pass":
            b = np.array(e.PolynomB, dtype=np.float64)
            k = int(np.flatnonzero(b)[-1])
            b[k] *= 1.0 + strength_rel * rng.standard_normal()
            e.PolynomB = b
    return ring


def serving_pool(nfodo: int = 8, nlarge: int = 8):
    """The 16 lattices of the serving workload: FODO and large-ring copies
    with different error seeds.  Returns ({name: lattice}, {name: orbit})."""
    lats, orbits = {}, {}
    for s in range(nfodo):
        lats["fodo%d" % s] = fodo_variant(1000 + s)
        orbits["fodo%d" % s] = np.zeros(6)
    for s in range(nlarge):
        lats["large%d" % s] = large_ring_variant(2000 + s)
        orbits["large%d" % s] = np.asarray(LARGE_ORBIT)
    return lats, orbits
