"""Element and lattice cases shared by the golden-fixture generator and the
parity tests.

Each element case is a plain dict of reference attribute names (so the same
case builds a pyat ``Element`` in the generator and an ``at_b200`` element in
the tests); each covers one PassMethod with a set of its options.
"""
from __future__ import annotations

import math

import numpy as np

PI = math.pi


def _tilt(theta):
    c, s = math.cos(theta), math.sin(theta)
    r = np.eye(6)
    r[0, 0] = r[1, 1] = r[2, 2] = r[3, 3] = c
    r[0, 2] = r[1, 3] = s
    r[2, 0] = r[3, 1] = -s
    return r


def _dense(seed):
    rng = np.random.default_rng(seed)
    return np.eye(6) + 1e-3 * rng.standard_normal((6, 6))


MIS = dict(T1=[1e-4, 2e-5, -5e-5, 1e-5, 0.0, 0.0], T2=[-1e-4, -2e-5, 5e-5, -1e-5, 0.0, 0.0],
           R1=_tilt(2e-3), R2=_tilt(-2e-3))
MIS_DENSE = dict(T1=[3e-5, -1e-6, 2e-5, 4e-6, 1e-5, -2e-6],
                 T2=[-3e-5, 1e-6, -2e-5, -4e-6, -1e-5, 2e-6],
                 R1=_dense(11), R2=_dense(12))
FINT_M = [0.01, 0.02, 0.03, 0.004, 0.005]
FINT_P = [0.015, 0.025, 0.002, 0.003, 0.006]


def quad(name, L, k, **kw):
    d = dict(FamName=name, Length=L, PolynomA=[0.0, 0.0], PolynomB=[0.0, k], MaxOrder=1,
             NumIntSteps=10, PassMethod="StrMPoleSymplectic4Pass")
    d.update(kw)
    return d


def multipole(name, L, pa, pb, **kw):
    n = max(len(pa), len(pb))
    pa = list(pa) + [0.0] * (n - len(pa))
    pb = list(pb) + [0.0] * (n - len(pb))
    d = dict(FamName=name, Length=L, PolynomA=pa, PolynomB=pb, MaxOrder=n - 1, NumIntSteps=10,
             PassMethod="StrMPoleSymplectic4Pass")
    d.update(kw)
    return d


def bend(name, L, angle, k=0.0, e1=0.0, e2=0.0, **kw):
    d = dict(FamName=name, Length=L, BendingAngle=angle, EntranceAngle=e1, ExitAngle=e2,
             PolynomA=[0.0, 0.0], PolynomB=[0.0, k], MaxOrder=1, NumIntSteps=10,
             PassMethod="BndMPoleSymplectic4Pass")
    d.update(kw)
    return d


def element_cases():
    """(case name, attribute dict) for every option of every pass method."""
    c = []
    c.append(("drift", dict(FamName="D", Length=1.0, PassMethod="DriftPass")))
    c.append(("drift_mis", dict(FamName="D", Length=0.7, PassMethod="DriftPass", **MIS,
                                RApertures=[-4e-3, 4e-3, -3e-3, 3e-3], EApertures=[5e-3, 4e-3])))
    c.append(("drift_dense", dict(FamName="D", Length=0.5, PassMethod="DriftPass", **MIS_DENSE)))
    c.append(("identity_mis", dict(FamName="M", Length=0.0, PassMethod="IdentityPass", **MIS_DENSE,
                                   RApertures=[-2e-3, 2e-3, -2e-3, 2e-3])))
    c.append(("quad", quad("Q", 0.4, 1.0)))
    c.append(("quad_full", quad("Q", 0.5, -1.3, PolynomA=[1e-4, 2e-3], KickAngle=[2e-5, -3e-5],
                                FieldScaling=1.02, FringeQuadEntrance=1, FringeQuadExit=1,
                                **MIS, RApertures=[-5e-3, 5e-3, -4e-3, 4e-3],
                                EApertures=[6e-3, 5e-3])))
    c.append(("quad_linfringe", quad("Q", 0.3, 2.1, FringeQuadEntrance=2, FringeQuadExit=2,
                                     fringeIntM0=FINT_M, fringeIntP0=FINT_P)))
    c.append(("quad_dense", quad("Q", 0.35, 0.8, NumIntSteps=7, **MIS_DENSE)))
    c.append(("sext", multipole("S", 0.2, [0, 0, 0], [0, 0, 15.0])))
    c.append(("oct", multipole("O", 0.1, [0, 0, 0, 10.0], [1e-3, 0.1, -5.0, 120.0])))
    c.append(("mpole_o6", multipole("M", 0.25, [0, 1e-3, 0, 0, 0, 0, 2e3],
                                    [0, 0.5, 3.0, 10.0, 1e2, -1e3, 1e4], NumIntSteps=4)))
    c.append(("bend", bend("B", 1.0, 0.1, e1=0.05, e2=0.05)))
    c.append(("bend_k", bend("B", 1.2, 2 * PI / 64, k=-0.3, e1=PI / 64, e2=PI / 64)))
    for m in (0, 1, 2, 3, 7):
        c.append(("bend_fringe%d" % m, bend("B", 0.8, 0.05, k=0.2, e1=0.02, e2=0.03,
                                          FringeBendEntrance=m, FringeBendExit=m, FullGap=0.04,
                                          FringeInt1=0.5, FringeInt2=0.45)))
    c.append(("bend_full", bend("B", 0.9, 0.07, k=0.4, e1=0.03, e2=0.04, FullGap=0.03,
                                FringeInt1=0.6, FringeInt2=0.6, FieldScaling=0.98,
                                KickAngle=[1e-5, 2e-5], FringeQuadEntrance=1,
                                FringeQuadExit=1, **MIS, RApertures=[-5e-3, 5e-3, -4e-3, 4e-3])))
    c.append(("bend_sext", bend("B", 0.6, 0.04, e1=0.01, e2=0.01, MaxOrder=2,
                                PolynomA=[0.0, 0.0, 0.0], PolynomB=[0.0, 0.3, 4.0])))
    c.append(("bend_linfringe", bend("B", 0.7, 0.05, k=1.1, FringeQuadEntrance=2,
                                     FringeQuadExit=2, fringeIntM0=FINT_M, fringeIntP0=FINT_P)))
    c.append(("thin", dict(FamName="T", Length=0.0, PassMethod="ThinMPolePass",
                           PolynomA=[1e-5, 2e-3, 5.0], PolynomB=[2e-5, 0.1, 20.0], MaxOrder=2)))
    c.append(("thin_full", dict(FamName="T", Length=0.0, PassMethod="ThinMPolePass",
                                PolynomA=[0.0, 0.0, 0.0], PolynomB=[0.0, 0.2, 10.0], MaxOrder=2,
                                BendingAngle=[[1e-3, -5e-4]], KickAngle=[1e-5, -2e-5],
                                FieldScaling=1.01, **MIS,
                                RApertures=[-5e-3, 5e-3, -4e-3, 4e-3])))
    c.append(("thin_ba1d", dict(FamName="T", Length=0.0, PassMethod="ThinMPolePass",
                                PolynomA=[0.0, 0.0], PolynomB=[0.0, 0.2], MaxOrder=1,
                                BendingAngle=[1e-3, -5e-4])))
    c.append(("corr_thin", dict(FamName="C", Length=0.0, PassMethod="CorrectorPass",
                                KickAngle=[0.9e-4, 0.5e-4])))
    c.append(("corr_thick", dict(FamName="C", Length=0.3, PassMethod="CorrectorPass",
                                 KickAngle=[2e-4, -1e-4], FieldScaling=1.01, **MIS,
                                 EApertures=[6e-3, 5e-3])))
    c.append(("aperture", dict(FamName="A", Length=0.0, PassMethod="AperturePass",
                               Limits=[-1.5e-3, 1.5e-3, -1e-3, 1e-3])))
    c.append(("rf_thin", dict(FamName="RF", Length=0.0, PassMethod="RFCavityPass",
                              Voltage=3e6, Frequency=352.2e6, HarmNumber=992, Energy=6e9,
                              TimeLag=0.01, PhaseLag=0.1)))
    c.append(("rf_thick", dict(FamName="RF", Length=0.5, PassMethod="RFCavityPass",
                               Voltage=2e6, Frequency=499.6e6, HarmNumber=320, Energy=6e9,
                               TimeLag=0.0)))
    rad = []
    for name, d in c:
        if d["PassMethod"] in ("StrMPoleSymplectic4Pass", "BndMPoleSymplectic4Pass"):
            dd = dict(d)
            dd["PassMethod"] = d["PassMethod"].replace("4Pass", "4RadPass")
            rad.append((name + "_rad", dd))
    return c + rad


def make_element(d, cls):
    """Build ``cls(FamName)`` with the case's attributes; lists become
    Fortran-ordered float64 arrays (R1/R2 as 6x6)."""
    el = cls(d.get("FamName", "E"))
    for k, v in d.items():
        if k == "FamName":
            continue
        if isinstance(v, (list, tuple, np.ndarray)):
            a = np.asarray(v, dtype=np.float64)
            if k in ("R1", "R2"):
                a = a.reshape(6, 6)
            v = np.asfortranarray(a)
        object.__setattr__(el, k, v)
    return el


def element_particles(n: int = 48, seed: int = 7, scale: float = 1.0) -> np.ndarray:
    """Seeded particles at a few millimetres / milliradians (plus a few large
    ones that trip apertures)."""
    rng = np.random.default_rng(seed)
    sig = np.array([2e-3, 2e-4, 1.5e-3, 1.5e-4, 5e-3, 3e-3]) * scale
    r = rng.standard_normal((6, n)) * sig[:, None]
    r[:, 0] = 0.0
    r[0, 1] = 1e-6
    return np.asfortranarray(r)


def kitchen_sink():
    """A short lattice with every pass method, for multi-turn engine cases."""
    names = ["quad_full", "drift_mis", "sext", "bend_full", "corr_thick", "thin_full",
             "oct", "bend_fringe2", "quad_linfringe", "drift", "aperture", "bend_fringe3",
             "identity_mis", "quad", "corr_thin", "rf_thick", "mpole_o6", "drift"]
    table = dict(element_cases())
    out = []
    for n in names:
        d = dict(table[n])
        for k in ("RApertures", "EApertures"):
            if k in d:
                d[k] = [5 * v for v in d[k]]
        if d["PassMethod"] == "AperturePass":
            d["Limits"] = [-2e-2, 2e-2, -1e-2, 1e-2]
        out.append(d)
    return out
