"""Minimal element classes with pyat's attribute names and defaults.

The tracking entry points read elements by attribute, so pyat's own
``at.lattice.elements`` objects work unchanged.  These light classes exist so
the package (and its tests and benchmark) can build lattices where pyat is not
installed.  Constructors follow ``pyat/at/lattice/elements/basic_elements.py``
and ``magnet_elements.py``: the same positional arguments, the same default
PassMethod, ``NumIntSteps=10`` for thick multipoles
(``magnet_elements.py:411``), ``MaxOrder`` inferred from the longest of
PolynomA/PolynomB and the class default order (``magnet_elements.py:242-253``),
and every array attribute stored as a Fortran-ordered float64 array
(``elements/conversions.py:10-18``).
"""
from __future__ import annotations

import copy as _copy

import numpy as np

__all__ = [
    "Element", "Marker", "Monitor", "Drift", "ThinMultipole", "Multipole",
    "Quadrupole", "Sextupole", "Octupole", "Dipole", "Bend", "RFCavity",
    "Corrector", "Aperture", "Lattice", "Particle",
]

_ARRAYS = {
    "PolynomA", "PolynomB", "KickAngle", "T1", "T2", "R1", "R2", "RApertures",
    "EApertures", "Limits", "fringeIntM0", "fringeIntP0", "BendingAngleArray",
}


def _farray(value, shape=(-1,)):
    return np.require(value, dtype=np.float64, requirements=["F", "A"]).reshape(shape, order="F")


class Element:
    """Base element: a family name, a PassMethod and free attributes."""

    def __init__(self, family_name: str, length: float = 0.0, **kwargs):
        self.FamName = family_name
        self.Length = float(length)
        kwargs.setdefault("PassMethod", "IdentityPass")
        for k, v in kwargs.items():
            setattr(self, k, v)

    def __setattr__(self, key, value):
        if key in ("R1", "R2", "Lmatp"):
            value = _farray(value, (6, 6))
        elif key in _ARRAYS:
            value = _farray(value)
        elif key in ("MaxOrder", "NumIntSteps", "FringeBendEntrance", "FringeBendExit",
                     "FringeQuadEntrance", "FringeQuadExit"):
            value = int(value)
        super().__setattr__(key, value)

    def copy(self):
        return _copy.deepcopy(self)

    def deepcopy(self):
        return _copy.deepcopy(self)

    def __repr__(self):
        return "%s(%r, PassMethod=%r)" % (type(self).__name__, self.FamName, self.PassMethod)


class Marker(Element):
    def __init__(self, family_name: str, **kwargs):
        super().__init__(family_name, 0.0, **kwargs)


class Monitor(Marker):
    pass


class Drift(Element):
    def __init__(self, family_name: str, length: float, **kwargs):
        kwargs.setdefault("PassMethod", "DriftPass")
        super().__init__(family_name, length, **kwargs)


class Aperture(Element):
    def __init__(self, family_name: str, limits, **kwargs):
        kwargs.setdefault("PassMethod", "AperturePass")
        super().__init__(family_name, 0.0, Limits=limits, **kwargs)


class ThinMultipole(Element):
    DefaultOrder = 0

    def __init__(self, family_name: str, poly_a, poly_b, length: float = 0.0, **kwargs):
        pa = np.asarray(kwargs.pop("PolynomA", poly_a), dtype=np.float64).ravel()
        pb = np.asarray(kwargs.pop("PolynomB", poly_b), dtype=np.float64).ravel()
        deforder = max(self.DefaultOrder, len(pa) - 1, len(pb) - 1)
        maxorder = int(kwargs.pop("MaxOrder", deforder))
        kwargs.setdefault("PassMethod", "ThinMPolePass")
        super().__init__(family_name, length, **kwargs)
        self.MaxOrder = maxorder
        n = max(maxorder, deforder) + 1
        self.PolynomA = np.pad(pa, (0, n - len(pa)))
        self.PolynomB = np.pad(pb, (0, n - len(pb)))


class Multipole(ThinMultipole):
    def __init__(self, family_name: str, length: float, poly_a, poly_b, **kwargs):
        kwargs.setdefault("PassMethod", "StrMPoleSymplectic4Pass")
        kwargs.setdefault("NumIntSteps", 10)
        super().__init__(family_name, poly_a, poly_b, length=length, **kwargs)

    @property
    def K(self) -> float:
        return float(self.PolynomB[1])

    @K.setter
    def K(self, value: float):
        self.PolynomB[1] = value


class Quadrupole(Multipole):
    DefaultOrder = 1

    def __init__(self, family_name: str, length: float, k: float = 0.0, **kwargs):
        super().__init__(family_name, length, [], [0.0, k], **kwargs)


class Sextupole(Multipole):
    DefaultOrder = 2

    def __init__(self, family_name: str, length: float, h: float = 0.0, **kwargs):
        super().__init__(family_name, length, [], [0.0, 0.0, h], **kwargs)


class Octupole(Multipole):
    DefaultOrder = 3


class Dipole(Multipole):
    DefaultOrder = 1

    def __init__(self, family_name: str, length: float, bending_angle: float = 0.0,
                 k: float = 0.0, **kwargs):
        kwargs.setdefault("BendingAngle", float(bending_angle))
        kwargs.setdefault("EntranceAngle", 0.0)
        kwargs.setdefault("ExitAngle", 0.0)
        kwargs.setdefault("PassMethod", "BndMPoleSymplectic4Pass")
        super().__init__(family_name, length, [], [0.0, k], **kwargs)


Bend = Dipole


class RFCavity(Element):
    def __init__(self, family_name: str, length: float, voltage: float, frequency: float,
                 harmonic_number: int, energy: float, **kwargs):
        kwargs.setdefault("TimeLag", 0.0)
        kwargs.setdefault("PassMethod", "RFCavityPass")
        super().__init__(family_name, length, Voltage=float(voltage),
                         Frequency=float(frequency), HarmNumber=int(harmonic_number),
                         Energy=float(energy), **kwargs)


class QuantumDiffusion(Element):
    """Lumped quantum excitation: random kicks r += L z, L the lower
    triangular ``Lmatp`` (6x6), z six standard normals (QuantDiffPass)."""

    def __init__(self, family_name: str, lmatp, **kwargs):
        kwargs.setdefault("PassMethod", "QuantDiffPass")
        lm = np.asfortranarray(np.asarray(lmatp, dtype=np.float64).reshape(6, 6))
        super().__init__(family_name, 0.0, Lmatp=lm, **kwargs)


class Corrector(Element):
    def __init__(self, family_name: str, length: float, kick_angle, **kwargs):
        kwargs.setdefault("PassMethod", "CorrectorPass")
        super().__init__(family_name, length, KickAngle=kick_angle, **kwargs)


class Particle:
    """Particle type: rest energy [eV] and charge, as ``at.lattice.Particle``."""

    _known = {
        "relativistic": (0.0, -1.0),
        "electron": (510998.95069, -1.0),
        "positron": (510998.95069, 1.0),
        "proton": (938272089.4300001, 1.0),
    }

    def __init__(self, name: str = "relativistic", rest_energy: float | None = None,
                 charge: float | None = None):
        re0, ch0 = self._known.get(name, (0.0, -1.0))
        self.name = name
        self.rest_energy = float(re0 if rest_energy is None else rest_energy)
        self.charge = float(ch0 if charge is None else charge)


class Lattice(list):
    """A list of elements with ``energy``/``particle`` ring attributes."""

    def __init__(self, elems=(), energy: float = 0.0, particle="relativistic",
                 name: str = "", periodicity: int = 1):
        super().__init__(elems)
        self.energy = float(energy)
        self.particle = particle if isinstance(particle, Particle) else Particle(particle)
        self.name = name
        self.periodicity = periodicity

    @property
    def circumference(self) -> float:
        return float(sum(getattr(e, "Length", 0.0) for e in self))

    @property
    def revolution_frequency(self) -> float:
        from .lattice import C0
        return C0 / self.circumference

    def copy(self):
        return _copy.copy(self)

    def deepcopy(self):
        return _copy.deepcopy(self)
