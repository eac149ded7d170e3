"""Lattice compiler: a list of AT elements -> flat element table.

This is the host half of the drop-in for the reference's per-element
attribute readers (``atintegrators/atelem.c:219-352``) and per-pass-method
set-up code (``trackFunction`` of each ``atintegrators/<PassMethod>.c``).
Elements are read by attribute, exactly like the reference's
``PyObject_GetAttrString`` calls, so any object with the reference's
attribute names works (pyat's ``Element`` subclasses, or
:mod:`at_b200.elements`).

Everything that the reference computes once per element (slice lengths,
KickAngle folded into the dipole coefficients, edge-focusing tangents, RF
harmonic number, radiation constant) is evaluated here with IEEE double
arithmetic in the reference's operation order, so the device integrators see
the same constants bit for bit.  Errors follow the reference: a missing
required attribute is an ``AttributeError``, a wrong array type a
``RuntimeError`` (``atelem.c:287-317``), an unknown PassMethod a
``RuntimeError`` (``pyat/at.c:256-262``) and a non-positive energy for an RF or
radiating element a ``ValueError`` (``atelem.c:203-211``).  Element errors are
raised lazily, only when tracking reaches the element, as the reference does.
"""
from __future__ import annotations

import math
import operator
from dataclasses import dataclass, field

import numpy as np

from . import table as T

# ---------------------------------------------------------------------------
# Reference constants (atintegrators/atconstants.h:16-31, pyat/at.c:52-53)
# ---------------------------------------------------------------------------
THIRD_ROOT_2 = 1.25992104989487316477
DRIFT1 = 1.0 / (2.0 * (2.0 - THIRD_ROOT_2))
DRIFT2 = 0.5 - (1.0 / (2.0 * (2.0 - THIRD_ROOT_2)))
KICK1 = 1.0 / (2.0 - THIRD_ROOT_2)
KICK2 = 1.0 - 2.0 / (2.0 - THIRD_ROOT_2)
TWOPI = 2.0 * math.pi
C0 = 2.99792458e8
RE = 2.8179403205e-15
E0_GEV = 510.99895069e-6
RAD_CONST = 2.0 / 3.0 * RE
ROOT_3 = 1.7320508075688772
HBAR_C = 197.3269804e-18            # reduced Planck constant x c [GeV.m]
# atconstants.h:30, evaluated in the same order
DIF_CONST = 55.0 / 24.0 / ROOT_3 * HBAR_C / E0_GEV * RE


def diffusion_constant(energy: float, rest_energy: float) -> float:
    """DIF_CONST * gamma^5, the quantum-diffusion strength of the radiating
    multipole passes (StrMPoleSymplectic4RadPass.c: diff_const)."""
    return DIF_CONST * math.pow(_gamma(energy, rest_energy), 5)
LIMIT_AMPLITUDE = 1.0

_f64 = np.float64


def _ieee(op, a, b):
    """One IEEE double operation with C semantics (no Python exceptions)."""
    with np.errstate(all="ignore"):
        return float(op(_f64(a), _f64(b)))


def _div(a, b):
    return _ieee(np.divide, a, b)


def c_round(x: float) -> float:
    """C ``round()``: nearest integer, halfway cases away from zero."""
    if not math.isfinite(x):
        return x
    ax = abs(x)
    fl = math.floor(ax)
    r = fl + 1.0 if (ax - fl) >= 0.5 else fl
    return math.copysign(r, x)


# ---------------------------------------------------------------------------
# attribute readers mirroring atelem.c
# ---------------------------------------------------------------------------
def _get_double(el, name: str) -> float:
    return float(getattr(el, name))                     # atelem.c:228-235


def _get_long(el, name: str) -> int:
    return operator.index(getattr(el, name))            # atelem.c:219-226


def _opt_double(el, name: str, default: float) -> float:
    try:
        return _get_double(el, name)
    except (AttributeError, TypeError, ValueError):     # atelem.c:247-255
        return default


def _opt_long(el, name: str, default: int) -> int:
    try:
        return _get_long(el, name)
    except (AttributeError, TypeError, ValueError):     # atelem.c:237-245
        return default


def _check_array(a, name: str) -> np.ndarray:
    """atelem.c:287-317: ndarray, float64, Fortran-contiguous."""
    if not isinstance(a, np.ndarray):
        raise RuntimeError("The attribute %s is not an array." % name)
    if a.dtype != np.float64:
        raise RuntimeError("The attribute %s is not a double array." % name)
    if not (a.flags.f_contiguous and a.flags.aligned):
        raise RuntimeError("The attribute %s is not Fortran-aligned." % name)
    return a.ravel(order="F")


def _get_array(el, name: str) -> np.ndarray:
    return _check_array(getattr(el, name), name)        # atelem.c:319-328


def _opt_array(el, name: str):
    try:
        a = getattr(el, name)                           # atelem.c:336-346
    except AttributeError:
        return None
    return _check_array(a, name)


def _need(arr, n: int, name: str):
    if arr is not None and arr.size < n:
        raise ValueError("The attribute %s has %d values, %d required" % (name, arr.size, n))
    return arr


# ---------------------------------------------------------------------------
# record builder
# ---------------------------------------------------------------------------
def _pack_header(op: int, max_order: int, flags: int, nsteps: int, nwords: int) -> int:
    return ((op & T.ATB_H_OP_MASK) << T.ATB_H_OP_SHIFT
            | (max_order & T.ATB_H_MO_MASK) << T.ATB_H_MO_SHIFT
            | (flags & T.ATB_H_FL_MASK) << T.ATB_H_FL_SHIFT
            | (nsteps & T.ATB_H_NS_MASK) << T.ATB_H_NS_SHIFT
            | (nwords & T.ATB_H_LEN_MASK) << T.ATB_H_LEN_SHIFT)


def _tilt_pattern(r: np.ndarray):
    """8 rotation entries if the 6x6 (column-major) R only couples x/y planes."""
    m = r.reshape(6, 6, order="F")
    keep = {(0, 0), (0, 2), (1, 1), (1, 3), (2, 0), (2, 2), (3, 1), (3, 3)}
    for i in range(6):
        for j in range(6):
            if (i, j) in keep:
                continue
            if i == j and i >= 4:
                if m[i, j] != 1.0:
                    return None
            elif m[i, j] != 0.0:
                return None
    return [m[0, 0], m[0, 2], m[1, 1], m[1, 3], m[2, 0], m[2, 2], m[3, 1], m[3, 3]]


class _Record:
    def __init__(self, op: int, nfixed: int):
        self.op = op
        self.fields = [0.0] * nfixed        # words 2.. nfixed+1 (index = word)
        self.flags = 0
        self.max_order = 0
        self.nsteps = 0
        self.blocks: list[tuple[int, list[float]]] = []

    def set(self, word: int, value: float):
        while len(self.fields) <= word:
            self.fields.append(0.0)
        self.fields[word] = float(value)

    def add_block(self, slot: int, values):
        self.blocks.append((slot, [float(v) for v in values]))

    def words(self) -> np.ndarray:
        body = list(self.fields[2:])
        pos = 2 + len(body)
        offs = [0] * T.ATB_NUM_OPT
        for slot, vals in self.blocks:
            if pos % 2:                      # 16-byte align every block
                body.append(0.0)
                pos += 1
            offs[slot] = pos
            body.extend(vals)
            pos += len(vals)
        if pos % 2:
            body.append(0.0)
            pos += 1
        if pos > T.ATB_MAX_RECORD_WORDS:
            raise ValueError("element record too long (%d words)" % pos)
        out = np.zeros(pos, dtype=np.float64)
        out[2:] = body
        u = out.view(np.uint64)
        u[0] = _pack_header(self.op, self.max_order, self.flags, self.nsteps, pos)
        optw = 0
        for s, o in enumerate(offs):
            optw |= (o & T.ATB_OPT_MASK) << (s * T.ATB_OPT_BITS)
        u[1] = optw
        return out


def _add_misalign_entrance(rec: _Record, el):
    t1 = _need(_opt_array(el, "T1"), 6, "T1")
    r1 = _need(_opt_array(el, "R1"), 36, "R1")
    rap = _need(_opt_array(el, "RApertures"), 4, "RApertures")
    eap = _need(_opt_array(el, "EApertures"), 2, "EApertures")
    r2 = _need(_opt_array(el, "R2"), 36, "R2")
    t2 = _need(_opt_array(el, "T2"), 6, "T2")
    if t1 is not None:
        rec.add_block(T.ATB_OPT_T1, t1[:6])
    if r1 is not None:
        tilt = _tilt_pattern(r1[:36])
        if tilt is None:
            rec.flags |= T.ATB_F_R1_DENSE
            rec.add_block(T.ATB_OPT_R1, r1[:36])
        else:
            rec.add_block(T.ATB_OPT_R1, tilt)
    if rap is not None:
        rec.add_block(T.ATB_OPT_RAP, rap[:4])
    if eap is not None:
        rec.add_block(T.ATB_OPT_EAP, eap[:2])
    if r2 is not None:
        tilt = _tilt_pattern(r2[:36])
        if tilt is None:
            rec.flags |= T.ATB_F_R2_DENSE
            rec.add_block(T.ATB_OPT_R2, r2[:36])
        else:
            rec.add_block(T.ATB_OPT_R2, tilt)
    if t2 is not None:
        rec.add_block(T.ATB_OPT_T2, t2[:6])


def _fringe_matrix(k1: float, fint: np.ndarray, part: int):
    """2x2 x/y blocks of quadfringe.c:quadPartialFringeMatrix (lines 3-43)."""
    in_fringe = 1.0
    k1sqr = k1 * k1
    if part == 1:
        j1x = in_fringe * (k1 * fint[1] - 2 * k1sqr * fint[3] / 3. - k1sqr * fint[0] * fint[2] / 2)
        j2x = in_fringe * k1 * fint[2]
        j3x = in_fringe * k1sqr * (fint[2] + fint[4] + fint[0] * fint[1])
        j1y = in_fringe * (-k1 * fint[1] - 2 * k1sqr * fint[3] / 3. - k1sqr * fint[0] * fint[2] / 2)
    else:
        j1x = in_fringe * (k1 * fint[1] + k1sqr * fint[0] * fint[2] / 2)
        j2x = in_fringe * k1 * fint[2]
        j3x = in_fringe * k1sqr * (fint[4] - fint[0] * fint[1])
        j1y = in_fringe * (-k1 * fint[1] + k1sqr * fint[0] * fint[2] / 2)
    j2y = -j2x
    j3y = j3x
    ex = math.exp(j1x)
    ey = math.exp(j1y)
    mx = [ex, _div(j2x, ex), ex * j3x, _div(1 + j2x * j3x, ex)]
    my = [ey, _div(j2y, ey), ey * j3y, _div(1 + j2y * j3y, ey)]
    return mx, my


def _fringe_block(b1: float, fm, fp):
    """Entrance maps (P part 2, swapped; M part 1, swapped) and exit maps
    (M part 1; P part 2), quadfringe.c:45-112, as 4 x (x 2x2 + y 2x2)."""
    def swapped(m):
        return [m[3], m[1], m[2], m[0]]
    out = []
    mx, my = _fringe_matrix(b1, fp, 2)
    out += swapped(mx) + swapped(my)
    mx, my = _fringe_matrix(b1, fm, 1)
    out += swapped(mx) + swapped(my)
    mx, my = _fringe_matrix(b1, fm, 1)
    out += mx + my
    mx, my = _fringe_matrix(b1, fp, 2)
    out += mx + my
    return out


def _gamma(energy: float, rest_energy: float) -> float:
    """atelem.c:364-371 (atGamma) with the PYAT atEnergy rule (:203-211)."""
    if not energy > 0.0:
        raise ValueError("Energy must be positive. Check lattice or set the track() keyword argument.")
    if rest_energy == 0.0:
        return 1.0E-9 * energy / E0_GEV
    return energy / rest_energy


def _multipole_common(rec: _Record, el, op: int, bend: bool, integrator: int = 4):
    le = _get_double(el, "Length")
    pa = _get_array(el, "PolynomA")
    pb = _get_array(el, "PolynomB")
    mo = _get_long(el, "MaxOrder")
    ns = _get_long(el, "NumIntSteps")
    if bend:
        bending_angle = _get_double(el, "BendingAngle")
        entrance_angle = _get_double(el, "EntranceAngle")
        exit_angle = _get_double(el, "ExitAngle")
    if op in (T.ATB_OP_STRMPOLE_RAD, T.ATB_OP_BNDMPOLE_RAD):
        _opt_double(el, "Energy", 0.0)
    if bend:
        fbe = _opt_long(el, "FringeBendEntrance", 1)
        fbx = _opt_long(el, "FringeBendExit", 1)
        gap = _opt_double(el, "FullGap", 0)
    scaling = _opt_double(el, "FieldScaling", 1.0)
    if bend:
        fint1 = _opt_double(el, "FringeInt1", 0)
        fint2 = _opt_double(el, "FringeInt2", 0)
    fqe = _opt_long(el, "FringeQuadEntrance", 0)
    fqx = _opt_long(el, "FringeQuadExit", 0)
    fim = _opt_array(el, "fringeIntM0")
    fip = _opt_array(el, "fringeIntP0")
    _add_misalign_entrance(rec, el)
    ka = _need(_opt_array(el, "KickAngle"), 2, "KickAngle")
    if mo < 0 or mo > T.ATB_MAX_ORDER:
        raise ValueError("MaxOrder %d outside [0, %d]" % (mo, T.ATB_MAX_ORDER))
    if ns < 0 or ns > T.ATB_H_NS_MASK:
        raise ValueError("NumIntSteps %d out of range" % ns)
    _need(pa, mo + 1, "PolynomA")
    _need(pb, mo + 1, "PolynomB")
    A = [float(v) for v in pa[: mo + 1]]
    B = [float(v) for v in pb[: mo + 1]]
    b1_fringe = float(pb[1]) if pb.size > 1 else 0.0
    # StrMPoleSymplectic4Pass.c:39-52 (same lines in the Bnd and Rad variants)
    sl = _div(le, ns)
    rec.set(T.ATB_SM_L1, sl * DRIFT1)
    rec.set(T.ATB_SM_L2, sl * DRIFT2)
    rec.set(T.ATB_SM_K1, sl * KICK1)
    rec.set(T.ATB_SM_K2, sl * KICK2)
    if integrator != 4:
        # another integrator of the GPU call: the step and the id replace the
        # Forest-Ruth lengths (atgpu/SymplecticIntegrator.cpp:140-171)
        rec.flags |= T.ATB_F_INTEG
        rec.set(T.ATB_SM_SL, sl)
        rec.set(T.ATB_SM_ONE, 1.0)
        rec.set(T.ATB_SM_INTEG, float(integrator))
        rec.set(T.ATB_SM_K2, 0.0)
    if ka is not None:
        B[0] = B[0] - _div(math.sin(ka[0]), le)
        A[0] = A[0] + _div(math.sin(ka[1]), le)
    rec.set(T.ATB_SM_SCALE, scaling)
    rec.set(T.ATB_SM_ISCALE, _div(1.0, scaling))
    if scaling != 1.0:
        rec.flags |= T.ATB_F_SCALING
    rec.set(T.ATB_SM_B1, b1_fringe)
    rec.max_order = mo
    rec.nsteps = ns
    use_lin_in = fim is not None and fip is not None and fqe == 2
    use_lin_out = fim is not None and fip is not None and fqx == 2
    if fqe and b1_fringe != 0:
        rec.flags |= T.ATB_F_FQ_IN
        if use_lin_in:
            rec.flags |= T.ATB_F_FQ_IN_LIN
    if fqx and b1_fringe != 0:
        rec.flags |= T.ATB_F_FQ_OUT
        if use_lin_out:
            rec.flags |= T.ATB_F_FQ_OUT_LIN
    if (rec.flags & (T.ATB_F_FQ_IN_LIN | T.ATB_F_FQ_OUT_LIN)):
        _need(fim, 5, "fringeIntM0")
        _need(fip, 5, "fringeIntP0")
        rec.add_block(T.ATB_OPT_FRINGE, _fringe_block(b1_fringe, fim, fip))
    if bend:
        irho = _div(bending_angle, le)
        k1 = sl * KICK1
        k2 = sl * KICK2
        rec.set(T.ATB_BM_IRHO, irho)
        rec.set(T.ATB_BM_K1IRHO, k1 * irho)
        rec.set(T.ATB_BM_K2IRHO, k2 * irho)
        for (w_e, w_fc, w_fx, w_fy, angle, fint, method, shift, fc0) in (
            (T.ATB_BM_EIN, T.ATB_BM_FCIN, T.ATB_BM_FXIN, T.ATB_BM_FYIN,
             entrance_angle, fint1, fbe, T.ATB_F_BM_IN_SHIFT, T.ATB_F_FC0_IN),
            (T.ATB_BM_EOUT, T.ATB_BM_FCOUT, T.ATB_BM_FXOUT, T.ATB_BM_FYOUT,
             exit_angle, fint2, fbx, T.ATB_F_BM_OUT_SHIFT, T.ATB_F_FC0_OUT),
        ):
            # atphyslib.c:15-79, diff_bend_fringe.c:1-30
            if fint == 0.0 or gap == 0.0 or method == 0:
                fc = 0.0
            else:
                sedge = math.sin(angle)
                cedge = math.cos(angle)
                fc = _div(irho * gap * fint * (1 + sedge * sedge), cedge)
            tn = math.tan(angle)
            rec.set(w_e, angle)
            rec.set(w_fc, fc)
            rec.set(w_fx, irho * tn)
            rec.set(w_fy, irho * tn)
            code = method if method in (1, 2, 3) else T.ATB_BM_LEGACY
            rec.flags |= (code & T.ATB_F_BM_MASK) << shift
            if fc == 0.0:
                rec.flags |= fc0
            if fint > 0 and gap > 0:
                rec.flags |= T.ATB_F_FINT_IN if shift == T.ATB_F_BM_IN_SHIFT else T.ATB_F_FINT_OUT
        base = T.ATB_BM_POLY
    else:
        base = T.ATB_SM_POLY
    for i, v in enumerate(A):
        rec.set(base + i, v)
    for i, v in enumerate(B):
        rec.set(base + mo + 1 + i, v)
    if all(v == 0.0 for v in A):
        rec.flags |= T.ATB_F_NOSKEW


@dataclass
class ElementInfo:
    opcode: int
    pass_method: str
    length: float
    max_order: int = 0
    nsteps: int = 0
    flags: int = 0
    error: BaseException | None = None


@dataclass
class CompiledLattice:
    """A lattice compiled to a flat element table."""
    words: np.ndarray                      #: float64 words (headers bit-cast)
    offsets: np.ndarray                    #: uint32, nelem + 1 entries
    info: list[ElementInfo]
    ring_length: float
    t0: float
    energy: float
    rest_energy: float
    charge: float = -1.0
    #: (word index, element index, kind) of energy-dependent fields
    energy_fields: list[tuple[int, int, str]] = field(default_factory=list)
    voltages: dict[int, float] = field(default_factory=dict)

    @property
    def nelem(self) -> int:
        return len(self.info)

    def first_error(self, start: int, end: int, nturns: int):
        """The error the reference would raise first while tracking."""
        if nturns <= 0:
            return None
        order = list(range(start, end))
        if nturns > 1:
            order += list(range(0, start))
        for i in order:
            if self.info[i].error is not None:
                return self.info[i].error
        return None

    def set_energy(self, energy: float, rest_energy: float):
        """Refresh the fields that the reference recomputes on every call
        (RF ``Voltage/energy``: RFCavityPass.c:387-390; ``RAD_CONST*gamma^3``:
        StrMPoleSymplectic4RadPass.c:50,171)."""
        if energy == self.energy and rest_energy == self.rest_energy:
            return
        for w, i, kind in self.energy_fields:
            info = self.info[i]
            try:
                if kind == "nv":
                    if not energy > 0.0:
                        raise ValueError("Energy must be positive. Check lattice or set the track() keyword argument.")
                    self.words[w] = _div(self.voltages[i], energy)
                else:
                    g = _gamma(energy, rest_energy)
                    self.words[w] = RAD_CONST * math.pow(g, 3)
                if info.error is not None and getattr(info.error, "_energy", False):
                    info.error = None
            except ValueError as exc:
                exc._energy = True
                info.error = exc
        self.energy = energy
        self.rest_energy = rest_energy


def _compile_element(el, idx: int, energy: float, rest_energy: float, t0: float,
                     cl_fields: list, voltages: dict, integrator: int = 4):
    pm = getattr(el, "PassMethod")
    op = T.PASS_OPCODES[pm]
    if op == T.ATB_OP_IDENTITY:
        rec = _Record(op, 2)
        _add_misalign_entrance(rec, el)
    elif op == T.ATB_OP_DRIFT:
        rec = _Record(op, 3)
        rec.set(T.ATB_DR_LE, _get_double(el, "Length"))
        _add_misalign_entrance(rec, el)
    elif op in (T.ATB_OP_STRMPOLE, T.ATB_OP_STRMPOLE_RAD):
        rec = _Record(op, T.ATB_SM_POLY)
        _multipole_common(rec, el, op, bend=False, integrator=integrator)
    elif op in (T.ATB_OP_BNDMPOLE, T.ATB_OP_BNDMPOLE_RAD):
        rec = _Record(op, T.ATB_BM_POLY)
        _multipole_common(rec, el, op, bend=True, integrator=integrator)
    elif op == T.ATB_OP_THINMPOLE:
        rec = _Record(op, T.ATB_TM_POLY)
        pa = _get_array(el, "PolynomA")
        pb = _get_array(el, "PolynomB")
        mo = _get_long(el, "MaxOrder")
        scaling = _opt_double(el, "FieldScaling", 1.0)
        bax = bay = 0.0
        try:
            ba = getattr(el, "BendingAngle")           # ThinMPolePass.c:219-224
        except AttributeError:
            ba = None
        if ba is not None:
            flat = _check_array(ba, "BendingAngle")
            # atelem.c:312-315: the size is dims[0]*dims[1], and dims[1] is 0
            # for a 1-D array, so only a 2-D BendingAngle is used
            sz = ba.shape[0] * ba.shape[1] if ba.ndim >= 2 else 0
            if sz >= 2:
                bay = float(flat[1])
            if sz >= 1:
                bax = float(flat[0])
        _add_misalign_entrance(rec, el)
        ka = _need(_opt_array(el, "KickAngle"), 2, "KickAngle")
        if mo < 0 or mo > T.ATB_MAX_ORDER:
            raise ValueError("MaxOrder %d outside [0, %d]" % (mo, T.ATB_MAX_ORDER))
        _need(pa, mo + 1, "PolynomA")
        _need(pb, mo + 1, "PolynomB")
        A = [float(v) for v in pa[: mo + 1]]
        B = [float(v) for v in pb[: mo + 1]]
        if ka is not None:                             # ThinMPolePass.c:170-173
            B[0] = B[0] - float(ka[0])
            A[0] = A[0] + float(ka[1])
        rec.max_order = mo
        rec.set(T.ATB_TM_BAX, bax)
        rec.set(T.ATB_TM_BAY, bay)
        rec.set(T.ATB_TM_SCALE, scaling)
        rec.set(T.ATB_TM_ISCALE, _div(1.0, scaling))
        if scaling != 1.0:
            rec.flags |= T.ATB_F_SCALING
        for i, v in enumerate(A):
            rec.set(T.ATB_TM_POLY + i, v)
        for i, v in enumerate(B):
            rec.set(T.ATB_TM_POLY + mo + 1 + i, v)
    elif op == T.ATB_OP_RFCAVITY:
        rec = _Record(op, T.ATB_RF_HALF + 1)
        le = _get_double(el, "Length")                  # RFCavityPass.c:367-373
        voltage = _get_double(el, "Voltage")
        freq = _get_double(el, "Frequency")
        _opt_double(el, "Energy", energy)
        lag = _opt_double(el, "TimeLag", 0)
        philag = _opt_double(el, "PhaseLag", 0)
        harm = c_round(freq * t0)
        rec.set(T.ATB_RF_LE, le)
        rec.set(T.ATB_RF_TF, TWOPI * freq)
        rec.set(T.ATB_RF_LAG, lag)
        rec.set(T.ATB_RF_HT, _div(harm, freq) - t0)
        rec.set(T.ATB_RF_PHI, philag)
        rec.set(T.ATB_RF_HALF, le / 2)
        if le != 0.0:
            rec.flags |= T.ATB_F_THICK
        voltages[idx] = voltage
        cl_fields.append((T.ATB_RF_NV, idx, "nv"))
        rec.set(T.ATB_RF_NV, _div(voltage, energy) if energy > 0.0 else 0.0)
        if voltage != 0.0:
            rec.flags |= T.ATB_F_NV
    elif op == T.ATB_OP_CORRECTOR:
        rec = _Record(op, T.ATB_CO_HY + 1)
        le = _get_double(el, "Length")
        ka = _need(_get_array(el, "KickAngle"), 2, "KickAngle")
        scaling = _opt_double(el, "FieldScaling", 1.0)
        _add_misalign_entrance(rec, el)
        xk, yk = float(ka[0]), float(ka[1])
        rec.set(T.ATB_CO_XK, xk)
        rec.set(T.ATB_CO_YK, yk)
        rec.set(T.ATB_CO_LE, le)
        rec.set(T.ATB_CO_SCALE, scaling)
        rec.set(T.ATB_CO_ISCALE, _div(1.0, scaling))
        rec.set(T.ATB_CO_K2, xk * xk / 3 + yk * yk / 3)   # CorrectorPass.c:72
        rec.set(T.ATB_CO_HX, xk / 2)
        rec.set(T.ATB_CO_HY, yk / 2)
        if scaling != 1.0:
            rec.flags |= T.ATB_F_SCALING
        if le != 0.0:
            rec.flags |= T.ATB_F_THICK
    elif op == T.ATB_OP_APERTURE:
        rec = _Record(op, T.ATB_AP_LIM + 4)
        lim = _need(_get_array(el, "Limits"), 4, "Limits")
        for i in range(4):
            rec.set(T.ATB_AP_LIM + i, lim[i])
    elif op == T.ATB_OP_QUANTDIFF:
        # QuantDiffPass.c:47-57: Lmatp, 6x6 (column-major as pyat stores it)
        rec = _Record(op, T.ATB_QD_L + 36)
        lm = _need(_get_array(el, "Lmatp"), 36, "Lmatp")
        for i in range(36):
            rec.set(T.ATB_QD_L + i, lm[i])
    else:  # pragma: no cover
        raise RuntimeError("unhandled opcode %d" % op)
    if op in (T.ATB_OP_STRMPOLE_RAD, T.ATB_OP_BNDMPOLE_RAD):
        cl_fields.append((T.ATB_SM_RADC, idx, "radc"))
        if energy > 0.0:
            rec.set(T.ATB_SM_RADC, RAD_CONST * math.pow(_gamma(energy, rest_energy), 3))
    return rec


def element_length(el) -> float:
    """pyat/at.c:495-503: Length, or 0 when absent."""
    try:
        return float(getattr(el, "Length"))
    except (AttributeError, TypeError, ValueError):
        return 0.0


def check_pass_methods(line) -> list[str]:
    """pyat/at.c:486-494: every element needs a known PassMethod."""
    names = []
    for el in line:
        pm = getattr(el, "PassMethod")                 # AttributeError if absent
        if not isinstance(pm, str):
            raise TypeError("PassMethod must be a string")
        if pm not in T.PASS_OPCODES:
            raise RuntimeError("PassMethod %s: library, module or trackFunction not found" % pm)
        names.append(pm)
    return names


def check_integrator(integrator) -> int:
    """The GPU call's ``integrator`` (1-6, atgpu/PyInterface.cpp:44-50); other
    values fail as the reference backend's lattice build does
    (atgpu/SymplecticIntegrator.cpp:82-84, PyInterface.cpp:292-296)."""
    k = int(integrator)
    if k < 1 or k > 6:
        raise RuntimeError("at_gpupass() build lattice failed: SymplecticIntegrator, type %d "
                           "not supported" % k)
    return k


def compile_lattice(line, energy: float = 0.0, rest_energy: float = 0.0,
                    charge: float = -1.0, t0: float | None = None,
                    integrator: int = 4) -> CompiledLattice:
    """Compile ``line`` (a sequence of elements) to a flat element table.

    ``t0`` defaults to the revolution time ``RingLength/C0`` of the line
    (pyat/at.c:540-551); single-element tracking passes ``t0=0``
    (pyat/at.c:728-729).  ``integrator`` selects the thick multipoles'
    symplectic integrator (4, Forest-Ruth, is the CPU engine's).
    """
    integrator = check_integrator(integrator)
    names = check_pass_methods(line)
    ring_length = 0.0
    for el in line:
        ring_length += element_length(el)
    if t0 is None:
        t0 = ring_length / C0
    chunks = []
    offsets = [0]
    infos: list[ElementInfo] = []
    efields: list[tuple[int, int, str]] = []
    voltages: dict[int, float] = {}
    pos = 0
    for i, (el, pm) in enumerate(zip(line, names)):
        op = T.PASS_OPCODES[pm]
        local: list = []
        try:
            rec = _compile_element(el, i, energy, rest_energy, t0, local, voltages,
                                   integrator)
            w = rec.words()
            info = ElementInfo(op, pm, element_length(el), rec.max_order, rec.nsteps, rec.flags)
            if local and not energy > 0.0:
                # RFCavityPass.c:376 / StrMPoleSymplectic4RadPass.c:148 refuse a
                # non-positive energy; the record stays valid for a later call
                # that supplies one (set_energy clears this error).
                exc = ValueError("Energy must be positive. Check lattice or set the "
                                 "track() keyword argument.")
                exc._energy = True
                info.error = exc
        except (AttributeError, RuntimeError, ValueError, TypeError, KeyError, IndexError) as exc:
            local = []
            w = _Record(T.ATB_OP_IDENTITY, 2).words()   # never executed
            info = ElementInfo(T.ATB_OP_IDENTITY, pm, element_length(el), error=exc)
        for (fw, _, kind) in local:
            efields.append((pos + fw, i, kind))
        chunks.append(w)
        infos.append(info)
        pos += len(w)
        offsets.append(pos)
    words = np.concatenate(chunks) if chunks else np.zeros(0, dtype=np.float64)
    cl = CompiledLattice(words=words, offsets=np.asarray(offsets, dtype=np.uint32),
                         info=infos, ring_length=ring_length, t0=t0, energy=energy,
                         rest_energy=rest_energy, charge=charge,
                         energy_fields=efields, voltages=voltages)
    return cl


def segment_plan(cl: CompiledLattice, cap_words: int):
    """Split the table into consecutive element runs of at most ``cap_words``.

    Returns an int64 array of shape (nseg, 4): first element, element count,
    first word, word count (padded to a multiple of 2 words = 16 bytes)."""
    segs = []
    n = cl.nelem
    i = 0
    off = cl.offsets
    while i < n:
        j = i
        while j < n and (off[j + 1] - off[i]) <= cap_words:
            j += 1
        if j == i:
            raise ValueError("element %d record (%d words) exceeds the segment capacity %d"
                             % (i, off[i + 1] - off[i], cap_words))
        nw = int(off[j] - off[i])
        segs.append((i, j - i, int(off[i]), nw + (nw & 1)))
        i = j
    return np.asarray(segs, dtype=np.int64).reshape(-1, 4)
