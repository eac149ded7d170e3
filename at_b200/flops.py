"""Algorithmic FP64 operation counts per particle and element.

Counts every +, -, *, / written in the reference integrators, per particle,
per pass (a division counts 1; a fused multiply-add, were the reference to
write one, would count 2; comparisons, ``fabs`` and sign flips count 0).
``sin``/``tan``/``exp`` calls are counted separately.  These are the
numerators of the roofline: what the reference algorithm computes, not what
the fast kernel happens to execute.

Per-routine counts (reference file:lines):
  fastdrift            12        driftkick.c:37-48
  strthinkick          8n+4      driftkick.c:92-115
  bndthinkick          8n+11     driftkick.c:51-89
  ATdrift6 / drift6    14        atlalib.c:59-68, driftkickrad.c:36-45
  diff_drift           16        diff_drift.c:30-43 (xpr, ypr computed)
  diff_str_kick        8n+37     diff_str_kick.c:19-83 with B2perp :1-17
  diff_bnd_kick        8n+56     diff_bnd_kick.c:101-174 with B2perp :85-99
  edge_fringe          9 + 2 tan atphyslib.c:15-79 (method 0/1 with fc = 0)
  diff_bend_fringe     10 + 2 tan diff_bend_fringe.c:1-52 (psi = 0)
  ATaddvv / ATmultmv   6 / 72    atlalib.c:17-57
  ATChangePRef         5 (+1)    atlalib.c:70-75
  QuadFringePassP/N    38        quadfringe.c:3-51
  RF kick              11 + sin  attrackfunc.c:24,36
"""
from __future__ import annotations

from . import table as T
from .lattice import CompiledLattice


def element_flops(info, words, off) -> tuple[int, int]:
    """(flops, transcendental calls) per particle for one compiled element."""
    import numpy as np

    op = info.opcode
    rec = words[off: off + 2].view(np.uint64)
    optw = int(rec[1])

    def has(slot):
        return ((optw >> (slot * T.ATB_OPT_BITS)) & T.ATB_OPT_MASK) != 0

    mis = (6 if has(T.ATB_OPT_T1) else 0) + (72 if has(T.ATB_OPT_R1) else 0) + \
          (72 if has(T.ATB_OPT_R2) else 0) + (6 if has(T.ATB_OPT_T2) else 0)
    ell = 5 if has(T.ATB_OPT_EAP) else 0
    fl = info.flags
    n = info.max_order
    ns = info.nsteps
    scal = 11 if (fl & T.ATB_F_SCALING) else 0
    trans = 0
    if op == T.ATB_OP_IDENTITY:
        f = mis + ell
    elif op == T.ATB_OP_DRIFT:
        f = mis + 2 * ell + 14
    elif op in (T.ATB_OP_STRMPOLE, T.ATB_OP_BNDMPOLE, T.ATB_OP_STRMPOLE_RAD,
                T.ATB_OP_BNDMPOLE_RAD):
        rad = op in (T.ATB_OP_STRMPOLE_RAD, T.ATB_OP_BNDMPOLE_RAD)
        bend = op in (T.ATB_OP_BNDMPOLE, T.ATB_OP_BNDMPOLE_RAD)
        f = mis + 2 * ell + scal
        if rad:
            kick = 8 * n + (56 if bend else 37)
            f += ns * (4 * 16 + 3 * kick)
            if bend:
                f += 2 * 10
                trans += 4
        else:
            kick = 8 * n + (11 if bend else 4)
            f += 4 + ns * (4 * 12 + 3 * kick)
            if bend:
                f += 2 * 9
                trans += 4
        for bit, lin in ((T.ATB_F_FQ_IN, T.ATB_F_FQ_IN_LIN), (T.ATB_F_FQ_OUT, T.ATB_F_FQ_OUT_LIN)):
            if fl & bit:
                f += 38 + (2 * (25 + 12) if fl & lin else 0)
                trans += 4 if fl & lin else 0
    elif op == T.ATB_OP_THINMPOLE:
        f = mis + ell + scal + 8 * n + 12
    elif op == T.ATB_OP_RFCAVITY:
        f = 11 if (fl & T.ATB_F_NV) else 0
        trans = 1 if (fl & T.ATB_F_NV) else 0
        if fl & T.ATB_F_THICK:
            f += 2 * 14
    elif op == T.ATB_OP_CORRECTOR:
        f = mis + scal + (30 + 2 * ell if fl & T.ATB_F_THICK else 2 + ell)
    elif op == T.ATB_OP_APERTURE:
        f = 0
    elif op == T.ATB_OP_QUANTDIFF:
        f, trans = 21 * 2 + 6 + 3 * 6, 9          # L z, six adds, Box-Muller; log/sqrt/sincos
    else:
        f = 0
    return f, trans


def flops_per_particle_turn(cl: CompiledLattice) -> tuple[int, int]:
    """Algorithmic (flops, transcendental calls) for one particle and one turn."""
    tot = 0
    tr = 0
    for i, info in enumerate(cl.info):
        f, t = element_flops(info, cl.words, int(cl.offsets[i]))
        tot += f
        tr += t
    return tot, tr
