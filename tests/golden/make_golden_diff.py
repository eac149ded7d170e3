"""Generate ``tests/golden/diff_fd.npz``: finite-difference derivatives of the
tracked coordinates, computed in binary128 by the oracle's integrators
(``oracle/oracle_q.c``), for the exact-derivative (tangent kernel) tests.

Central differences with h = 1e-7, and fourth-order ones (five-point
stencil; h = 1e-8 for the coordinates, 1e-5 for the strengths) as an
independent estimate with a smaller truncation error, with respect to the
initial coordinates and to quadrupole/sextupole strengths.  In binary128
their rounding floor is ~1e-30 relative, so they resolve even the
second-order sextupole terms of particles 1e-6 from the closed orbit, which
a double-precision difference with h = 1e-7 cannot.  Steps are the exact
double differences fl(v +- h) - v (the oracle reads inputs and element data
in double) and the stencil weights are solved for those steps.

    python tests/golden/make_golden_diff.py      (a few minutes on 8 cores)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from at_b200 import diff, rings  # noqa: E402
from oracle import oracle  # noqa: E402

H = 1e-7
H4_COORD = 1e-8
H4_STRENGTH = 1e-5


def _weights(t):
    """First-derivative weights for the stencil offsets ``t`` (k, ...): exact
    for polynomials up to degree k-1 (Vandermonde solve, per trailing
    index)."""
    t = np.asarray(t, dtype=np.float64)
    k = t.shape[0]
    flat = t.reshape(k, -1)
    w = np.empty_like(flat)
    rhs = np.zeros(k)
    rhs[1] = 1.0
    for c in range(flat.shape[1]):
        v = np.vander(flat[:, c], k, increasing=True).T       # v[m, i] = t_i^m
        w[:, c] = np.linalg.solve(v, rhs)
    return w.reshape(t.shape)


def _track(line, x, nturns):
    hi, lo = oracle.track_quad(line, x, nturns, energy=line.energy,
                               rest_energy=line.particle.rest_energy)
    return hi, lo


def _diff(a, b):
    """(hi, lo) pairs a - b in double, without losing the low bits."""
    return (a[0] - b[0]) + (a[1] - b[1])


def coord_fd(line, x, nturns):
    """(central h, fourth order) Jacobians, shape (N, 6, 6) [particle, i, j]."""
    n = x.shape[1]
    offs = (H, -H, 2 * H4_COORD, H4_COORD, 0.0, -H4_COORD, -2 * H4_COORD)
    cols, steps = [], []
    for j in range(6):
        for o in offs:
            xx = x.copy()
            xx[j] += o
            steps.append(xx[j] - x[j])                      # exact step per particle
            cols.append(xx)
    hi, lo = _track(line, np.asfortranarray(np.concatenate(cols, axis=1)), nturns)
    k = len(offs)
    hi = hi.reshape(6, 6, k, n)
    lo = lo.reshape(6, 6, k, n)
    st = np.array(steps).reshape(6, k, n)                    # [j, offset, particle]
    c = np.empty((n, 6, 6))
    c4 = np.empty((n, 6, 6))
    for j in range(6):
        def r(i):
            return hi[:, j, i], lo[:, j, i]
        c[:, :, j] = (_diff(r(0), r(1)) / (st[j, 0] - st[j, 1])).T
        # five-point stencil on the exact offsets; the weights sum to zero,
        # so the values enter as differences from the unperturbed point
        w = _weights(st[j, 2:])                                # (5, n)
        acc = np.zeros((6, n))
        for i in range(5):
            acc += w[i] * _diff(r(2 + i), r(4))
        c4[:, :, j] = acc.T
    return c, c4


def strength_fd(line, params, x, nturns, fourth=True):
    """(central, fourth order) d r / d K, shape (P, 6, N)."""
    g = np.empty((len(params), 6, x.shape[1]))
    g4 = np.full((len(params), 6, x.shape[1]), np.nan)
    f0 = _track(line, x, nturns)
    for q, p in enumerate(params):
        k0 = float(line[p.index].PolynomB[p.order])

        def run(delta):
            lat = line.copy()
            el = line[p.index].copy()
            pb = np.array(el.PolynomB, dtype=np.float64)
            pb[p.order] = k0 + delta
            el.PolynomB = pb
            lat[p.index] = el
            return _track(lat, x, nturns), (k0 + delta) - k0
        (fp, hp), (fm, hm) = run(H), run(-H)
        g[q] = _diff(fp, fm) / (hp - hm)
        if fourth:
            runs = [run(o) for o in (2 * H4_STRENGTH, H4_STRENGTH, -H4_STRENGTH,
                                     -2 * H4_STRENGTH)]
            runs.insert(2, (f0, 0.0))
            w = _weights(np.array([h for _, h in runs]))
            g4[q] = sum(wi * _diff(f, f0) for wi, (f, _) in zip(w, runs))
    return g, g4


def main():
    out = {}
    fodo = rings.fodo_ring()
    orbit = np.load(os.path.join(HERE, "fodo_m66.npz"))["orbit"]
    params = diff.multipole_strengths(fodo)

    x = rings.gaussian(16, [1e-6] * 6, seed=21, centre=orbit)
    out["fodo1_x"] = x
    out["fodo1_jac"], out["fodo1_jac4"] = coord_fd(fodo, x, 1)
    out["fodo1_grad"], out["fodo1_grad4"] = strength_fd(fodo, params, x, 1)
    print("fodo, 1 turn done", flush=True)

    x = rings.gaussian(8, [1e-6] * 6, seed=22, centre=orbit)
    sel = np.arange(0, 128, 8)
    out["fodo100_x"] = x
    out["fodo100_params"] = sel
    out["fodo100_jac"], out["fodo100_jac4"] = coord_fd(fodo, x, 100)
    out["fodo100_grad"], out["fodo100_grad4"] = strength_fd(fodo, [params[q] for q in sel], x,
                                                            100)
    print("fodo, 100 turns done", flush=True)

    large = rings.large_ring(seed=1)
    x = rings.gaussian(8, [1e-6] * 6, seed=23, centre=rings.LARGE_ORBIT)
    out["large1_x"] = x
    out["large1_jac"], out["large1_jac4"] = coord_fd(large, x, 1)
    lp = diff.multipole_strengths(large)[::40]
    out["large10_idx"] = np.array([p.index for p in lp])
    out["large10_order"] = np.array([p.order for p in lp])
    out["large10_x"] = x
    out["large10_grad"], out["large10_grad4"] = strength_fd(large, lp, x, 10)
    print("large ring done", flush=True)
    np.savez_compressed(os.path.join(HERE, "diff_fd.npz"), **out)


if __name__ == "__main__":
    main()
