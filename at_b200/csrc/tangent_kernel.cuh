/*
 * The tangent kernel: multi-turn tracking in forward-mode automatic
 * differentiation.
 *
 * Each thread carries its particle as six dual numbers with seven derivative
 * slots.  Slots 0-5 hold the tangent map J(s) = d r(s) / d r0, seeded with
 * the identity; every pass method of track_kernel.cuh runs unchanged on this
 * type, so J is propagated through exactly the arithmetic the tracking
 * kernels execute (values are those of the "exact" kernel).  Slot 6 is the
 * derivative with respect to one multipole strength K = PolynomB[k]: at an
 * element that carries a differentiated strength, the slot is seeded inside
 * the element (the explicit partial d field / d B_k = (x + i y)^k, plus the
 * quadrupole-fringe gradient for k = 1) and, on exit, holds g = d r(s_out) /
 * d K for the element alone.  Its effect on the final coordinates is
 * M(s_out -> end) g = J_end J(s_out)^-1 g, so the kernel accumulates the
 * equivalent initial-coordinate perturbation u_K += J(s_out)^-1 g (a 6x6
 * solve with partial pivoting, valid with radiation as well) and clears the
 * slot.  A strength met on several turns accumulates every occurrence.  At
 * the end d r_end / d K = J_end u_K is written out with J_end.
 *
 * This replaces the reference's finite-difference Jacobians
 * (pyat/at/physics/matrix.py:105-165 find_m66, which tracks 12 displaced
 * particles) with exact derivatives of the integrators; the reference's own
 * diff_* routines (atintegrators/diff_*.c) propagate a diffusion matrix, not
 * a tangent map, and are not used here.
 */
#ifndef ATB_TANGENT_KERNEL_CUH
#define ATB_TANGENT_KERNEL_CUH

#include "track_kernel.cuh"

namespace atb {

constexpr int kTanDirs = 7;
using TD = Dual<kTanDirs>;

/* rows of the state as an array of dual numbers (compile-time indices only) */
#define ATB_ROWS(r) {&(r).x, &(r).px, &(r).y, &(r).py, &(r).dp, &(r).ct}

/* w = J^-1 g for J[i][j] = row_i.d[j], g_i = row_i.d[6]: Gaussian elimination
 * with partial pivoting on a 6x7 augmented matrix held in registers (row
 * swaps are selects, so every index is known at compile time). */
__device__ __forceinline__ void solve_tangent(P6T<TD>& r, double w[6]) {
    TD* rows[6] = ATB_ROWS(r);
    double M[6][7];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j < 7; ++j) M[i][j] = rows[i]->d[j];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        /* pivot: the largest |M[i][c]|, i >= c */
        double best = fabs(M[c][c]);
        int piv = c;
#pragma unroll
        for (int i = c + 1; i < 6; ++i) {
            const double a = fabs(M[i][c]);
            if (a > best) { best = a; piv = i; }
        }
#pragma unroll
        for (int i = c + 1; i < 6; ++i) {
            const bool sw = (piv == i);
#pragma unroll
            for (int j = c; j < 7; ++j) {
                const double t = M[c][j];
                M[c][j] = sw ? M[i][j] : t;
                M[i][j] = sw ? t : M[i][j];
            }
        }
        const double inv = 1.0 / M[c][c];
#pragma unroll
        for (int i = c + 1; i < 6; ++i) {
            const double f = M[i][c] * inv;
#pragma unroll
            for (int j = c + 1; j < 7; ++j) M[i][j] -= f * M[c][j];
        }
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double s = M[i][6];
#pragma unroll
        for (int j = i + 1; j < 6; ++j) s -= M[i][j] * w[j];
        w[i] = s / M[i][i];
    }
}

extern "C" __global__ void __launch_bounds__(ATB_TANGENT_THREADS)
atb_tangent_kernel(const AtbTangent A) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const long long np = A.np;

    P6T<TD> r;
    {
        P6 r0;
        load6(A.r + 6 * p, r0);
        r.x = TD(r0.x); r.px = TD(r0.px); r.y = TD(r0.y);
        r.py = TD(r0.py); r.dp = TD(r0.dp); r.ct = TD(r0.ct);
        r.x.d[0] = 1.0; r.px.d[1] = 1.0; r.y.d[2] = 1.0;
        r.py.d[3] = 1.0; r.dp.d[4] = 1.0; r.ct.d[5] = 1.0;
    }
    for (int q = 0; q < A.nparam; ++q) {
#pragma unroll
        for (int i = 0; i < 6; ++i) A.grad[(6LL * q + i) * np + p] = 0.0;
    }

    bool lost = false;
    for (int tt = 0; tt < A.nturns && !lost; ++tt) {
        const int nturn = A.turn0 + tt;
        for (int ei = 0; ei < A.nelem; ++ei) {
            Rec e;
            e.p = A.table + A.elem_off[ei];
            const uint64_t* hp = reinterpret_cast<const uint64_t*>(e.p);
            e.hdr = hp[0];
            e.opt = hp[1];
            const int q = A.pelem ? A.pelem[ei] : -1;
            Param pm{-1, 0.0};
            if (q >= 0) { pm.k = A.porder[q]; pm.v = A.pvalue[q]; }
            track_element(r, e, nturn, pm);
            if (is_bad(r)) {          /* pyat/at.c:115-139 */
                lost = true;
                break;
            }
            if (q >= 0) {
                double w[6];
                solve_tangent(r, w);
#pragma unroll
                for (int i = 0; i < 6; ++i) A.grad[(6LL * q + i) * np + p] += w[i];
                r.x.d[6] = 0.0; r.px.d[6] = 0.0; r.y.d[6] = 0.0;
                r.py.d[6] = 0.0; r.dp.d[6] = 0.0; r.ct.d[6] = 0.0;
            }
        }
    }

    TD* rows[6] = ATB_ROWS(r);
    const double nan = nan_d();
    for (int q = 0; q < A.nparam; ++q) {
        double u[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) u[j] = A.grad[(6LL * q + j) * np + p];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 6; ++j) s += rows[i]->d[j] * u[j];
            A.grad[(6LL * q + i) * np + p] = lost ? nan : s;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int j = 0; j < 6; ++j) A.jac[36 * p + 6 * i + j] = lost ? nan : rows[i]->d[j];
    }
    P6 out;
    if (lost) {
        out.x = nan; out.px = 0.0; out.y = 0.0; out.py = 0.0; out.dp = 0.0; out.ct = 0.0;
    } else {
        out.x = r.x.v; out.px = r.px.v; out.y = r.y.v;
        out.py = r.py.v; out.dp = r.dp.v; out.ct = r.ct.v;
    }
    store6(A.r + 6 * p, out);
    if (A.lost) A.lost[p] = lost ? 1 : 0;
}

}  // namespace atb

#endif  // ATB_TANGENT_KERNEL_CUH
