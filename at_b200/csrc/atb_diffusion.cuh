/*
 * Element maps for Ohmi's envelope: every element's transfer matrix (exact
 * derivatives, the tangent machinery on Dual numbers) and its radiation
 * diffusion matrix, one thread per element, for a particle entering it on
 * the closed orbit.
 *
 * The diffusion matrix restates the bdiff branch of the radiating multipole
 * passes (StrMPoleSymplectic4RadPass.c:30-115, BndMPoleSymplectic4RadPass.c:
 * 39-128) as driven by pyat/at.c:755-831 (diffusion_matrix): B starts at zero
 * and is propagated through every drift (diff_drift.c:1-28), thin kick
 * (thinkickM, diff_thinkick.c:1-33 / diff_bnd_kick.c:1-47) and bend edge
 * (diff_bend_fringe.c:31-46), with the kick's own contribution added
 * (thinkickB, diff_thinkick.c:35-70).  Misalignment rotations, apertures and
 * quadrupole fringes move the orbit but not B, as in the reference.  B is
 * kept column-major ([i][j] at i + 6 j) with the reference's summation order,
 * in the exact arithmetic of this compilation unit.
 */
#ifndef ATB_DIFFUSION_CUH
#define ATB_DIFFUSION_CUH

#include "tangent_kernel.cuh"

namespace atb {

/* B <- M B M^T: M B column by column, then (M B) M^T row by row
 * (atlalib.c:92-147) */
__device__ __forceinline__ void bd_sandwich(const double* M, double* B) {
    double t[6];
    for (int i = 0; i < 6; ++i) {
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += M[j + 6 * k] * B[k + 6 * i];
            t[j] = s;
        }
        for (int j = 0; j < 6; ++j) B[j + 6 * i] = t[j];
    }
    for (int i = 0; i < 6; ++i) {
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += B[i + 6 * k] * M[j + 6 * k];
            t[j] = s;
        }
        for (int j = 0; j < 6; ++j) B[i + 6 * j] = t[j];
    }
}

__device__ __forceinline__ void bd_identity(double* M) {
    for (int m = 0; m < 36; ++m) M[m] = 0.0;
    for (int m = 0; m < 6; ++m) M[7 * m] = 1.0;
}

/* drift: x' and y' enter the path-length terms */
__device__ __forceinline__ void bd_drift(P6& r, double L, double* B) {
    const double p_norm = 1.0 / (1.0 + r.dp);
    const double xpr = r.px * p_norm;
    const double ypr = r.py * p_norm;
    const double NormL = L * p_norm;
    double M[36];
    bd_identity(M);
    M[6] = NormL;
    M[20] = NormL;
    M[24] = -NormL * xpr;
    M[26] = -NormL * ypr;
    M[11] = NormL * xpr;
    M[23] = NormL * ypr;
    M[29] = -NormL * (xpr * xpr + ypr * ypr);
    bd_sandwich(M, B);
    r.x += NormL * r.px;
    r.y += NormL * r.py;
    r.ct += NormL * p_norm * (r.px * r.px + r.py * r.py) / 2.0;
}

/* the symplectic part of a thin kick: field gradients at the particle */
template <bool BEND>
__device__ __forceinline__ void bd_kick_m(const P6& r, const double* A, const double* Bp, int n,
                                          double L, double irho, double* B) {
    double im = n * A[n], rn = n * Bp[n];
    for (int k = n - 1; k > 0; --k) {
        const double t = (rn * r.x - im * r.y) + k * Bp[k];
        im = im * r.x + rn * r.y + k * A[k];
        rn = t;
    }
    double M[36];
    bd_identity(M);
    M[1] = -L * rn;
    M[13] = L * im;
    M[3] = L * im;
    M[15] = L * rn;
    if (BEND) {
        M[25] = L * irho;
        M[1] += -L * irho * irho;
        M[5] = L * irho;
    }
    bd_sandwich(M, B);
}

/* the kick's diffusion: B3P = B2P^(3/2) along the particle direction */
__device__ __forceinline__ void bd_kick_b(const P6& r, double diffc, double b2p, double factor,
                                          double* B) {
    const double p_norm = 1.0 / (1.0 + r.dp);
    const double p_norm2 = p_norm * p_norm;
    const double b3p = b2p * sqrt(b2p);
    const double bb = diffc * b3p * factor / p_norm2;
    const double b11 = bb * (r.px * r.px) * p_norm2;
    const double b13 = bb * r.px * r.py * p_norm2;
    const double b33 = bb * (r.py * r.py) * p_norm2;
    const double b14 = bb * r.px * p_norm;
    const double b34 = bb * r.py * p_norm;
    B[7] += b11;
    B[19] += b13;
    B[9] += b13;
    B[21] += b33;
    B[10] += b14;
    B[25] += b14;
    B[22] += b34;
    B[27] += b34;
    B[28] += bb;
}

/* radiating thin kick with B (diff_str_kick.c:19-83, diff_bnd_kick.c:101-174) */
template <bool BEND>
__device__ __forceinline__ void bd_kick(P6& r, const double* A, const double* Bp, int n, double L,
                                        double irho, double lirho, double radc, double diffc,
                                        double* B) {
    double re, im;
    horner_dyn(A, Bp, n, r.x, r.y, re, im);
    const double p_norm = 1.0 / (1.0 + r.dp);
    const double x = r.x;
    const double xpr = r.px * p_norm;
    const double ypr = r.py * p_norm;
    double b2p, factor;
    if (BEND) {
        const double bx = im, by = re + irho;
        const double v_norm2 =
            1.0 / ((1.0 + x * irho) * (1.0 + x * irho) + xpr * xpr + ypr * ypr);
        b2p = ((by * (1 + x * irho)) * (by * (1 + x * irho)) +
               (bx * (1 + x * irho)) * (bx * (1 + x * irho)) +
               (bx * ypr - by * xpr) * (bx * ypr - by * xpr)) * v_norm2;
        factor = (1.0 + x * irho + (xpr * xpr + ypr * ypr) / 2.0) / (p_norm * p_norm) * L;
    } else {
        const double v_norm2 = 1.0 / (1.0 + xpr * xpr + ypr * ypr);
        const double bx = im, by = re;
        b2p = (by * by + bx * bx + (bx * ypr - by * xpr) * (bx * ypr - by * xpr)) * v_norm2;
        factor = (1.0 + (xpr * xpr + ypr * ypr) / 2.0) / (p_norm * p_norm) * L;
    }
    bd_kick_m<BEND>(r, A, Bp, n, L, irho, B);
    bd_kick_b(r, diffc, b2p, factor, B);
    const double dp_0 = r.dp;
    r.dp -= radc * b2p * factor;
    const double pn2 = 1.0 / (1.0 + r.dp);
    r.px = xpr / pn2;
    r.py = ypr / pn2;
    if (BEND) {
        r.px -= L * (re - (dp_0 - r.x * irho) * irho);
        r.py += L * im;
        r.ct += lirho * r.x;
    } else {
        r.px -= L * re;
        r.py += L * im;
    }
}

/* bend edge with B (diff_bend_fringe.c:1-52) */
__device__ __forceinline__ void bd_edge(P6& r, double irho, double edge, double psi, double fx,
                                        double fy_c, int method, double sgn, bool fint_pos,
                                        double* B) {
    const double p_norm = 1.0 / (1.0 + r.dp);
    double fy;
    if (method == ATB_BM_3) {
        fy = irho * tan(edge - psi + sgn * r.px * p_norm);
    } else {
        const double t = edge - psi * p_norm;
        const double tn = (t == edge) ? fy_c : irho * tan(t);
        fy = (method == ATB_BM_2) ? tn * p_norm : tn;
    }
    for (int m = 0; m < 6; ++m) {
        B[1 + 6 * m] += fx * B[6 * m];
        B[3 + 6 * m] -= fy * B[2 + 6 * m];
    }
    if (fint_pos)
        for (int m = 0; m < 6; ++m)
            B[3 + 6 * m] -= B[4 + 6 * m] * r.y * (irho * irho + fy * fy) * psi * p_norm * p_norm /
                            irho;
    for (int m = 0; m < 6; ++m) {
        B[m + 6] += fx * B[m];
        B[m + 18] -= fy * B[m + 12];
    }
    if (fint_pos)
        for (int m = 0; m < 6; ++m)
            B[m + 18] -= B[m + 24] * r.y * (irho * irho + fy * fy) * psi * p_norm * p_norm / irho;
    r.px += r.x * fx;
    r.py -= r.y * fy;
}

/* a radiating multipole with B, as the radiating multipole pass of the exact kernel */
template <bool BEND>
__device__ void bd_multipole(P6& r, const Rec& e, double diffc, double* B) {
    const uint32_t fl = e.flags();
    const double L1 = e.f(ATB_SM_L1), L2 = e.f(ATB_SM_L2);
    const double K1 = e.f(ATB_SM_K1), K2 = e.f(ATB_SM_K2);
    const double radc = e.f(ATB_SM_RADC);
    const int mo = e.mo();
    const double* A = e.p + (BEND ? ATB_BM_POLY : ATB_SM_POLY);
    const double* Bp = A + mo + 1;
    if (fl & ATB_F_SCALING) change_pref<false>(r, e.f(ATB_SM_SCALE));
    entrance_misalign(r, e);
    apertures(r, e);
    double irho = 0.0, k1i = 0.0, k2i = 0.0;
    if (BEND) {
        irho = e.f(ATB_BM_IRHO);
        k1i = e.f(ATB_BM_K1IRHO);
        k2i = e.f(ATB_BM_K2IRHO);
        bd_edge(r, irho, e.f(ATB_BM_EIN), e.f(ATB_BM_FCIN), e.f(ATB_BM_FXIN), e.f(ATB_BM_FYIN),
                (int)((fl >> ATB_F_BM_IN_SHIFT) & ATB_F_BM_MASK), 1.0, fl & ATB_F_FINT_IN, B);
    }
    if (fl & ATB_F_FQ_IN) {
        const double b1 = e.f(ATB_SM_B1);
        if (fl & ATB_F_FQ_IN_LIN) {
            const double* fm = e.blk(ATB_OPT_FRINGE);
            lin_fringe_map(r, fm);
            quad_fringe<false>(r, b1, true);
            lin_fringe_map(r, fm + 8);
        } else {
            quad_fringe<false>(r, b1, true);
        }
    }
    const int ns = e.nsteps();
    for (int m = 0; m < ns; ++m) {
        bd_drift(r, L1, B);
        bd_kick<BEND>(r, A, Bp, mo, K1, irho, k1i, radc, diffc, B);
        bd_drift(r, L2, B);
        bd_kick<BEND>(r, A, Bp, mo, K2, irho, k2i, radc, diffc, B);
        bd_drift(r, L2, B);
        bd_kick<BEND>(r, A, Bp, mo, K1, irho, k1i, radc, diffc, B);
        bd_drift(r, L1, B);
    }
    if (fl & ATB_F_FQ_OUT) {
        const double b1 = e.f(ATB_SM_B1);
        if (fl & ATB_F_FQ_OUT_LIN) {
            const double* fm = e.blk(ATB_OPT_FRINGE);
            lin_fringe_map(r, fm + 16);
            quad_fringe<false>(r, b1, false);
            lin_fringe_map(r, fm + 24);
        } else {
            quad_fringe<false>(r, b1, false);
        }
    }
    if (BEND)
        bd_edge(r, irho, e.f(ATB_BM_EOUT), e.f(ATB_BM_FCOUT), e.f(ATB_BM_FXOUT),
                e.f(ATB_BM_FYOUT), (int)((fl >> ATB_F_BM_OUT_SHIFT) & ATB_F_BM_MASK), -1.0,
                fl & ATB_F_FINT_OUT, B);
    apertures(r, e);
    exit_misalign(r, e);
    if (fl & ATB_F_SCALING) change_pref<false>(r, e.f(ATB_SM_ISCALE));
}

extern "C" __global__ void __launch_bounds__(ATB_TANGENT_THREADS)
atb_element_maps_kernel(const AtbElemMaps A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nelem) return;
    Rec e;
    e.p = A.table + A.elem_off[i];
    const uint64_t* hp = reinterpret_cast<const uint64_t*>(e.p);
    e.hdr = hp[0];
    e.opt = hp[1];
    const double* o = A.orbits + 6 * (long long)i;

    /* transfer matrix: the element on dual numbers seeded with the identity
       (their values are the exact-arithmetic exit coordinates) */
    if (A.m66 || A.exits) {
        P6T<TD> r;
        r.x = TD(o[0]); r.px = TD(o[1]); r.y = TD(o[2]);
        r.py = TD(o[3]); r.dp = TD(o[4]); r.ct = TD(o[5]);
        r.x.d[0] = 1.0; r.px.d[1] = 1.0; r.y.d[2] = 1.0;
        r.py.d[3] = 1.0; r.dp.d[4] = 1.0; r.ct.d[5] = 1.0;
        track_element(r, e, 0);
        TD* rows[6] = ATB_ROWS(r);
        if (A.m66) {
            double* m = A.m66 + 36 * (long long)i;
#pragma unroll
            for (int a = 0; a < 6; ++a) {
#pragma unroll
                for (int b = 0; b < 6; ++b) m[6 * a + b] = rows[a]->d[b];
            }
        }
        if (A.exits) {
            double* x = A.exits + 6 * (long long)i;
#pragma unroll
            for (int a = 0; a < 6; ++a) x[a] = rows[a]->v;
        }
    }
    if (!A.b66) return;
    /* diffusion matrix */
    double B[36];
    for (int k = 0; k < 36; ++k) B[k] = 0.0;
    P6 r;
    r.x = o[0]; r.px = o[1]; r.y = o[2]; r.py = o[3]; r.dp = o[4]; r.ct = o[5];
    const int op = e.op();
    if (op == ATB_OP_STRMPOLE_RAD) bd_multipole<false>(r, e, A.diff_const, B);
    else if (op == ATB_OP_BNDMPOLE_RAD) bd_multipole<true>(r, e, A.diff_const, B);
    double* b = A.b66 + 36 * (long long)i;
    for (int a = 0; a < 6; ++a)
        for (int c = 0; c < 6; ++c) b[6 * a + c] = B[a + 6 * c];
}

}  // namespace atb

#endif  // ATB_DIFFUSION_CUH
