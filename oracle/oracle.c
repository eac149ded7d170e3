/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of the reference tracking path (atcollab/at: the
 * pyat/at.c turn/element engine and the atintegrators pass methods on the
 * accelerated path), used as the checker of the CUDA engine in tests/ and as
 * the "port" CPU baseline.  It is never linked into the product.
 *
 * Every function names the reference routine it restates.  Arithmetic keeps
 * the reference's expression trees and evaluation order and is compiled with
 * -ffp-contract=off, so on the +,-,*,/ path it is bit-identical to the
 * reference C build (checked against oracle/_ref and the golden fixtures).
 * Particles are independent, so the loop runs particle-outermost (one OpenMP
 * iteration per particle through all turns); the per-particle sequence of
 * operations is the reference's element-by-element sequence.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* The arithmetic type.  The oracle proper is double; oracle_q.c includes
 * this file with ORACLE_REAL set to a wider type (and the R_* functions to
 * its math library) for finite differences whose rounding floor lies far
 * below double's.  Element data and the interface stay double. */
#ifndef ORACLE_REAL
typedef double real;
#define R_SIN sin
#define R_COS cos
#define R_TAN tan
#define R_EXP exp
#define R_POW pow
#define R_ROUND round
#define R_FABS fabs
#define R_SQRT sqrt
#else
typedef ORACLE_REAL real;
#endif

/* pass methods (must match oracle.py) */
enum {
    O_IDENTITY = 0, O_DRIFT, O_STRMPOLE, O_STRMPOLE_RAD, O_BNDMPOLE, O_BNDMPOLE_RAD,
    O_THINMPOLE, O_RFCAVITY, O_CORRECTOR, O_APERTURE, O_QUANTDIFF
};

typedef struct {
    int32_t pass;
    int32_t MaxOrder;
    int32_t NumIntSteps;
    int32_t FringeBendEntrance;
    int32_t FringeBendExit;
    int32_t FringeQuadEntrance;
    int32_t FringeQuadExit;
    int32_t Integrator;   /* 0 or 4: Forest-Ruth; 1-6: the GPU call's integrators */
    double Length, BendingAngle, EntranceAngle, ExitAngle;
    double FringeInt1, FringeInt2, FullGap, Scaling;
    double Voltage, Frequency, TimeLag, PhaseLag;
    double bax, bay;
    const double *PolynomA, *PolynomB, *fringeIntM0, *fringeIntP0;
    const double *R1, *R2, *T1, *T2, *RApertures, *EApertures, *KickAngle, *Limits;
    const double *Lmatp;
} OElem;

/* ---- constants: atintegrators/atconstants.h:16-31, pyat/at.c:52-53 ----- */
#define O_PI 3.14159265358979323846
#define O_THIRD_ROOT_2 1.25992104989487316477
static const double O_TWOPI = 2.0 * O_PI;
static const double O_DRIFT1 = 1.0 / (2.0 * (2.0 - O_THIRD_ROOT_2));
static const double O_DRIFT2 = 0.5 - (1.0 / (2.0 * (2.0 - O_THIRD_ROOT_2)));
static const double O_KICK1 = 1.0 / (2.0 - O_THIRD_ROOT_2);
static const double O_KICK2 = 1.0 - 2.0 / (2.0 - O_THIRD_ROOT_2);
static const double O_C0 = 2.99792458e8;
#define O_RE 2.8179403205e-15
#define O_E0 510.99895069e-6
static const double O_RAD_CONST = 2.0 / 3.0 * O_RE;
#define O_ROOT_3 1.7320508075688772
#define O_HBAR_C 197.3269804e-18
static const double O_DIF_CONST = 55.0 / 24.0 / O_ROOT_3 * O_HBAR_C / O_E0 * O_RE;

/* ---- small vector helpers ---------------------------------------------- */

/* atlalib.c:50-57 */
static void o_addv(real *r, const double *d) {
    for (int i = 0; i < 6; i++) r[i] += d[i];
}

/* atlalib.c:17-32: column-major 6x6 times vector, accumulated from 0 */
static void o_mulmv(real *r, const double *m) {
    real out[6];
    for (int i = 0; i < 6; i++) {
        real acc = 0;
        for (int j = 0; j < 6; j++) acc += m[i + j * 6] * r[j];
        out[i] = acc;
    }
    memcpy(r, out, sizeof(out));
}

/* atlalib.c:169-175 */
static void o_rect_ap(real *r, const double *lim) {
    if (r[0] < lim[0] || r[0] > lim[1]) r[5] = INFINITY;
    else if (r[2] < lim[2] || r[2] > lim[3]) r[5] = INFINITY;
}

/* atlalib.c:185-190 */
static void o_ellip_ap(real *r, const double *ax) {
    real u = r[0] / ax[0];
    real v = r[2] / ax[1];
    if ((u * u + v * v) >= 1) r[5] = INFINITY;
}

/* atlalib.c:70-75 */
static void o_pref(real *r, real s) {
    r[1] /= s;
    r[3] /= s;
    r[4] = (r[4] + 1.0 - s) / s;
}

/* atlalib.c:59-68 (== driftkickrad.c drift6 and diff_drift without bdiff) */
static void o_drift6(real *r, real L) {
    real pn = 1 / (1 + r[4]);
    real nl = L * pn;
    r[0] += nl * r[1];
    r[2] += nl * r[3];
    r[5] += nl * pn * (r[1] * r[1] + r[3] * r[3]) / 2;
}

/* ---- Ohmi diffusion matrix (the bdiff branch of the Rad passes) ---------
 * B is 6x6 column-major, [i][j] at i + 6 j, as in the reference. */

/* atlalib.c:92-147 ATmultmm then the row pass of ATsandwichmmt: B <- M B M' */
static void o_sandwich(const real *M, real *B) {
    real col[6], row[6];
    for (int i = 0; i < 6; i++) {
        for (int j = 0; j < 6; j++) {
            col[j] = 0;
            for (int k = 0; k < 6; k++) col[j] += M[j + 6 * k] * B[k + 6 * i];
        }
        for (int j = 0; j < 6; j++) B[j + 6 * i] = col[j];
    }
    for (int i = 0; i < 6; i++) {
        for (int j = 0; j < 6; j++) {
            row[j] = 0;
            for (int k = 0; k < 6; k++) row[j] += B[i + 6 * k] * M[j + 6 * k];
        }
        for (int j = 0; j < 6; j++) B[i + 6 * j] = row[j];
    }
}

static void o_ident(real *M) {
    for (int m = 0; m < 36; m++) M[m] = 0.0;
    for (int m = 0; m < 6; m++) M[m * 7] = 1.0;
}

/* diff_drift.c:1-28 drift_propagateB */
static void o_drift_b(real nl, real xp, real yp, real *bd) {
    real M[36];
    o_ident(M);
    M[6] = nl;
    M[20] = nl;
    M[24] = -nl * xp;
    M[26] = -nl * yp;
    M[11] = nl * xp;
    M[23] = nl * yp;
    M[29] = -nl * (xp * xp + yp * yp);
    o_sandwich(M, bd);
}

/* diff_thinkick.c:1-33 and diff_bnd_kick.c:1-47 thinkickM (bend = 0: the
 * straight form, without the curvature terms) */
static void o_thinkick_m(const real *r, const real *A, const real *B, int n, real L, real h,
                         int bend, real *bd) {
    real M[36];
    real in = n * A[n], rn = n * B[n];
    for (int k = n - 1; k > 0; k--) {
        real t = (rn * r[0] - in * r[2]) + k * B[k];
        in = in * r[0] + rn * r[2] + k * A[k];
        rn = t;
    }
    o_ident(M);
    M[1] = -L * rn;
    M[13] = L * in;
    M[3] = L * in;
    M[15] = L * rn;
    if (bend) {
        M[25] = L * h;
        M[1] += -L * h * h;
        M[5] = L * h;
    }
    o_sandwich(M, bd);
}

/* diff_thinkick.c:35-70 thinkickB */
static void o_thinkick_b(const real *r, real diffc, real b2p, real factor, real *bd) {
    real pn = 1.0 / (1.0 + r[4]);
    real pn2 = pn * pn;
    real b3p = b2p * R_SQRT(b2p);
    real bb = diffc * b3p * factor / pn2;
    real b11 = bb * (r[1] * r[1]) * pn2;
    real b13 = bb * r[1] * r[3] * pn2;
    real b33 = bb * (r[3] * r[3]) * pn2;
    real b14 = bb * r[1] * pn;
    real b34 = bb * r[3] * pn;
    bd[7] += b11;
    bd[19] += b13;
    bd[9] += b13;
    bd[21] += b33;
    bd[10] += b14;
    bd[25] += b14;
    bd[22] += b34;
    bd[27] += b34;
    bd[28] += bb;
}

/* diff_drift.c:30-43 (its literal constants are 1.0 and 2.0) */
static void o_ddrift(real *r, real L, real *bd) {
    real pn = 1.0 / (1.0 + r[4]);
    real nl = L * pn;
    if (bd) o_drift_b(nl, r[1] * pn, r[3] * pn, bd);
    r[0] += nl * r[1];
    r[2] += nl * r[3];
    r[5] += nl * pn * (r[1] * r[1] + r[3] * r[3]) / 2.0;
}

/* driftkick.c:37-48 */
static void o_fastdrift(real *r, real nl) {
    r[0] += nl * r[1];
    r[2] += nl * r[3];
    r[5] += nl * (r[1] * r[1] + r[3] * r[3]) / (2 * (1 + r[4]));
}

/* the multipole field, highest order first (driftkick.c:92-115 et al.) */
static void o_field(const real *r, const real *A, const real *B, int n,
                    real *re, real *im) {
    real a = B[n], b = A[n];
    for (int k = n - 1; k >= 0; k--) {
        real t = a * r[0] - b * r[2] + B[k];
        b = b * r[0] + a * r[2] + A[k];
        a = t;
    }
    *re = a;
    *im = b;
}

/* driftkick.c:92-115 strthinkick */
static void o_strkick(real *r, const real *A, const real *B, real L, int n) {
    real re, im;
    o_field(r, A, B, n, &re, &im);
    r[1] -= L * re;
    r[3] += L * im;
}

/* driftkick.c:51-89 bndthinkick */
static void o_bndkick(real *r, const real *A, const real *B, real L, real h, int n) {
    real re, im;
    o_field(r, A, B, n, &re, &im);
    r[1] -= L * (re - (r[4] - r[0] * h) * h);
    r[3] += L * im;
    r[5] += L * h * r[0];
}

/* diff_str_kick.c:19-83 (bdiff == NULL) */
static void o_strkick_rad(real *r, const real *A, const real *B, int n, real L,
                          real radc, real diffc, real *bd) {
    real re, im;
    o_field(r, A, B, n, &re, &im);
    real pn = 1.0 / (1.0 + r[4]);
    real xp = r[1] * pn, yp = r[3] * pn;
    real bx = im, by = re;
    real vn = 1.0 / (1.0 + xp * xp + yp * yp);
    real b2 = (by * by + bx * bx + (bx * yp - by * xp) * (bx * yp - by * xp)) * vn;
    real f = (1.0 + (xp * xp + yp * yp) / 2.0) / (pn * pn) * L;
    if (bd) {
        o_thinkick_m(r, A, B, n, L, 0.0, 0, bd);
        o_thinkick_b(r, diffc, b2, f, bd);
    }
    r[4] -= radc * b2 * f;
    pn = 1.0 / (1.0 + r[4]);
    r[1] = xp / pn;
    r[3] = yp / pn;
    r[1] -= L * re;
    r[3] += L * im;
}

/* diff_bnd_kick.c:101-174 with its B2perp (:85-99), bdiff == NULL */
static void o_bndkick_rad(real *r, const real *A, const real *B, int n, real L,
                          real h, real radc, real diffc, real *bd) {
    real re, im;
    o_field(r, A, B, n, &re, &im);
    real pn = 1.0 / (1.0 + r[4]);
    real x = r[0];
    real xp = r[1] * pn, yp = r[3] * pn;
    real bx = im, by = re + h;
    real vn = 1.0 / ((1.0 + x * h) * (1.0 + x * h) + xp * xp + yp * yp);
    real b2 = ((by * (1 + x * h)) * (by * (1 + x * h)) + (bx * (1 + x * h)) * (bx * (1 + x * h)) +
                 (bx * yp - by * xp) * (bx * yp - by * xp)) * vn;
    real f = (1.0 + x * h + (xp * xp + yp * yp) / 2.0) / (pn * pn) * L;
    if (bd) {
        o_thinkick_m(r, A, B, n, L, h, 1, bd);
        o_thinkick_b(r, diffc, b2, f, bd);
    }
    real d0 = r[4];
    r[4] -= radc * b2 * f;
    pn = 1.0 / (1.0 + r[4]);
    r[1] = xp / pn;
    r[3] = yp / pn;
    r[1] -= L * (re - (d0 - r[0] * h) * h);
    r[3] += L * im;
    r[5] += L * h * r[0];
}

/* quadfringe.c:3-51: sgn = +1 (QuadFringePassP) or -1 (QuadFringePassN) */
static void o_quad_fringe(real *r, real b2, int sgn) {
    real u = b2 / (12.0 * (1.0 + r[4]));
    real x2 = r[0] * r[0], z2 = r[2] * r[2], xz = r[0] * r[2];
    real gx = u * (x2 + 3 * z2) * r[0];
    real gz = u * (z2 + 3 * x2) * r[2];
    real t1 = 3 * u * (2 * xz * r[3] - (x2 + z2) * r[1]);
    real t3 = 3 * u * (2 * xz * r[1] - (x2 + z2) * r[3]);
    real dc = (gz * r[3] - gx * r[1]) / (1 + r[4]);
    if (sgn > 0) {
        r[0] += gx; r[2] -= gz; r[5] -= dc; r[1] += t1; r[3] -= t3;
    } else {
        r[0] -= gx; r[2] += gz; r[5] += dc; r[1] -= t1; r[3] += t3;
    }
}

/* quadfringe.c: quadPartialFringeMatrix, 2x2 blocks (m[0..3] x, m[4..7] y) */
static void o_fringe_matrix(real K1, const double *fi, int part, real *m) {
    real in = 1.0, k2 = K1 * K1, j1x, j2x, j3x, j1y, j2y, j3y;
    if (part == 1) {
        j1x = in * (K1 * fi[1] - 2 * k2 * fi[3] / 3. - k2 * fi[0] * fi[2] / 2);
        j2x = in * K1 * fi[2];
        j3x = in * k2 * (fi[2] + fi[4] + fi[0] * fi[1]);
        j1y = in * (-K1 * fi[1] - 2 * k2 * fi[3] / 3. - k2 * fi[0] * fi[2] / 2);
    } else {
        j1x = in * (K1 * fi[1] + k2 * fi[0] * fi[2] / 2);
        j2x = in * K1 * fi[2];
        j3x = in * k2 * (fi[4] - fi[0] * fi[1]);
        j1y = in * (-K1 * fi[1] + k2 * fi[0] * fi[2] / 2);
    }
    j2y = -j2x;
    j3y = j3x;
    real ex = R_EXP(j1x), ey = R_EXP(j1y);
    m[0] = ex; m[1] = j2x / ex; m[2] = ex * j3x; m[3] = (1 + j2x * j3x) / ex;
    m[4] = ey; m[5] = j2y / ey; m[6] = ey * j3y; m[7] = (1 + j2y * j3y) / ey;
}

static void o_apply22(real *r, const real *m) {
    real x = r[0], px = r[1], y = r[2], py = r[3];
    r[0] = m[0] * x + m[1] * px;
    r[1] = m[2] * x + m[3] * px;
    r[2] = m[4] * y + m[5] * py;
    r[3] = m[6] * y + m[7] * py;
}

/* quadfringe.c:45-112 linearQuadFringeElegantEntrance/Exit */
static void o_lin_fringe(real *r, real b2, const double *fm, const double *fp, int entrance) {
    real m[8], s;
    if (entrance) {
        o_fringe_matrix(b2, fp, 2, m);
        s = m[0]; m[0] = m[3]; m[3] = s;
        s = m[4]; m[4] = m[7]; m[7] = s;
        o_apply22(r, m);
        o_quad_fringe(r, b2, +1);
        o_fringe_matrix(b2, fm, 1, m);
        s = m[0]; m[0] = m[3]; m[3] = s;
        s = m[4]; m[4] = m[7]; m[7] = s;
        o_apply22(r, m);
    } else {
        o_fringe_matrix(b2, fm, 1, m);
        o_apply22(r, m);
        o_quad_fringe(r, b2, -1);
        o_fringe_matrix(b2, fp, 2, m);
        o_apply22(r, m);
    }
}

/* atphyslib.c:15-79 edge_fringe_entrance/exit; sgn +1 entrance, -1 exit */
static void o_edge(real *r, real h, real edge, real fint, real gap, int method,
                   int sgn) {
    real fc = 0.0, fy;
    if (!((fint == 0.0) || (gap == 0.0) || (method == 0))) {
        real se = R_SIN(edge), ce = R_COS(edge);
        fc = h * gap * fint * (1 + se * se) / ce;
    }
    real fx = h * R_TAN(edge);
    if (method == 2)
        fy = h * R_TAN(edge - fc / (1 + r[4])) / (1 + r[4]);
    else if (method == 3)
        fy = (sgn > 0) ? h * R_TAN(edge - fc + r[1] / (1 + r[4]))
                       : h * R_TAN(edge - fc - r[1] / (1 + r[4]));
    else
        fy = h * R_TAN(edge - fc / (1 + r[4]));
    r[1] += r[0] * fx;
    r[3] -= r[2] * fy;
}

/* diff_bend_fringe.c:1-52 (bdiff == NULL) */
static void o_edge_rad(real *r, real h, real edge, real fint, real gap, int method,
                       real sgn, real *bd) {
    real pn = 1.0 / (1.0 + r[4]);
    real psi = 0.0, fy;
    if (!((fint == 0.0) || (gap == 0.0) || (method == 0))) {
        real se = R_SIN(edge), ce = R_COS(edge);
        psi = h * gap * fint * (1.0 + se * se) / ce;
    }
    real fx = h * R_TAN(edge);
    if (method == 2)
        fy = h * R_TAN(edge - psi * pn) * pn;
    else if (method == 3)
        fy = h * R_TAN(edge - psi + sgn * r[1] * pn);
    else
        fy = h * R_TAN(edge - psi * pn);
    /* diff_bend_fringe.c:31-46: B propagated through the edge map */
    if (bd) {
        int ff = (fint > 0 && gap > 0);
        for (int m = 0; m < 6; m++) {
            bd[1 + 6 * m] += fx * bd[6 * m];
            bd[3 + 6 * m] -= fy * bd[2 + 6 * m];
        }
        if (ff)
            for (int m = 0; m < 6; m++)
                bd[3 + 6 * m] -= bd[4 + 6 * m] * r[2] * (h * h + fy * fy) * psi * pn * pn / h;
        for (int m = 0; m < 6; m++) {
            bd[m + 6 * 1] += fx * bd[m + 6 * 0];
            bd[m + 6 * 3] -= fy * bd[m + 6 * 2];
        }
        if (ff)
            for (int m = 0; m < 6; m++)
                bd[m + 6 * 3] -= bd[m + 6 * 4] * r[2] * (h * h + fy * fy) * psi * pn * pn / h;
    }
    r[1] += r[0] * fx;
    r[3] -= r[2] * fy;
}

/* ---- pass methods -------------------------------------------------------- */

static double o_gamma(double energy, double rest) {
    /* atelem.c:364-371 */
    return (rest == 0.0) ? 1.0E-9 * energy / O_E0 : energy / rest;
}

/* The symplectic integrators of the reference GPU backend's gpupass
 * (atgpu/SymplecticIntegrator.cpp:28-80): per step SL, stages of a drift
 * SL*c[i] and a kick SL*d[i].  Euler; McLachlan-Atela optimal 2nd order;
 * Ruth 3rd order; Forest-Ruth 4th order; McLachlan-Atela optimal 4th order;
 * Yoshida 6th order (solution A).  Returns the number of stages. */
static int o_integ(int id, double *c, double *d) {
    static const double mc5[4] = {0.1288461583653843, 0.4415830236164665,
                                  -0.0857820194129737, 0.5153528374311229};
    static const double md5[4] = {0.3340036032863214, 0.7563200005156683,
                                  -0.2248198030794208, 0.1344961992774311};
    static const double yc6[8] = {0.3922568052387800, 0.5100434119184585, -0.4710533854097566,
                                  0.0687531682525181, 0.0687531682525181, -0.4710533854097566,
                                  0.5100434119184585, 0.3922568052387800};
    static const double yd6[8] = {0.7845136104775600, 0.2355732133593570, -1.1776799841788701,
                                  1.3151863206839063, -1.1776799841788701, 0.2355732133593570,
                                  0.7845136104775600, 0.0};
    switch (id) {
        case 1:
            c[0] = 1.0; d[0] = 1.0;
            return 1;
        case 2:
            c[0] = d[0] = 1.0 - 1.0 / sqrt(2.0);
            c[1] = d[1] = 1.0 / sqrt(2.0);
            return 2;
        case 3:
            c[0] = 1.0; c[1] = -2.0 / 3.0; c[2] = 2.0 / 3.0;
            d[0] = -1.0 / 24.0; d[1] = 3.0 / 4.0; d[2] = 7.0 / 24.0;
            return 3;
        case 5:
            for (int i = 0; i < 4; i++) { c[i] = mc5[i]; d[i] = md5[i]; }
            return 4;
        case 6:
            for (int i = 0; i < 8; i++) { c[i] = yc6[i]; d[i] = yd6[i]; }
            return 8;
        default:
            c[0] = O_DRIFT1; c[1] = O_DRIFT2; c[2] = O_DRIFT2; c[3] = O_DRIFT1;
            d[0] = O_KICK1; d[1] = O_KICK2; d[2] = O_KICK1; d[3] = 0.0;
            return 4;
    }
}

/* the coefficient table of integrator ``id`` (for the tests) */
int oracle_integ(int id, double *c, double *d) { return o_integ(id, c, d); }

/* StrMPole/BndMPole (Rad) Symplectic4: StrMPoleSymplectic4Pass.c:29-109,
 * BndMPoleSymplectic4Pass.c:38-129, StrMPoleSymplectic4RadPass.c:30-115,
 * BndMPoleSymplectic4RadPass.c:39-128 */
static void o_multipole(real *r, const OElem *e, const real *A, const real *B, int bend,
                        int rad, real radc, real diffc, real *bd) {
    real le = e->Length;
    real SL = le / e->NumIntSteps;
    real L1 = SL * O_DRIFT1, L2 = SL * O_DRIFT2, K1 = SL * O_KICK1, K2 = SL * O_KICK2;
    int n = e->MaxOrder;
    real h = bend ? e->BendingAngle / e->Length : 0.0;
    int lin_in = (e->fringeIntM0 && e->fringeIntP0 && e->FringeQuadEntrance == 2);
    int lin_out = (e->fringeIntM0 && e->fringeIntP0 && e->FringeQuadExit == 2);
    real s = e->Scaling;
    real nl1 = 0, nl2 = 0, pn = 0;
    if (s != 1.0) o_pref(r, s);
    if (!rad) {
        pn = 1.0 / (1.0 + r[4]);
        nl1 = L1 * pn;
        nl2 = L2 * pn;
    }
    if (e->T1) o_addv(r, e->T1);
    if (e->R1) o_mulmv(r, e->R1);
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    if (bend) {
        if (rad) o_edge_rad(r, h, e->EntranceAngle, e->FringeInt1, e->FullGap, e->FringeBendEntrance, 1.0, bd);
        else o_edge(r, h, e->EntranceAngle, e->FringeInt1, e->FullGap, e->FringeBendEntrance, 1);
    }
    if (e->FringeQuadEntrance && B[1] != 0) {
        if (lin_in) o_lin_fringe(r, B[1], e->fringeIntM0, e->fringeIntP0, 1);
        else o_quad_fringe(r, B[1], +1);
    }
    if (e->Integrator > 0 && e->Integrator != 4) {
        double c[8], d[8];
        const int ni = o_integ(e->Integrator, c, d);
        for (int m = 0; m < e->NumIntSteps; m++) {
            for (int i = 0; i < ni; i++) {
                if (c[i] != 0.0) {
                    real ld = SL * c[i];
                    if (rad) o_ddrift(r, ld, bd); else o_fastdrift(r, ld * pn);
                }
                if (d[i] != 0.0) {
                    real lk = SL * d[i];
                    if (rad) {
                        if (bend) o_bndkick_rad(r, A, B, n, lk, h, radc, diffc, bd);
                        else o_strkick_rad(r, A, B, n, lk, radc, diffc, bd);
                    } else {
                        if (bend) o_bndkick(r, A, B, lk, h, n); else o_strkick(r, A, B, lk, n);
                    }
                }
            }
        }
    }
    for (int m = 0; m < e->NumIntSteps && !(e->Integrator > 0 && e->Integrator != 4); m++) {
        if (rad) {
            o_ddrift(r, L1, bd);
            if (bend) o_bndkick_rad(r, A, B, n, K1, h, radc, diffc, bd);
            else o_strkick_rad(r, A, B, n, K1, radc, diffc, bd);
            o_ddrift(r, L2, bd);
            if (bend) o_bndkick_rad(r, A, B, n, K2, h, radc, diffc, bd);
            else o_strkick_rad(r, A, B, n, K2, radc, diffc, bd);
            o_ddrift(r, L2, bd);
            if (bend) o_bndkick_rad(r, A, B, n, K1, h, radc, diffc, bd);
            else o_strkick_rad(r, A, B, n, K1, radc, diffc, bd);
            o_ddrift(r, L1, bd);
        } else {
            o_fastdrift(r, nl1);
            if (bend) o_bndkick(r, A, B, K1, h, n); else o_strkick(r, A, B, K1, n);
            o_fastdrift(r, nl2);
            if (bend) o_bndkick(r, A, B, K2, h, n); else o_strkick(r, A, B, K2, n);
            o_fastdrift(r, nl2);
            if (bend) o_bndkick(r, A, B, K1, h, n); else o_strkick(r, A, B, K1, n);
            o_fastdrift(r, nl1);
        }
    }
    if (e->FringeQuadExit && B[1] != 0) {
        if (lin_out) o_lin_fringe(r, B[1], e->fringeIntM0, e->fringeIntP0, 0);
        else o_quad_fringe(r, B[1], -1);
    }
    if (bend) {
        if (rad) o_edge_rad(r, h, e->ExitAngle, e->FringeInt2, e->FullGap, e->FringeBendExit, -1.0, bd);
        else o_edge(r, h, e->ExitAngle, e->FringeInt2, e->FullGap, e->FringeBendExit, -1);
    }
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    if (e->R2) o_mulmv(r, e->R2);
    if (e->T2) o_addv(r, e->T2);
    if (s != 1.0) o_pref(r, 1.0 / s);
}

/* ThinMPolePass.c:28-70 */
static void o_thin(real *r, const OElem *e, const real *A, const real *B) {
    real s = e->Scaling;
    if (s != 1.0) o_pref(r, s);
    if (e->T1) o_addv(r, e->T1);
    if (e->R1) o_mulmv(r, e->R1);
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    o_strkick(r, A, B, 1.0, e->MaxOrder);
    r[1] += e->bax * r[4];
    r[3] -= e->bay * r[4];
    r[5] -= e->bax * r[0] - e->bay * r[2];
    if (e->R2) o_mulmv(r, e->R2);
    if (e->T2) o_addv(r, e->T2);
    if (s != 1.0) o_pref(r, 1.0 / s);
}

/* attrackfunc.c:5-42 trackRFCavity, via RFCavityPass.c:359-392 */
static void o_rf(real *r, const OElem *e, real nv, real hn, int nturn, real T0) {
    real le = e->Length, f = e->Frequency, lag = e->TimeLag, phi = e->PhaseLag;
    if (le == 0) {
        if (nv != 0)
            r[4] += -nv * R_SIN(O_TWOPI * f * ((r[5] - lag) / O_C0 - (hn / f - T0) * nturn) - phi);
    } else {
        real half = le / 2;
        o_drift6(r, half);
        if (nv != 0.0)
            r[4] += -nv * R_SIN(O_TWOPI * f * ((r[5] - lag) / O_C0 - (hn / f - T0) * nturn) - phi);
        o_drift6(r, half);
    }
}

/* CorrectorPass.c:25-90 */
static void o_corr(real *r, const OElem *e) {
    real xk = e->KickAngle[0], yk = e->KickAngle[1], le = e->Length, s = e->Scaling;
    if (s != 1.0) o_pref(r, s);
    if (le == 0.0) {
        if (e->T1) o_addv(r, e->T1);
        if (e->R1) o_mulmv(r, e->R1);
        if (e->RApertures) o_rect_ap(r, e->RApertures);
        if (e->EApertures) o_ellip_ap(r, e->EApertures);
        r[1] += xk;
        r[3] += yk;
    } else {
        real pn = 1.0 / (1.0 + r[4]);
        real nl = le * pn;
        if (e->T1) o_addv(r, e->T1);
        if (e->R1) o_mulmv(r, e->R1);
        if (e->RApertures) o_rect_ap(r, e->RApertures);
        if (e->EApertures) o_ellip_ap(r, e->EApertures);
        r[5] += nl * pn * (xk * xk / 3 + yk * yk / 3 + r[1] * r[1] + r[3] * r[3] + r[1] * xk + r[3] * yk) / 2;
        r[0] += nl * (r[1] + xk / 2);
        r[1] += xk;
        r[2] += nl * (r[3] + yk / 2);
        r[3] += yk;
        if (e->RApertures) o_rect_ap(r, e->RApertures);
        if (e->EApertures) o_ellip_ap(r, e->EApertures);
    }
    if (e->R2) o_mulmv(r, e->R2);
    if (e->T2) o_addv(r, e->T2);
    if (s != 1.0) o_pref(r, 1.0 / s);
}

/* DriftPass.c:16-48 */
static void o_driftpass(real *r, const OElem *e) {
    if (e->T1) o_addv(r, e->T1);
    if (e->R1) o_mulmv(r, e->R1);
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    o_drift6(r, e->Length);
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    if (e->R2) o_mulmv(r, e->R2);
    if (e->T2) o_addv(r, e->T2);
}

/* IdentityPass.c:20-43 */
static void o_identity(real *r, const OElem *e) {
    if (e->T1) o_addv(r, e->T1);
    if (e->R1) o_mulmv(r, e->R1);
    if (e->RApertures) o_rect_ap(r, e->RApertures);
    if (e->EApertures) o_ellip_ap(r, e->EApertures);
    if (e->R2) o_mulmv(r, e->R2);
    if (e->T2) o_addv(r, e->T2);
}

/* Per-element constants the reference derives once per call or per cached
 * element: KickAngle folded into the dipole terms (the reference writes it
 * into the coefficient arrays and restores them afterwards), the RF harmonic
 * number round(F*T0) and the normalised voltage. */
typedef struct {
    real A[64], B[64];
    real nv, hn, radc, diffc;
} OPrep;

static void o_prepare(const OElem *e, OPrep *p, double energy, double rest, double T0) {
    int n = e->MaxOrder;
    if (e->pass == O_STRMPOLE || e->pass == O_STRMPOLE_RAD || e->pass == O_BNDMPOLE ||
        e->pass == O_BNDMPOLE_RAD || e->pass == O_THINMPOLE) {
        for (int k = 0; k <= n && k < 64; k++) {
            p->A[k] = e->PolynomA[k];
            p->B[k] = e->PolynomB[k];
        }
        if (e->KickAngle) {
            if (e->pass == O_THINMPOLE) {
                p->B[0] -= e->KickAngle[0];
                p->A[0] += e->KickAngle[1];
            } else {
                p->B[0] -= R_SIN(e->KickAngle[0]) / e->Length;
                p->A[0] += R_SIN(e->KickAngle[1]) / e->Length;
            }
        }
    }
    if (e->pass == O_STRMPOLE_RAD || e->pass == O_BNDMPOLE_RAD) {
        p->radc = O_RAD_CONST * R_POW(o_gamma(energy, rest), 3);
        p->diffc = O_DIF_CONST * R_POW(o_gamma(energy, rest), 5);
    }
    if (e->pass == O_RFCAVITY) {
        p->hn = R_ROUND(e->Frequency * T0);
        p->nv = e->Voltage / energy;
    }
}

static void o_element(real *r, const OElem *e, const OPrep *p, int nturn, double T0) {
    if (isnan(r[0])) return;
    switch (e->pass) {
        case O_IDENTITY: o_identity(r, e); break;
        case O_DRIFT: o_driftpass(r, e); break;
        case O_STRMPOLE: o_multipole(r, e, p->A, p->B, 0, 0, 0.0, 0.0, NULL); break;
        case O_STRMPOLE_RAD: o_multipole(r, e, p->A, p->B, 0, 1, p->radc, 0.0, NULL); break;
        case O_BNDMPOLE: o_multipole(r, e, p->A, p->B, 1, 0, 0.0, 0.0, NULL); break;
        case O_BNDMPOLE_RAD: o_multipole(r, e, p->A, p->B, 1, 1, p->radc, 0.0, NULL); break;
        case O_THINMPOLE: o_thin(r, e, p->A, p->B); break;
        case O_RFCAVITY: o_rf(r, e, p->nv, p->hn, nturn, T0); break;
        case O_CORRECTOR: o_corr(r, e); break;
        case O_APERTURE: o_rect_ap(r, e->Limits); break;
        case O_QUANTDIFF: break;   /* needs the random stream: element-major engine */
        default: break;
    }
}

/* pyat/at.c:123 */
static int o_bad(const real *r) {
    for (int k = 0; k < 6; k++)
        if (!isfinite(r[k]) || (R_FABS(r[k]) > 1 && k < 5)) return 1;
    return 0;
}

static void o_put6(double *dst, const real *src) {
    for (int k = 0; k < 6; k++) dst[k] = (double)src[k];
}

/* The engine of pyat/at.c:596-654 for one particle; returns 0. */
static void o_particle(real *r, const OElem *el, const OPrep *pp, int nelem, int nturns,
                       int turn0, int start, int end, const uint32_t *refs, int nref,
                       int losses, int check, double T0, double *rout, int64_t np, int64_t p,
                       uint8_t *lost, uint32_t *lturn, uint32_t *lelem, double *lcoord) {
    int64_t slot = 0;
    int is_lost = losses ? (lost[p] != 0) : 0;
    for (int t = 0; t < nturns; t++) {
        int nturn = turn0 + t;
        int s0 = (t == 0) ? start : 0;
        int ri = 0;
        uint32_t next = (ri < nref) ? refs[ri++] : 0x7fffffffu;
        for (int i = s0; i < end; i++) {
            if ((uint32_t)i == next) {
                if (rout) o_put6(rout + 6 * (p + np * slot), r);
                slot++;
                next = (ri < nref) ? refs[ri++] : 0x7fffffffu;
            }
            o_element(r, &el[i], &pp[i], nturn, T0);
            if (!check) continue;
            if (losses) {
                if (!is_lost && o_bad(r)) {
                    is_lost = 1;
                    lturn[p] = (uint32_t)nturn;
                    lelem[p] = (uint32_t)i;
                    o_put6(lcoord + 6 * p, r);
                    r[0] = NAN; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = 0; r[5] = 0;
                }
            } else if (isfinite(r[0]) && o_bad(r)) {
                r[0] = NAN; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = 0; r[5] = 0;
            }
        }
        if ((uint32_t)nelem == next) {
            if (rout) o_put6(rout + 6 * (p + np * slot), r);
            slot++;
        }
    }
    if (losses) lost[p] = (uint8_t)is_lost;
}

/* ---- the random stream of QuantDiffPass ---------------------------------
 * atintegrators/atrandom.c: O'Neill's PCG32 (XSH-RR output of a 64-bit LCG
 * with stream increment) and normals by Marsaglia's polar method, one spare
 * value kept for the next call; the stream is the engine's thread_state,
 * seeded like pyat/at.c:833-852 reset_rng. */
typedef struct {
    uint64_t state, inc;
    double spare;
    int has_spare;
} ORng;

static uint32_t o_pcg32(ORng *g) {
    uint64_t old = g->state;
    g->state = old * 6364136223846793005ULL + g->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

void oracle_rng_seed(ORng *g, uint64_t initstate, uint64_t initseq) {
    g->state = 0U;
    g->inc = (initseq << 1u) | 1u;
    o_pcg32(g);
    g->state += initstate;
    o_pcg32(g);
    g->has_spare = 0;
}

static double o_randn(ORng *g) {
    if (g->has_spare) {
        g->has_spare = 0;
        return 0.0 + 1.0 * g->spare;
    }
    g->has_spare = 1;
    double u, v, s;
    do {
        u = 2.0 * ldexp(o_pcg32(g), -32) - 1.0;
        v = 2.0 * ldexp(o_pcg32(g), -32) - 1.0;
        s = u * u + v * v;
    } while ((s >= 1.0) || (s == 0.0));
    s = sqrt(-2.0 * log(s) / s);
    g->spare = v * s;
    return 0.0 + 1.0 * u * s;
}

/* QuantDiffPass.c:9-45: six normals per particle (drawn for lost ones too),
 * r += L z with L lower triangular, column-major */
static void o_quantdiff(real *r, const double *L, ORng *g) {
    double z[6];
    real d[6];
    for (int i = 0; i < 6; i++) {
        d[i] = 0.0;
        z[i] = o_randn(g);
    }
    for (int i = 0; i < 6; i++)
        for (int j = 0; j <= i; j++) d[i] += z[j] * L[i + 6 * j];
    if (!isnan(r[0]))
        for (int i = 0; i < 6; i++) r[i] += d[i];
}

static OPrep *o_prepare_all(const OElem *el, int nelem, double energy, double rest, double T0) {
    OPrep *pp = (OPrep *)calloc((size_t)(nelem > 0 ? nelem : 1), sizeof(OPrep));
    if (!pp) return NULL;
    for (int i = 0; i < nelem; i++) o_prepare(&el[i], &pp[i], energy, rest, T0);
    return pp;
}

/* The engine in the reference's own order (element-major: every particle
 * through element i before element i + 1), single-threaded, for lattices
 * whose QuantDiffPass elements draw from the sequential random stream. */
static void o_track_em(real *R, const OElem *el, const OPrep *pp, int nelem, int nturns,
                       int turn0, int start, int end, const uint32_t *refs, int nref,
                       int losses, int check, double T0, double *rout, int64_t np,
                       uint8_t *lost, uint32_t *lturn, uint32_t *lelem, double *lcoord,
                       ORng *g) {
    int64_t slot = 0;
    for (int t = 0; t < nturns; t++) {
        int nturn = turn0 + t;
        int s0 = (t == 0) ? start : 0;
        int ri = 0;
        uint32_t next = (ri < nref) ? refs[ri++] : 0x7fffffffu;
        for (int i = s0; i < end; i++) {
            if ((uint32_t)i == next) {
                if (rout)
                    for (int64_t p = 0; p < np; p++) o_put6(rout + 6 * (p + np * slot), R + 6 * p);
                slot++;
                next = (ri < nref) ? refs[ri++] : 0x7fffffffu;
            }
            for (int64_t p = 0; p < np; p++) {
                real *r = R + 6 * p;
                if (el[i].pass == O_QUANTDIFF) o_quantdiff(r, el[i].Lmatp, g);
                else o_element(r, &el[i], &pp[i], nturn, T0);
                if (!check) continue;
                if (losses) {
                    if (!lost[p] && o_bad(r)) {
                        lost[p] = 1;
                        lturn[p] = (uint32_t)nturn;
                        lelem[p] = (uint32_t)i;
                        o_put6(lcoord + 6 * p, r);
                        r[0] = NAN; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = 0; r[5] = 0;
                    }
                } else if (isfinite(r[0]) && o_bad(r)) {
                    r[0] = NAN; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = 0; r[5] = 0;
                }
            }
        }
        if ((uint32_t)nelem == next) {
            if (rout)
                for (int64_t p = 0; p < np; p++) o_put6(rout + 6 * (p + np * slot), R + 6 * p);
            slot++;
        }
    }
}

/* Track np particles (6, np Fortran order) in place.  Mirrors at_atpass.
 * ``rng`` is the random stream of QuantDiffPass elements (NULL: they are
 * skipped). */
int oracle_track(const OElem *el, int nelem, double *r, int64_t np, int nturns, int turn0,
                 int start, int end, const uint32_t *refs, int nref, int losses, int check,
                 double energy, double rest, double T0, double *rout, uint8_t *lost,
                 uint32_t *lturn, uint32_t *lelem, double *lcoord, int nthreads, ORng *rng) {
    OPrep *pp = o_prepare_all(el, nelem, energy, rest, T0);
    if (!pp) return -1;
    if (losses) {
        memset(lost, 0, (size_t)np);
        memset(lturn, 0, (size_t)np * 4);
        memset(lelem, 0, (size_t)np * 4);
        memset(lcoord, 0, (size_t)np * 48);
    }
    int has_rng = 0;
    for (int i = 0; i < nelem; i++) has_rng |= (el[i].pass == O_QUANTDIFF);
    if (has_rng && rng) {
        real *R = (real *)malloc((size_t)(np > 0 ? np : 1) * 6 * sizeof(real));
        if (!R) { free(pp); return -1; }
        for (int64_t k = 0; k < 6 * np; k++) R[k] = r[k];
        o_track_em(R, el, pp, nelem, nturns, turn0, start, end, refs, nref, losses, check, T0,
                   rout, np, lost, lturn, lelem, lcoord, rng);
        for (int64_t p = 0; p < np; p++) o_put6(r + 6 * p, R + 6 * p);
        free(R);
        free(pp);
        return 0;
    }
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t p = 0; p < np; p++) {
        real buf[6];
        for (int k = 0; k < 6; k++) buf[k] = r[6 * p + k];
        o_particle(buf, el, pp, nelem, nturns, turn0, start, end, refs, nref, losses, check,
                   T0, rout, np, p, lost, lturn, lelem, lcoord);
        o_put6(r + 6 * p, buf);
    }
    free(pp);
    return 0;
}

/* pyat/at.c:755-831 diffusion_matrix: the Ohmi diffusion matrix of one
 * element for one particle at ``orbit`` (T0 = 0, turn 0), accumulated from
 * zero by the bdiff branch of the radiating multipole passes; other pass
 * methods leave it zero.  ``out`` is 6x6 column-major ([i][j] at i + 6 j). */
int oracle_diffmatrix(const OElem *e, const double *orbit, double energy, double rest,
                      double *out) {
    OPrep pp;
    memset(&pp, 0, sizeof(pp));
    o_prepare(e, &pp, energy, rest, 0.0);
    real r[6], bd[36];
    for (int k = 0; k < 6; k++) r[k] = orbit[k];
    for (int k = 0; k < 36; k++) bd[k] = 0.0;
    if (e->pass == O_STRMPOLE_RAD)
        o_multipole(r, e, pp.A, pp.B, 0, 1, pp.radc, pp.diffc, bd);
    else if (e->pass == O_BNDMPOLE_RAD)
        o_multipole(r, e, pp.A, pp.B, 1, 1, pp.radc, pp.diffc, bd);
    for (int k = 0; k < 36; k++) out[k] = (double)bd[k];
    return 0;
}
