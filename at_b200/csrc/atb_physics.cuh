/*
 * Per-particle integrators of the accelerated pass methods, as device
 * functions over a register-resident 6-vector.
 *
 * Two arithmetic modes are compiled from this one source:
 *   FAST == false  "exact": the reference's expression trees in the
 *                  reference's evaluation order, compiled without FMA
 *                  contraction (-fmad=false), IEEE division.  On the
 *                  +,-,*,/ path this reproduces the reference C build bit for
 *                  bit; only sin/tan go through CUDA's libdevice.
 *   FAST == true   "fast": FMA contraction plus algebraic rewrites that drop
 *                  divisions where the reference recomputes the same
 *                  reciprocal (1/(1+delta) is carried through a slice, and
 *                  x/p_norm becomes x*(1+delta)).  Each rewrite changes a
 *                  result by at most a few ulp.
 *
 * Each function cites the reference routine it restates.
 */
#ifndef ATB_PHYSICS_CUH
#define ATB_PHYSICS_CUH

#include "atb_table.h"
#include "atb_dual.cuh"

namespace atb {

/* The particle state.  T is double in the tracking kernels and a dual number
 * (value + partial derivatives) in the tangent kernel; every function below
 * is a template on T so both run the same expressions. */
template <class T>
struct P6T {
    T x, px, y, py, dp, ct;
};
using P6 = P6T<double>;

#define ATB_C0 2.99792458e8

__device__ __forceinline__ double inf_d() { return __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ double nan_d() { return __longlong_as_double(0x7ff8000000000000LL); }

template <class T>
__device__ __forceinline__ bool all_finite(const P6T<T>& r) {
    return isfinite(val(r.x)) && isfinite(val(r.px)) && isfinite(val(r.y)) &&
           isfinite(val(r.py)) && isfinite(val(r.dp)) && isfinite(val(r.ct));
}

/* Fast-mode reciprocal of a positive operand near 1: the hardware estimate
 * (rcp.approx.ftz.f64) refined by two Newton-Raphson steps
 * y <- y + y(1 - d y) (Markstein's iteration; each step squares the relative
 * error), within an ulp of 1/d.  Only the "fast" kernels use it. */
__device__ __forceinline__ double rcp_nr(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

/* atlalib.c:50-57 ATaddvv */
template <class T>
__device__ __forceinline__ void add_t(P6T<T>& r, const double* t) {
    r.x += t[0]; r.px += t[1]; r.y += t[2]; r.py += t[3]; r.dp += t[4]; r.ct += t[5];
}

/* atlalib.c:17-32 ATmultmv: temp[i] = 0 + sum_j A[i+6j]*r[j], j ascending */
template <class T>
__device__ __forceinline__ void mult_dense(P6T<T>& r, const double* A) {
    const T r0 = r.x, r1 = r.px, r2 = r.y, r3 = r.py, r4 = r.dp, r5 = r.ct;
    T t[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        T s = 0.0;
        s += A[i] * r0;
        s += A[i + 6] * r1;
        s += A[i + 12] * r2;
        s += A[i + 18] * r3;
        s += A[i + 24] * r4;
        s += A[i + 30] * r5;
        t[i] = s;
    }
    r.x = t[0]; r.px = t[1]; r.y = t[2]; r.py = t[3]; r.dp = t[4]; r.ct = t[5];
}

/* ATmultmv for a matrix that only rotates the x/y planes: the dense sum with
 * its zero terms dropped, which is value-identical for finite coordinates.
 * A non-finite coordinate takes the full sum with the zero entries written
 * out, so 0*inf -> NaN propagates exactly as in the reference. */
template <class T>
__device__ __forceinline__ void mult_tilt(P6T<T>& r, const double* m) {
    const T x = r.x, px = r.px, y = r.y, py = r.py, d = r.dp, c = r.ct;
    if (!all_finite(r)) {
        const double z = 0.0;
        r.x = 0.0 + m[0] * x + z * px + m[1] * y + z * py + z * d + z * c;
        r.px = 0.0 + z * x + m[2] * px + z * y + m[3] * py + z * d + z * c;
        r.y = 0.0 + m[4] * x + z * px + m[5] * y + z * py + z * d + z * c;
        r.py = 0.0 + z * x + m[6] * px + z * y + m[7] * py + z * d + z * c;
        r.dp = 0.0 + z * x + z * px + z * y + z * py + 1.0 * d + z * c;
        r.ct = 0.0 + z * x + z * px + z * y + z * py + z * d + 1.0 * c;
        return;
    }
    r.x = m[0] * x + m[1] * y;
    r.px = m[2] * px + m[3] * py;
    r.y = m[4] * x + m[5] * y;
    r.py = m[6] * px + m[7] * py;
}

template <class T>
__device__ __forceinline__ void mult_r(P6T<T>& r, const double* blk, bool dense) {
    if (dense) mult_dense(r, blk); else mult_tilt(r, blk);
}

/* atlalib.c:169-175 checkiflostRectangularAp */
template <class T>
__device__ __forceinline__ void check_rect(P6T<T>& r, const double* lim) {
    const double x = val(r.x), y = val(r.y);
    if (x < lim[0] || x > lim[1]) r.ct = T(inf_d());
    else if (y < lim[2] || y > lim[3]) r.ct = T(inf_d());
}

/* atlalib.c:185-190 checkiflostEllipticalAp */
template <class T>
__device__ __forceinline__ void check_ellip(P6T<T>& r, const double* ax) {
    double xn = val(r.x) / ax[0];
    double zn = val(r.y) / ax[1];
    if ((xn * xn + zn * zn) >= 1) r.ct = T(inf_d());
}

/* atlalib.c:70-75 ATChangePRef */
template <bool FAST, class T>
__device__ __forceinline__ void change_pref(P6T<T>& r, double s) {
    r.px /= s;
    r.py /= s;
    r.dp = (r.dp + 1.0 - s) / s;
}

/* atlalib.c:59-68 ATdrift6 == driftkickrad.c:36-45 drift6 == diff_drift.c:30-43
 * (without the diffusion-matrix branch) */
template <bool FAST, class T>
__device__ __forceinline__ void drift6(P6T<T>& r, double L) {
    if constexpr (FAST) {
        double pn = 1.0 / (1.0 + r.dp);
        double nl = L * pn;
        r.x += nl * r.px;
        r.y += nl * r.py;
        r.ct += (0.5 * nl * pn) * (r.px * r.px + r.py * r.py);
    } else {
        T pn = 1 / (1 + r.dp);
        T nl = L * pn;
        r.x = madd(r.x, nl, r.px);
        r.y = madd(r.y, nl, r.py);
        r.ct += nl * pn * (r.px * r.px + r.py * r.py) / 2;
    }
}

/* driftkick.c:37-48 fastdrift.  FAST: c2 = NormL/(2(1+delta)) precomputed. */
template <bool FAST, class T>
__device__ __forceinline__ void fastdrift(P6T<T>& r, const T& nl, const T& c2) {
    r.x = madd(r.x, nl, r.px);
    r.y = madd(r.y, nl, r.py);
    if constexpr (FAST) r.ct += c2 * (r.px * r.px + r.py * r.py);
    else r.ct += nl * (r.px * r.px + r.py * r.py) / (2 * (1 + r.dp));
}

/* The Horner recursion shared by every multipole kick
 * (driftkick.c:51-115, diff_str_kick.c:33-40, diff_bnd_kick.c:40-47):
 * Re + i Im = sum_n (B_n + i A_n)(x + i y)^n, highest order first. */
/* one Horner step (re, im) <- (re, im)(x + i y) + (b + i a).  The fast
 * kernels evaluate it as two FMA chains per component (a different
 * association from the reference, within an ulp); the others keep the
 * reference's expression. */
template <class T>
__device__ __forceinline__ void horner_step(T& re, T& im, const T& x, const T& y, double b,
                                            double a) {
#if ATB_FAST
    const T ret = fma(re, x, fma(-im, y, b));
    im = fma(im, x, fma(re, y, a));
    re = ret;
#else
    T ret = re * x - im * y + b;
    im = im * x + re * y + a;
    re = ret;
#endif
}

template <int MO, class T>
__device__ __forceinline__ void horner_fixed(const double* A, const double* B, const T& x,
                                             const T& y, T& re, T& im) {
    re = B[MO];
    im = A[MO];
#pragma unroll
    for (int i = MO - 1; i >= 0; --i) horner_step(re, im, x, y, B[i], A[i]);
}

/* The same recursion for an upright magnet (every A_n = 0, fast kernels
 * only): the first step starts from Im = 0, so it is re B_MO x + B_{MO-1},
 * im = B_MO y, and later steps add no A_n.  Equal to horner_fixed up to the
 * sign of a zero. */
template <int MO, class T>
__device__ __forceinline__ void horner_upright(const double* B, const T& x, const T& y, T& re,
                                               T& im) {
    if constexpr (MO == 0) {
        re = B[0];
        im = 0.0;
    } else {
        re = fma(B[MO], x, B[MO - 1]);
        im = B[MO] * y;
#pragma unroll
        for (int i = MO - 2; i >= 0; --i) {
            const T ret = fma(re, x, fma(-im, y, B[i]));
            im = fma(im, x, re * y);
            re = ret;
        }
    }
}

template <class T>
__device__ __forceinline__ void horner_dyn(const double* A, const double* B, int mo, const T& x,
                                           const T& y, T& re, T& im) {
    re = B[mo];
    im = A[mo];
    for (int i = mo - 1; i >= 0; --i) horner_step(re, im, x, y, B[i], A[i]);
}

/* Tangent kernel only: the explicit partial of the field with respect to the
 * differentiated coefficient B_k, d(Re + i Im)/dB_k = (x + i y)^k, added to
 * the last derivative slot (the parameter direction). */
template <class T>
__device__ __forceinline__ void seed_coef(double x, double y, int k, T& re, T& im) {
    if constexpr (is_dual<T>::value) {
        if (k < 0) return;
        double zr = 1.0, zi = 0.0;
        for (int i = 0; i < k; ++i) {
            const double t = zr * x - zi * y;
            zi = zr * y + zi * x;
            zr = t;
        }
        constexpr int K = sizeof(re.d) / sizeof(double);
        re.d[K - 1] += zr;
        im.d[K - 1] += zi;
    }
}

/* Coefficient holder: for MO >= 0 the coefficients are copied into
 * registers once per element; MO < 0 reads them (broadcast) from the staged
 * table on every kick.  set_param() (derivative kernels only) replaces B_k by
 * a runtime strength and marks it as the differentiated parameter. */
template <int MO, bool SKEW = true>
struct Poly {
    double a[SKEW ? MO + 1 : 1], b[MO + 1];
    int sk;
    __device__ __forceinline__ void load(const double* A, const double* B, int) {
#pragma unroll
        for (int i = 0; i <= MO; ++i) {
            if constexpr (SKEW) a[i] = A[i];
            b[i] = B[i];
        }
        sk = -1;
    }
    __device__ __forceinline__ void set_param(int k, double v) {
#pragma unroll
        for (int i = 0; i <= MO; ++i)
            if (i == k) b[i] = v;
        sk = k;
    }
    template <class T>
    __device__ __forceinline__ void field(const T& x, const T& y, T& re, T& im) const {
        if constexpr (SKEW) horner_fixed<MO>(a, b, x, y, re, im);
        else horner_upright<MO>(b, x, y, re, im);
        seed_coef(val(x), val(y), sk, re, im);
    }
};

template <>
struct Poly<-1> {
    const double* a;
    const double* b;
    int mo;
    int sk;
    double kv;
    __device__ __forceinline__ void load(const double* A, const double* B, int m) {
        a = A; b = B; mo = m; sk = -1; kv = 0.0;
    }
    __device__ __forceinline__ void set_param(int k, double v) { sk = k; kv = v; }
    template <class T>
    __device__ __forceinline__ void field(const T& x, const T& y, T& re, T& im) const {
        if constexpr (is_dual<T>::value) {
            re = (sk == mo) ? kv : b[mo];
            im = a[mo];
            for (int i = mo - 1; i >= 0; --i)
                horner_step_dual(re, im, x, y, (i == sk) ? kv : b[i], a[i]);
            seed_coef(val(x), val(y), sk, re, im);
        } else if (sk >= 0) {
            re = (sk == mo) ? kv : b[mo];
            im = a[mo];
            for (int i = mo - 1; i >= 0; --i)
                horner_step(re, im, x, y, (i == sk) ? kv : b[i], a[i]);
        } else {
            horner_dyn(a, b, mo, x, y, re, im);
        }
    }
};

/* driftkick.c:92-115 strthinkick */
template <class PL, class T>
__device__ __forceinline__ void strthinkick(P6T<T>& r, const PL& pl, double L) {
    T re, im;
    pl.field(r.x, r.y, re, im);
    r.px = msub(r.px, L, re);
    r.py = madd(r.py, L, im);
}

/* driftkick.c:51-89 bndthinkick; lirho = L*irho folded on the host */
template <class PL, class T>
__device__ __forceinline__ void bndthinkick(P6T<T>& r, const PL& pl, double L, double irho,
                                            double lirho) {
    T re, im;
    pl.field(r.x, r.y, re, im);
    r.px -= L * (re - (r.dp - r.x * irho) * irho);
    r.py = madd(r.py, L, im);
    r.ct = madd(r.ct, lirho, r.x);
}

/* Radiating kicks and drifts in the reference's expression order
 * (exact and tangent kernels). */

/* The reference evaluates 1/(1+delta) at the start of every radiating drift
 * and kick and again after each kick's energy loss.  delta changes only in
 * that energy loss, so between two kicks every evaluation repeats the last one
 * on the same operand and gives the same IEEE result.  The _pn forms take it
 * from the caller (pn == 1.0 / (1.0 + r.dp) as last evaluated; a kick hands
 * back the value after its loss), so a magnet's slice loop divides once per
 * kick for it instead of once per drift and twice per kick. */

/* diff_str_kick.c:19-83 with B2perp of diff_str_kick.c:1-17 (bdiff == NULL) */
template <class PL, class T>
__device__ __forceinline__ void str_kick_rad_pn(P6T<T>& r, const PL& pl, double L, double radc,
                                                T& pn) {
    T re, im;
    pl.field(r.x, r.y, re, im);
    T p_norm = pn;
    T xpr = r.px * p_norm;
    T ypr = r.py * p_norm;
    T v_norm2 = 1.0 / (1.0 + xpr * xpr + ypr * ypr);
    T bx = im, by = re;
    T b2p = (by * by + bx * bx + (bx * ypr - by * xpr) * (bx * ypr - by * xpr)) * v_norm2;
    T factor = (1.0 + (xpr * xpr + ypr * ypr) / 2.0) / (p_norm * p_norm) * L;
    r.dp -= radc * b2p * factor;
    p_norm = 1.0 / (1.0 + r.dp);
    pn = p_norm;
    r.px = xpr / p_norm;
    r.py = ypr / p_norm;
    r.px = msub(r.px, L, re);
    r.py = madd(r.py, L, im);
}

/* diff_bnd_kick.c:101-174 with its B2perp (:85-99), bdiff == NULL */
template <class PL, class T>
__device__ __forceinline__ void bnd_kick_rad_pn(P6T<T>& r, const PL& pl, double L, double irho,
                                                double lirho, double radc, T& pn) {
    T re, im;
    pl.field(r.x, r.y, re, im);
    T p_norm = pn;
    T x = r.x;
    T xpr = r.px * p_norm;
    T ypr = r.py * p_norm;
    T bx = im, by = re + irho;
    T v_norm2 = 1.0 / ((1.0 + x * irho) * (1.0 + x * irho) + xpr * xpr + ypr * ypr);
    T b2p = ((by * (1 + x * irho)) * (by * (1 + x * irho)) +
             (bx * (1 + x * irho)) * (bx * (1 + x * irho)) +
             (bx * ypr - by * xpr) * (bx * ypr - by * xpr)) * v_norm2;
    T factor = (1.0 + x * irho + (xpr * xpr + ypr * ypr) / 2.0) / (p_norm * p_norm) * L;
    T dp_0 = r.dp;
    r.dp -= radc * b2p * factor;
    p_norm = 1.0 / (1.0 + r.dp);
    pn = p_norm;
    r.px = xpr / p_norm;
    r.py = ypr / p_norm;
    r.px -= L * (re - (dp_0 - r.x * irho) * irho);
    r.py = madd(r.py, L, im);
    r.ct = madd(r.ct, lirho, r.x);
}

/* diff_drift.c:30-43 (bdiff == NULL) */
template <class T>
__device__ __forceinline__ void diff_drift_pn(P6T<T>& r, double L, const T& pn) {
    T p_norm = pn;
    T NormL = L * p_norm;
    r.x = madd(r.x, NormL, r.px);
    r.y = madd(r.y, NormL, r.py);
    r.ct += NormL * p_norm * (r.px * r.px + r.py * r.py) / 2.0;
}

/* The fast kernels' radiating integrator.  Inside a radiating magnet they
 * carry the angles x' = px/(1+delta), y' = py/(1+delta) in place of px, py:
 * the reference's drift (diff_drift.c:30-43) advances x by L x', y by L y'
 * and ct by L (x'^2 + y'^2)/2, and its kicks (diff_str_kick.c:19-83,
 * diff_bnd_kick.c:101-174) rescale px, py so that x', y' pass through the
 * energy loss unchanged before the field kick -L Re (px), +L Im (py), which
 * moves x' by -L Re/(1+delta').  Each drift hands s = x'^2 + y'^2 to the
 * kick after it, and each kick hands opd = 1 + delta to the next (drifts
 * leave delta alone).  The energy-loss product is grouped as
 * (rL q) g opd^2 with rL = radc * L folded per element, q = B2perp before
 * its normalisation and g the normalisation times the path-length factor:
 * (1 + s/2)/(1 + s) in a straight magnet, evaluated for s < 1e-5 as its
 * series 1 - s/2 + s^2/2 (truncation below 5e-16 of a loss that is itself
 * ~1e-8 of delta), and (h_x + s/2)/(h_x^2 + s) in a bend.  The caller
 * converts px = x' opd, py = y' opd at the magnet's exit. */
struct RadAngles {
    double xp, yp, s, opd;
};

/* drift of length L, hL = L/2 */
__device__ __forceinline__ void rad_drift_fast(P6T<double>& r, RadAngles& a, double L,
                                               double hL) {
    r.x = fma(L, a.xp, r.x);
    r.y = fma(L, a.yp, r.y);
    a.s = fma(a.xp, a.xp, a.yp * a.yp);
    r.ct = fma(hL, a.s, r.ct);
}

template <class PL>
__device__ __forceinline__ void str_kick_rad_fast(P6T<double>& r, RadAngles& a, const PL& pl,
                                                  double L, double rL) {
    double re, im;
    pl.field(r.x, r.y, re, im);
    const double g = a.s < 1e-5 ? fma(a.s, fma(0.5, a.s, -0.5), 1.0)
                                : fma(0.5, a.s, 1.0) * rcp_nr(1.0 + a.s);
    const double cr = fma(im, a.yp, -(re * a.xp));
    const double q = fma(re, re, fma(im, im, cr * cr));
    r.dp = fma(-(rL * q) * g, a.opd * a.opd, r.dp);
    a.opd = 1.0 + r.dp;
    const double pn = rcp_nr(a.opd);
    a.xp = fma(-L * re, pn, a.xp);
    a.yp = fma(L * im, pn, a.yp);
}

template <class PL>
__device__ __forceinline__ void bnd_kick_rad_fast(P6T<double>& r, RadAngles& a, const PL& pl,
                                                  double L, double irho, double lirho,
                                                  double rL) {
    double re, im;
    pl.field(r.x, r.y, re, im);
    const double hx = fma(r.x, irho, 1.0);
    const double hx2 = hx * hx;
    const double vn = rcp_nr(hx2 + a.s);
    const double by = re + irho;
    const double cr = fma(im, a.yp, -(by * a.xp));
    const double q = fma(fma(by, by, im * im), hx2, cr * cr);
    const double h = fma(0.5, a.s, hx);
    const double dp0 = r.dp;
    r.dp = fma(-(rL * q) * (h * vn), a.opd * a.opd, r.dp);
    a.opd = 1.0 + r.dp;
    const double pn = rcp_nr(a.opd);
    const double u = fma(-fma(-r.x, irho, dp0), irho, re);
    a.xp = fma(-L * u, pn, a.xp);
    a.yp = fma(L * im, pn, a.yp);
    r.ct = fma(lirho, r.x, r.ct);
}

/* quadfringe.c:3-51 QuadFringePassP (sign=+1) / QuadFringePassN (sign=-1) */
template <bool FAST, class T, class B2>
__device__ __forceinline__ void quad_fringe(P6T<T>& r, const B2& b2, bool entrance) {
    T u = b2 / (12.0 * (1.0 + r.dp));
    T x2 = r.x * r.x;
    T z2 = r.y * r.y;
    T xz = r.x * r.y;
    T gx = u * (x2 + 3 * z2) * r.x;
    T gz = u * (z2 + 3 * x2) * r.y;
    T r1tmp = 3 * u * (2 * xz * r.py - (x2 + z2) * r.px);
    T r3tmp = 3 * u * (2 * xz * r.px - (x2 + z2) * r.py);
    T dct = (gz * r.py - gx * r.px) / (1 + r.dp);
    if (entrance) {
        r.x += gx;
        r.y -= gz;
        r.ct -= dct;
        r.px += r1tmp;
        r.py -= r3tmp;
    } else {
        r.x -= gx;
        r.y += gz;
        r.ct += dct;
        r.px -= r1tmp;
        r.py += r3tmp;
    }
}

/* one linear map of quadfringe.c:45-112 (x and y 2x2 blocks) */
template <class T>
__device__ __forceinline__ void lin_fringe_map(P6T<T>& r, const double* m) {
    const T x = r.x, px = r.px, y = r.y, py = r.py;
    r.x = m[0] * x + m[1] * px;
    r.px = m[2] * x + m[3] * px;
    r.y = m[4] * y + m[5] * py;
    r.py = m[6] * y + m[7] * py;
}

/* Edge focusing of BndMPoleSymplectic4Pass: atphyslib.c:15-79
 * (edge_fringe_entrance / edge_fringe_exit).  sgn = +1 entrance, -1 exit.
 * fy_c = irho*tan(edge) is used whenever the tangent's argument is exactly
 * the edge angle (fringecorr == 0), as the reference then evaluates the same
 * tan(edge_angle). */
template <bool FAST, class T>
__device__ __forceinline__ void edge_fringe(P6T<T>& r, double irho, double edge, double fc,
                                            double fx, double fy_c, int method, bool fc0,
                                            double sgn) {
    T fy;
    if (method == ATB_BM_3) {
        T q = r.px / (1 + r.dp);
        fy = irho * tan(sgn > 0 ? (edge - fc + q) : (edge - fc - q));
    } else {
        if (FAST && fc0) {
            if (method == ATB_BM_2) fy = fy_c / (1 + r.dp); else fy = T(fy_c);
        } else {
            T t = edge - fc / (1 + r.dp);
            T tn = (val(t) == edge) ? T(fy_c) : irho * tan(t);
            if constexpr (is_dual<T>::value) {
                /* same value, with the derivative of tan(t) kept */
                if (val(t) == edge) { tn = irho * tan(t); tn.v = fy_c; }
            }
            if (method == ATB_BM_2) fy = tn / (1 + r.dp); else fy = tn;
        }
    }
    r.px += r.x * fx;
    r.py -= r.y * fy;
}

/* diff_bend_fringe.c:1-52 (bdiff == NULL) for the radiating bend */
template <bool FAST, class T>
__device__ __forceinline__ void edge_fringe_rad(P6T<T>& r, double irho, double edge, double psi,
                                                double fx, double fy_c, int method, bool fc0,
                                                double sgn) {
    T p_norm = 1.0 / (1.0 + r.dp);
    T fy;
    if (method == ATB_BM_3) {
        fy = irho * tan(edge - psi + sgn * r.px * p_norm);
    } else {
        if (FAST && fc0) {
            if (method == ATB_BM_2) fy = fy_c * p_norm; else fy = T(fy_c);
        } else {
            T t = edge - psi * p_norm;
            T tn = (val(t) == edge) ? T(fy_c) : irho * tan(t);
            if constexpr (is_dual<T>::value) {
                if (val(t) == edge) { tn = irho * tan(t); tn.v = fy_c; }
            }
            if (method == ATB_BM_2) fy = tn * p_norm; else fy = tn;
        }
    }
    r.px += r.x * fx;
    r.py -= r.y * fy;
}

/* ---- quantum diffusion ------------------------------------------------
 * The random kicks are counter-based: the normals of particle p at element
 * ei in turn nturn are a pure function of (key, p, nturn, ei), so every
 * thread draws its own without shared state and results do not depend on
 * the launch shape.  The 64-bit mixer is the splitmix64 finaliser
 * (Steele, Lea and Flood 2014; constants as published by Vigna); normals
 * come in pairs from the Box-Muller transform of two uniforms in (0, 1]. */
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ void quantdiff_normals(uint64_t key, long long p, int nturn, int ei,
                                                  double z[6]) {
    const uint64_t golden = 0x9e3779b97f4a7c15ULL;
    uint64_t s = mix64(key + golden * (uint64_t)(p + 1));
    s = mix64(s ^ ((uint64_t)(uint32_t)nturn << 32 | (uint32_t)ei));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s += golden;
        const uint64_t a = mix64(s);
        s += golden;
        const uint64_t b = mix64(s);
        const double u1 = (double)((a >> 11) + 1) * 0x1.0p-53;   /* (0, 1] */
        const double u2 = (double)(b >> 11) * 0x1.0p-53;         /* [0, 1) */
        const double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        z[2 * k] = rad * cs;
        z[2 * k + 1] = rad * sn;
    }
}

/* QuantDiffPass.c:9-45: r += L z, L lower triangular (column-major), z six
 * standard normals */
__device__ __forceinline__ void quantdiff_kick(P6& r, const double* L, const double z[6]) {
    double d[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j <= i; ++j) s += z[j] * L[i + 6 * j];
        d[i] = s;
    }
    r.x += d[0]; r.px += d[1]; r.y += d[2]; r.py += d[3]; r.dp += d[4]; r.ct += d[5];
}

}  // namespace atb

#endif  // ATB_PHYSICS_CUH
