/*
 * ORACLE -- test infrastructure only.
 *
 * The oracle's integrators (oracle.c) evaluated in IEEE binary128 (gcc's
 * __float128 and libquadmath), for finite differences of tracked
 * coordinates whose rounding floor (about 2^-113 relative per operation)
 * lies far below the 1e-7 agreement asked of the exact derivatives.  A
 * central difference of the double-precision map with h = 1e-7 carries a
 * rounding error of order sqrt(operations) * eps * |r| / h, which for the
 * second-order sextupole term near the closed orbit exceeds the derivative
 * itself; in binary128 it is some 1e-30 relative.  Element data arrive in
 * double (exactly representable in binary128), so this is the double map up
 * to rounding, and its derivatives agree with the double map's to far below
 * 1e-7.  The result is returned as a double-double pair (hi + lo), so the
 * caller can difference two runs without losing the low bits.
 */
#include <quadmath.h>

#define ORACLE_REAL __float128
#define R_SIN sinq
#define R_COS cosq
#define R_TAN tanq
#define R_EXP expq
#define R_POW powq
#define R_ROUND roundq
#define R_FABS fabsq
#define R_SQRT sqrtq

#include "oracle.c"

/* Whole turns from element 0 (setlost on loss, no loss map, no refpts):
 * r_in (6, np) double in, hi/lo (6, np) out with r = hi + lo. */
int oracle_track_hilo(const OElem *el, int nelem, const double *r_in, double *hi, double *lo,
                      int64_t np, int nturns, int turn0, double energy, double rest, double T0,
                      int nthreads) {
    OPrep *pp = o_prepare_all(el, nelem, energy, rest, T0);
    if (!pp) return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t p = 0; p < np; p++) {
        real buf[6];
        for (int k = 0; k < 6; k++) buf[k] = r_in[6 * p + k];
        o_particle(buf, el, pp, nelem, nturns, turn0, 0, nelem, NULL, 0, 0, 1, T0, NULL, np, p,
                   NULL, NULL, NULL, NULL);
        for (int k = 0; k < 6; k++) {
            double h = (double)buf[k];
            hi[6 * p + k] = h;
            lo[6 * p + k] = (double)(buf[k] - (real)h);
        }
    }
    free(pp);
    return 0;
}
