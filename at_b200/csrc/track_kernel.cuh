/*
 * The persistent multi-turn tracking kernel.
 *
 * One thread owns one particle's (x, px, y, py, delta, ct) in registers for
 * all the turns of a launch.  A block walks the lattice program (the flat
 * element table of atb_table.h) segment by segment: each segment is copied
 * from global memory into shared memory by the bulk-copy (TMA) engine,
 * double-buffered behind an mbarrier, and every element's parameters are then
 * read from shared memory as warp-uniform broadcasts.  When the whole table
 * fits in one buffer it is loaded once per block and stays resident.
 *
 * The turn/element loop, the refpts snapshots and the loss rule restate the
 * reference engine (pyat/at.c:596-654, checkiflost :115-139, setlost
 * :142-161); the per-element bodies restate the pass methods (see
 * atb_physics.cuh).  This header is compiled twice, once per arithmetic mode
 * (ATB_FAST = 0 / 1), into distinct kernel symbols.
 */
#ifndef ATB_TRACK_KERNEL_CUH
#define ATB_TRACK_KERNEL_CUH

#include <cstdint>
#include "atb_physics.cuh"
#include "atb_integrators.h"
#include "atb_kernel_api.h"

#ifndef ATB_FAST
#error "define ATB_FAST to 0 or 1"
#endif

#define ATB_CAT2(a, b) a##b
#define ATB_CAT(a, b) ATB_CAT2(a, b)
#if ATB_FAST
#define ATB_KSUFFIX _fast
#else
#define ATB_KSUFFIX _exact
#endif

namespace atb {

constexpr bool kFast = (ATB_FAST != 0);

/* ---------------- shared-memory staging (bulk copy + mbarrier) ---------- */

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

/* global -> shared bulk copy into this CTA's own shared memory, completion
 * signalled on the mbarrier; the source is always this GPU's own memory */
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

/* Bounded wait: gives up after ATB_WAIT_NS nanoseconds and reports it. */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > ATB_WAIT_NS) return false;
    }
}

/* ---------------- record access ------------------------------------------ */

struct Rec {
    const double* p;
    uint64_t hdr;
    uint64_t opt;
    __device__ __forceinline__ int op() const { return (int)((hdr >> ATB_H_OP_SHIFT) & ATB_H_OP_MASK); }
    __device__ __forceinline__ int mo() const { return (int)((hdr >> ATB_H_MO_SHIFT) & ATB_H_MO_MASK); }
    __device__ __forceinline__ uint32_t flags() const { return (uint32_t)((hdr >> ATB_H_FL_SHIFT) & ATB_H_FL_MASK); }
    __device__ __forceinline__ int nsteps() const { return (int)((hdr >> ATB_H_NS_SHIFT) & ATB_H_NS_MASK); }
    __device__ __forceinline__ int len() const { return (int)((hdr >> ATB_H_LEN_SHIFT) & ATB_H_LEN_MASK); }
    __device__ __forceinline__ const double* blk(int slot) const {
        uint32_t o = (uint32_t)((opt >> (slot * ATB_OPT_BITS)) & ATB_OPT_MASK);
        return o ? p + o : nullptr;
    }
    __device__ __forceinline__ double f(int w) const { return p[w]; }
};

/* ---------------- misalignment / aperture wrappers ----------------------- */

template <class T>
__device__ __forceinline__ void entrance_misalign(P6T<T>& r, const Rec& e) {
    const uint32_t fl = e.flags();
    if (const double* t1 = e.blk(ATB_OPT_T1)) add_t(r, t1);
    if (const double* r1 = e.blk(ATB_OPT_R1)) mult_r(r, r1, fl & ATB_F_R1_DENSE);
}

template <class T>
__device__ __forceinline__ void apertures(P6T<T>& r, const Rec& e) {
    if (const double* ra = e.blk(ATB_OPT_RAP)) check_rect(r, ra);
    if (const double* ea = e.blk(ATB_OPT_EAP)) check_ellip(r, ea);
}

template <class T>
__device__ __forceinline__ void exit_misalign(P6T<T>& r, const Rec& e) {
    const uint32_t fl = e.flags();
    if (const double* r2 = e.blk(ATB_OPT_R2)) mult_r(r, r2, fl & ATB_F_R2_DENSE);
    if (const double* t2 = e.blk(ATB_OPT_T2)) add_t(r, t2);
}

/* ---------------- pass methods ------------------------------------------- */

/* A differentiated strength (derivative kernels only): PolynomB[k] of the
 * element is replaced by v and, on dual numbers, carried as the last
 * derivative direction.  The tracking kernels pass k = -1. */
struct Param {
    int k;        /* coefficient order, -1: none */
    double v;
};

/* the quadrupole-fringe gradient b1 = PolynomB[1], seeded when it is the
 * differentiated strength */
template <class T>
__device__ __forceinline__ T fringe_b1(const Rec& e, const Param& pm) {
    T b1 = e.f(ATB_SM_B1);
    if constexpr (is_dual<T>::value) {
        if (pm.k == 1) {
            b1.v = pm.v;
            b1.d[sizeof(b1.d) / sizeof(double) - 1] = 1.0;
        }
    } else {
        if (pm.k == 1) b1 = pm.v;
    }
    return b1;
}

/* The integration steps of a thick multipole under integrator id
 * e.f(ATB_SM_INTEG) (1-6, atb_integrators.h), step SL = e.f(ATB_SM_SL): per
 * step, for each stage a drift of SL*c[i] and a kick of SL*d[i], skipping zero
 * coefficients.  The drift and kick are the ones the Forest-Ruth steps use:
 * fastdrift with the entrance 1/(1+delta) in plain magnets (pnorm: the
 * entrance L2 x 1/(1+delta) with the table's L2 word set to 1.0), the
 * radiating drift and kicks otherwise (the angle-carrying forms in the fast
 * kernels). */
template <int NP, bool BEND, bool RAD, class PL, class T>
__device__ __forceinline__ void multipole_steps_generic(P6T<T>* r, const Rec& e, const PL& pl,
                                                        const T* pnorm, double irho, int ns) {
    const double SL = e.f(ATB_SM_SL);
    int id = (int)e.f(ATB_SM_INTEG);
    if (id < 1 || id >= ATB_INTEG_COUNT) id = 4;   /* the host writes 1-6 only */
    const AtbInteg& ig = atb_integ[id];
    if (RAD) {
        const double radc = e.f(ATB_SM_RADC);
        if constexpr (kFast && !is_dual<T>::value) {
            if (ns <= 0) return;
            RadAngles a[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const double pn = 1.0 / (1.0 + r[k].dp);
                a[k] = RadAngles{r[k].px * pn, r[k].py * pn, 0.0, 1.0 + r[k].dp};
            }
            for (int m = 0; m < ns; ++m) {
                for (int i = 0; i < ig.n; ++i) {
                    if (ig.c[i] != 0.0) {
                        const double ld = SL * ig.c[i];
#pragma unroll
                        for (int k = 0; k < NP; ++k) rad_drift_fast(r[k], a[k], ld, 0.5 * ld);
                    }
                    if (ig.d[i] != 0.0) {
                        const double lk = SL * ig.d[i];
#pragma unroll
                        for (int k = 0; k < NP; ++k) {
                            if (BEND) bnd_kick_rad_fast(r[k], a[k], pl, lk, irho, lk * irho, radc * lk);
                            else str_kick_rad_fast(r[k], a[k], pl, lk, radc * lk);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                r[k].px = a[k].xp * a[k].opd;
                r[k].py = a[k].yp * a[k].opd;
            }
        } else {
            T pn[NP];   /* 1/(1+delta) as last evaluated, as in the steps below */
#pragma unroll
            for (int k = 0; k < NP; ++k) pn[k] = 1.0 / (1.0 + r[k].dp);
            for (int m = 0; m < ns; ++m) {
                for (int i = 0; i < ig.n; ++i) {
                    if (ig.c[i] != 0.0) {
                        const double ld = SL * ig.c[i];
#pragma unroll
                        for (int k = 0; k < NP; ++k) diff_drift_pn(r[k], ld, pn[k]);
                    }
                    if (ig.d[i] != 0.0) {
                        const double lk = SL * ig.d[i];
#pragma unroll
                        for (int k = 0; k < NP; ++k) {
                            if (BEND) bnd_kick_rad_pn(r[k], pl, lk, irho, lk * irho, radc, pn[k]);
                            else str_kick_rad_pn(r[k], pl, lk, radc, pn[k]);
                        }
                    }
                }
            }
        }
    } else {
        T h[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) h[k] = kFast ? T(0.5 / (1.0 + r[k].dp)) : T(0.0);
        for (int m = 0; m < ns; ++m) {
            for (int i = 0; i < ig.n; ++i) {
                if (ig.c[i] != 0.0) {
                    const double ld = SL * ig.c[i];
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        const T nl = ld * pnorm[k];
                        fastdrift<kFast>(r[k], nl, kFast ? T(nl * h[k]) : T(0.0));
                    }
                }
                if (ig.d[i] != 0.0) {
                    const double lk = SL * ig.d[i];
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        if (BEND) bndthinkick(r[k], pl, lk, irho, lk * irho);
                        else strthinkick(r[k], pl, lk);
                    }
                }
            }
        }
    }
}

/* StrMPoleSymplectic4Pass.c:29-109, BndMPoleSymplectic4Pass.c:38-129,
 * StrMPoleSymplectic4RadPass.c:30-115, BndMPoleSymplectic4RadPass.c:39-128.
 * NP particles of one thread pass the element together: every per-particle
 * step is an unrolled loop over them, so in the slice loop their drifts and
 * kicks form one straight-line block whose independent chains the compiler
 * interleaves (NP = 2), while the element's parameters are read once.  Each
 * particle sees the same operations as alone (NP = 1). */
template <int NP, int MO, bool BEND, bool RAD, bool SKEW = true, bool GEN = false, class T>
__device__ __forceinline__ void pass_multipole_n(P6T<T>* r, const Rec& e, const Param& pm) {
    const uint32_t fl = e.flags();
    const double L1 = e.f(ATB_SM_L1), L2 = e.f(ATB_SM_L2);
    const double K1 = e.f(ATB_SM_K1), K2 = e.f(ATB_SM_K2);
    const int mo = e.mo();
    const double* A = e.p + (BEND ? ATB_BM_POLY : ATB_SM_POLY);
    const double* B = A + mo + 1;
    Poly<MO, SKEW> pl;
    pl.load(A, B, mo);
    if (pm.k >= 0) pl.set_param(pm.k, pm.v);

    T nl1[NP], nl2[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        if (fl & ATB_F_SCALING) change_pref<kFast>(r[k], e.f(ATB_SM_SCALE));
        nl1[k] = 0.0;
        nl2[k] = 0.0;
        if (!RAD) {
            T p_norm = 1.0 / (1.0 + r[k].dp);
            nl1[k] = L1 * p_norm;
            nl2[k] = L2 * p_norm;
        }
        entrance_misalign(r[k], e);
        apertures(r[k], e);
    }
    double irho = 0.0, k1i = 0.0, k2i = 0.0;
    if (BEND) {
        irho = e.f(ATB_BM_IRHO);
        k1i = e.f(ATB_BM_K1IRHO);
        k2i = e.f(ATB_BM_K2IRHO);
        const int m_in = (int)((fl >> ATB_F_BM_IN_SHIFT) & ATB_F_BM_MASK);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (RAD)
                edge_fringe_rad<kFast>(r[k], irho, e.f(ATB_BM_EIN), e.f(ATB_BM_FCIN),
                                       e.f(ATB_BM_FXIN), e.f(ATB_BM_FYIN), m_in,
                                       fl & ATB_F_FC0_IN, 1.0);
            else
                edge_fringe<kFast>(r[k], irho, e.f(ATB_BM_EIN), e.f(ATB_BM_FCIN),
                                   e.f(ATB_BM_FXIN), e.f(ATB_BM_FYIN), m_in, fl & ATB_F_FC0_IN,
                                   1.0);
        }
    }
    if (fl & ATB_F_FQ_IN) {
        const T b1 = fringe_b1<T>(e, pm);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (fl & ATB_F_FQ_IN_LIN) {
                const double* fm = e.blk(ATB_OPT_FRINGE);
                lin_fringe_map(r[k], fm);
                quad_fringe<kFast>(r[k], b1, true);
                lin_fringe_map(r[k], fm + 8);
            } else {
                quad_fringe<kFast>(r[k], b1, true);
            }
        }
    }
    const int ns = e.nsteps();
    if constexpr (GEN) {
        /* another integrator of the GPU call: steps of SL*c[i] drift and
           SL*d[i] kick (atgpu/SymplecticIntegrator.cpp:140-171) */
        multipole_steps_generic<NP, BEND, RAD>(r, e, pl, nl2, irho, ns);
    } else if (RAD) {
        const double radc = e.f(ATB_SM_RADC);
        if constexpr (kFast && !is_dual<T>::value) {
            if (ns > 0) {
                const double rk1 = radc * K1, rk2 = radc * K2;
                const double h1 = 0.5 * L1, h2 = 0.5 * L2;
                RadAngles a[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    const double pn = 1.0 / (1.0 + r[k].dp);
                    a[k] = RadAngles{r[k].px * pn, r[k].py * pn, 0.0, 1.0 + r[k].dp};
                }
                for (int m = 0; m < ns; ++m) {
#pragma unroll
                    for (int k = 0; k < NP; ++k) rad_drift_fast(r[k], a[k], L1, h1);
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        if (BEND) bnd_kick_rad_fast(r[k], a[k], pl, K1, irho, k1i, rk1);
                        else str_kick_rad_fast(r[k], a[k], pl, K1, rk1);
                    }
#pragma unroll
                    for (int k = 0; k < NP; ++k) rad_drift_fast(r[k], a[k], L2, h2);
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        if (BEND) bnd_kick_rad_fast(r[k], a[k], pl, K2, irho, k2i, rk2);
                        else str_kick_rad_fast(r[k], a[k], pl, K2, rk2);
                    }
#pragma unroll
                    for (int k = 0; k < NP; ++k) rad_drift_fast(r[k], a[k], L2, h2);
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        if (BEND) bnd_kick_rad_fast(r[k], a[k], pl, K1, irho, k1i, rk1);
                        else str_kick_rad_fast(r[k], a[k], pl, K1, rk1);
                    }
#pragma unroll
                    for (int k = 0; k < NP; ++k) rad_drift_fast(r[k], a[k], L1, h1);
                }
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    r[k].px = a[k].xp * a[k].opd;
                    r[k].py = a[k].yp * a[k].opd;
                }
            }
        } else {
            /* pn: 1/(1+delta) as the reference last evaluated it (it changes
               only in a kick's energy loss, and the kick hands it on) */
            T pn[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) pn[k] = 1.0 / (1.0 + r[k].dp);
            for (int m = 0; m < ns; ++m) {
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    diff_drift_pn(r[k], L1, pn[k]);
                    if (BEND) bnd_kick_rad_pn(r[k], pl, K1, irho, k1i, radc, pn[k]);
                    else str_kick_rad_pn(r[k], pl, K1, radc, pn[k]);
                    diff_drift_pn(r[k], L2, pn[k]);
                    if (BEND) bnd_kick_rad_pn(r[k], pl, K2, irho, k2i, radc, pn[k]);
                    else str_kick_rad_pn(r[k], pl, K2, radc, pn[k]);
                    diff_drift_pn(r[k], L2, pn[k]);
                    if (BEND) bnd_kick_rad_pn(r[k], pl, K1, irho, k1i, radc, pn[k]);
                    else str_kick_rad_pn(r[k], pl, K1, radc, pn[k]);
                    diff_drift_pn(r[k], L1, pn[k]);
                }
            }
        }
    } else {
        T c1[NP], c2[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            c1[k] = 0.0;
            c2[k] = 0.0;
            if (kFast) {
                T h = 0.5 / (1.0 + r[k].dp);
                c1[k] = nl1[k] * h;
                c2[k] = nl2[k] * h;
            }
        }
        for (int m = 0; m < ns; ++m) {
#pragma unroll
            for (int k = 0; k < NP; ++k) fastdrift<kFast>(r[k], nl1[k], c1[k]);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (BEND) bndthinkick(r[k], pl, K1, irho, k1i); else strthinkick(r[k], pl, K1);
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) fastdrift<kFast>(r[k], nl2[k], c2[k]);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (BEND) bndthinkick(r[k], pl, K2, irho, k2i); else strthinkick(r[k], pl, K2);
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) fastdrift<kFast>(r[k], nl2[k], c2[k]);
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                if (BEND) bndthinkick(r[k], pl, K1, irho, k1i); else strthinkick(r[k], pl, K1);
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) fastdrift<kFast>(r[k], nl1[k], c1[k]);
        }
    }
    if (fl & ATB_F_FQ_OUT) {
        const T b1 = fringe_b1<T>(e, pm);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (fl & ATB_F_FQ_OUT_LIN) {
                const double* fm = e.blk(ATB_OPT_FRINGE);
                lin_fringe_map(r[k], fm + 16);
                quad_fringe<kFast>(r[k], b1, false);
                lin_fringe_map(r[k], fm + 24);
            } else {
                quad_fringe<kFast>(r[k], b1, false);
            }
        }
    }
    const int m_out = (int)((fl >> ATB_F_BM_OUT_SHIFT) & ATB_F_BM_MASK);
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        if (BEND) {
            if (RAD)
                edge_fringe_rad<kFast>(r[k], irho, e.f(ATB_BM_EOUT), e.f(ATB_BM_FCOUT),
                                       e.f(ATB_BM_FXOUT), e.f(ATB_BM_FYOUT), m_out,
                                       fl & ATB_F_FC0_OUT, -1.0);
            else
                edge_fringe<kFast>(r[k], irho, e.f(ATB_BM_EOUT), e.f(ATB_BM_FCOUT),
                                   e.f(ATB_BM_FXOUT), e.f(ATB_BM_FYOUT), m_out,
                                   fl & ATB_F_FC0_OUT, -1.0);
        }
        apertures(r[k], e);
        exit_misalign(r[k], e);
        if (fl & ATB_F_SCALING) change_pref<kFast>(r[k], e.f(ATB_SM_ISCALE));
    }
}

template <int NP, bool BEND, bool RAD, bool GEN = false, class T>
__device__ __forceinline__ void pass_multipole_dispatch_n(P6T<T>* r, const Rec& e,
                                                          const Param& pm) {
    if constexpr (is_dual<T>::value) {
        /* one generic instance for the tangent kernel keeps its size sane */
        pass_multipole_n<NP, -1, BEND, RAD>(r, e, pm);
    } else {
        /* tables compiled for another integrator of the GPU call take one
           generic instance, in the kernels built with them (GEN); the hosts
           of the other kernels send them none (atb_track_noalloc checks its
           raw table with a scan kernel, the tangent host refuses it) */
        if constexpr (GEN) {
            if (e.flags() & ATB_F_INTEG) {
                pass_multipole_n<NP, -1, BEND, RAD, true, true>(r, e, pm);
                return;
            }
        }
        /* the fast kernels evaluate upright magnets' fields without the
           zero skew terms */
        const bool upright = kFast && (e.flags() & ATB_F_NOSKEW);
        switch (e.mo()) {
            case 0: pass_multipole_n<NP, 0, BEND, RAD>(r, e, pm); break;
            case 1:
                if (upright) pass_multipole_n<NP, 1, BEND, RAD, !kFast>(r, e, pm);
                else pass_multipole_n<NP, 1, BEND, RAD>(r, e, pm);
                break;
            case 2:
                if (upright) pass_multipole_n<NP, 2, BEND, RAD, !kFast>(r, e, pm);
                else pass_multipole_n<NP, 2, BEND, RAD>(r, e, pm);
                break;
            case 3:
                if (upright) pass_multipole_n<NP, 3, BEND, RAD, !kFast>(r, e, pm);
                else pass_multipole_n<NP, 3, BEND, RAD>(r, e, pm);
                break;
            default: pass_multipole_n<NP, -1, BEND, RAD>(r, e, pm); break;
        }
    }
}

template <bool BEND, bool RAD, bool GEN = false, class T>
__device__ __forceinline__ void pass_multipole_dispatch(P6T<T>& r, const Rec& e, const Param& pm) {
    pass_multipole_dispatch_n<1, BEND, RAD, GEN>(&r, e, pm);
}

/* DriftPass.c:16-48 */
template <class T>
__device__ __forceinline__ void pass_drift(P6T<T>& r, const Rec& e) {
    entrance_misalign(r, e);
    apertures(r, e);
    drift6<kFast>(r, e.f(ATB_DR_LE));
    apertures(r, e);
    exit_misalign(r, e);
}

/* IdentityPass.c:20-43 */
template <class T>
__device__ __forceinline__ void pass_identity(P6T<T>& r, const Rec& e) {
    entrance_misalign(r, e);
    apertures(r, e);
    exit_misalign(r, e);
}

/* ThinMPolePass.c:28-70 */
template <class T>
__device__ __forceinline__ void pass_thinmpole(P6T<T>& r, const Rec& e, const Param& pm) {
    const uint32_t fl = e.flags();
    const int mo = e.mo();
    const double* A = e.p + ATB_TM_POLY;
    const double* B = A + mo + 1;
    Poly<-1> pl;
    pl.load(A, B, mo);
    if (pm.k >= 0) pl.set_param(pm.k, pm.v);
    const double bax = e.f(ATB_TM_BAX), bay = e.f(ATB_TM_BAY);
    if (fl & ATB_F_SCALING) change_pref<kFast>(r, e.f(ATB_TM_SCALE));
    entrance_misalign(r, e);
    apertures(r, e);
    strthinkick(r, pl, 1.0);
    r.px += bax * r.dp;
    r.py -= bay * r.dp;
    r.ct -= bax * r.x - bay * r.y;
    exit_misalign(r, e);
    if (fl & ATB_F_SCALING) change_pref<kFast>(r, e.f(ATB_TM_ISCALE));
}

/* RFCavityPass.c:23-68 -> attrackfunc.c:5-42 (trackRFCavity) */
template <class T>
__device__ __forceinline__ void rf_kick(P6T<T>& r, const Rec& e, int nturn) {
    const double nv = e.f(ATB_RF_NV), tf = e.f(ATB_RF_TF), lag = e.f(ATB_RF_LAG);
    const double ht = e.f(ATB_RF_HT), phi = e.f(ATB_RF_PHI);
    r.dp += -nv * sin(tf * ((r.ct - lag) / ATB_C0 - ht * (double)nturn) - phi);
}

template <class T>
__device__ __forceinline__ void pass_rfcavity(P6T<T>& r, const Rec& e, int nturn) {
    const uint32_t fl = e.flags();
    if (!(fl & ATB_F_THICK)) {
        if (fl & ATB_F_NV) rf_kick(r, e, nturn);
    } else {
        const double half = e.f(ATB_RF_HALF);
        drift6<kFast>(r, half);
        if (fl & ATB_F_NV) rf_kick(r, e, nturn);
        drift6<kFast>(r, half);
    }
}

/* CorrectorPass.c:25-90 */
template <class T>
__device__ __forceinline__ void pass_corrector(P6T<T>& r, const Rec& e) {
    const uint32_t fl = e.flags();
    const double xk = e.f(ATB_CO_XK), yk = e.f(ATB_CO_YK);
    if (fl & ATB_F_SCALING) change_pref<kFast>(r, e.f(ATB_CO_SCALE));
    if (!(fl & ATB_F_THICK)) {
        entrance_misalign(r, e);
        apertures(r, e);
        r.px += xk;
        r.py += yk;
    } else {
        const double le = e.f(ATB_CO_LE);
        T p_norm = 1.0 / (1.0 + r.dp);
        T nl = le * p_norm;
        entrance_misalign(r, e);
        apertures(r, e);
        r.ct += nl * p_norm * (e.f(ATB_CO_K2) + r.px * r.px + r.py * r.py + r.px * xk + r.py * yk) / 2;
        r.x += nl * (r.px + e.f(ATB_CO_HX));
        r.px += xk;
        r.y += nl * (r.py + e.f(ATB_CO_HY));
        r.py += yk;
        apertures(r, e);
    }
    exit_misalign(r, e);
    if (fl & ATB_F_SCALING) change_pref<kFast>(r, e.f(ATB_CO_ISCALE));
}

/* One element on one particle; lost particles (x is NaN) are skipped as every
 * reference pass method does (e.g. StrMPoleSymplectic4Pass.c:59). */
/* QuantDiffPass.c: random kicks keyed by (key, pbase + p, nturn, ei);
 * without a key (the derivative kernels) the element is the identity, as the
 * reference's envelope code disables it */
template <class T>
__device__ __forceinline__ void pass_quantdiff(P6T<T>& r, const Rec& e, const AtbRng* rng,
                                               long long p, int nturn, int ei) {
    if constexpr (!is_dual<T>::value) {
        if (rng) {
            double z[6];
            quantdiff_normals(rng->key, rng->pbase + p, nturn, ei, z);
            quantdiff_kick(r, e.p + ATB_QD_L, z);
        }
    }
}

template <bool GEN = false, class T>
__device__ __forceinline__ void track_element(P6T<T>& r, const Rec& e, int nturn,
                                              const Param& pm = Param{-1, 0.0},
                                              const AtbRng* rng = nullptr, long long p = 0,
                                              int ei = 0) {
    if (isnan(val(r.x))) return;
    switch (e.op()) {
        case ATB_OP_IDENTITY: pass_identity(r, e); break;
        case ATB_OP_DRIFT: pass_drift(r, e); break;
        case ATB_OP_STRMPOLE: pass_multipole_dispatch<false, false, GEN>(r, e, pm); break;
        case ATB_OP_STRMPOLE_RAD: pass_multipole_dispatch<false, true, GEN>(r, e, pm); break;
        case ATB_OP_BNDMPOLE: pass_multipole_dispatch<true, false, GEN>(r, e, pm); break;
        case ATB_OP_BNDMPOLE_RAD: pass_multipole_dispatch<true, true, GEN>(r, e, pm); break;
        case ATB_OP_THINMPOLE: pass_thinmpole(r, e, pm); break;
        case ATB_OP_RFCAVITY: pass_rfcavity(r, e, nturn); break;
        case ATB_OP_CORRECTOR: pass_corrector(r, e); break;
        case ATB_OP_APERTURE: check_rect(r, e.p + ATB_AP_LIM); break;
        case ATB_OP_QUANTDIFF: pass_quantdiff(r, e, rng, p, nturn, ei); break;
        default: break;
    }
}

/* The particles of a thread go through a thick multipole together when none
 * of them is lost (a lost particle skips every element). */
template <int NP>
__device__ __forceinline__ bool track_together(const P6 (&r)[NP], const Rec& e) {
    const int op = e.op();
    if (op != ATB_OP_STRMPOLE && op != ATB_OP_STRMPOLE_RAD && op != ATB_OP_BNDMPOLE &&
        op != ATB_OP_BNDMPOLE_RAD)
        return false;
    bool all = true;
#pragma unroll
    for (int k = 0; k < NP; ++k) all &= !isnan(r[k].x);
    return all;
}

template <int NP>
__device__ __forceinline__ void pass_multipoles_together(P6 (&r)[NP], const Rec& e) {
    const Param none{-1, 0.0};
    switch (e.op()) {
        case ATB_OP_STRMPOLE: pass_multipole_dispatch_n<NP, false, false>(r, e, none); break;
        case ATB_OP_STRMPOLE_RAD: pass_multipole_dispatch_n<NP, false, true>(r, e, none); break;
        case ATB_OP_BNDMPOLE: pass_multipole_dispatch_n<NP, true, false>(r, e, none); break;
        default: pass_multipole_dispatch_n<NP, true, true>(r, e, none); break;
    }
}

/* pyat/at.c:123: lost if any coordinate is non-finite or |r_n| > 1, n < 5 */
template <class T>
__device__ __forceinline__ bool is_bad(const P6T<T>& r) {
    return !all_finite(r) || fabs(val(r.x)) > 1.0 || fabs(val(r.px)) > 1.0 ||
           fabs(val(r.y)) > 1.0 || fabs(val(r.py)) > 1.0 || fabs(val(r.dp)) > 1.0;
}

__device__ __forceinline__ void load6(const double* src, P6& r) {
    const double2* s = reinterpret_cast<const double2*>(src);
    double2 a = s[0], b = s[1], c = s[2];
    r.x = a.x; r.px = a.y; r.y = b.x; r.py = b.y; r.dp = c.x; r.ct = c.y;
}

/* the same through L2 only: in the serving loop a tile's state may have been
   written by another SM's block since this SM last cached those lines */
__device__ __forceinline__ void load6_cg(const double* src, P6& r) {
    const double2* s = reinterpret_cast<const double2*>(src);
    double2 a = __ldcg(s), b = __ldcg(s + 1), c = __ldcg(s + 2);
    r.x = a.x; r.px = a.y; r.y = b.x; r.py = b.y; r.dp = c.x; r.ct = c.y;
}

__device__ __forceinline__ void store6(double* dst, const P6& r) {
    double2* d = reinterpret_cast<double2*>(dst);
    d[0] = make_double2(r.x, r.px);
    d[1] = make_double2(r.y, r.py);
    d[2] = make_double2(r.dp, r.ct);
}

/* segment index of the q-th segment visited by this launch */
__device__ __forceinline__ int seg_at(const AtbJob& J, long long q) {
    if (q < J.nseg_first) return J.seg_first0 + (int)q;
    return (int)((q - J.nseg_first) % J.nseg_turn);
}

/* ---------------- the kernel --------------------------------------------- */

/* The serving loop's claim (one thread per block).  New work first: the
 * next tile the host has published (taken by compare-and-swap on the counter
 * only while it is below `published`, so a block never holds a claim the host
 * has not published).  Then the continuation rings, class 0 first: a tile
 * that has run a chunk of its job's turns and waits for the next (an entry is
 * taken once its `seq` shows it written).  Without work the block sleeps between looks;
 * it leaves when the host sets `stop`, or after ATB_SERVE_IDLE_NS with
 * nothing claimed anywhere (no tile in flight that could still re-enqueue),
 * or after a hundred times that while tiles are in flight, and in any case
 * after two hundred times that in one claim.  Returns 1 with
 * the tile and the turns of its job already run, or 0 to leave. */
__device__ __forceinline__ int serve_claim(const AtbServeCtl* ctl, int* counter,
                                           const AtbTile* tiles, const AtbServeRing& ring,
                                           int* inflight, int* status, AtbTile* tile,
                                           int* turn_off) {
    uint64_t t0 = global_ns();
    const uint64_t entry = t0;
    while (true) {
        if (ctl->stop) return 0;
        /* a hard bound on the whole claim, whatever resets the idle clock:
           the block leaves and the host launches the kernel again while
           published or re-enqueued work waits */
        if (global_ns() - entry > 200ULL * ATB_SERVE_IDLE_NS) {
            atomicOr(status, ATB_STATUS_IDLE);
            return 0;
        }
        const int pub = ctl->published;
        const int c = atomicAdd(counter, 0);
        if (c < pub) {
            if (atomicCAS(counter, c, c + 1) == c) {
                atomicAdd(inflight, 1);
                __threadfence_system();          /* records read after the flag */
                const int4 tw = __ldcg(reinterpret_cast<const int4*>(tiles + c));
                *tile = *reinterpret_cast<const AtbTile*>(&tw);
                *turn_off = 0;
                return 1;
            }
            continue;                            /* another block took it */
        }
        /* continuations, the lowest class first; an entry reserved by a
           producer and not yet written, or lost to another block, sends the
           claim back to the top */
        bool again = false;
        for (int q = 0; q < ring.nring && !again; ++q) {
            const int h = atomicAdd(ring.head + q, 0);
            const int t = atomicAdd(ring.tail + q, 0);
            if (h >= t) continue;
            const AtbServeCont* e = ring.slots + (size_t)q * ring.cap + (h & (ring.cap - 1));
            if (__ldcg(&e->seq) == h + 1 && atomicCAS(ring.head + q, h, h + 1) == h) {
                atomicAdd(inflight, 1);
                __threadfence();
                const int4 tw = __ldcg(reinterpret_cast<const int4*>(&e->tile));
                *tile = *reinterpret_cast<const AtbTile*>(&tw);
                *turn_off = __ldcg(&e->turn_off);
                return 1;
            }
            again = true;
        }
        if (again) {
            t0 = global_ns();
            continue;
        }
        const bool busy = atomicAdd(inflight, 0) > 0;
        const uint64_t limit = busy ? 100ULL * ATB_SERVE_IDLE_NS : ATB_SERVE_IDLE_NS;
        if (global_ns() - t0 > limit) {
            atomicOr(status, ATB_STATUS_IDLE);
            return 0;
        }
        __nanosleep(4000);
    }
}

/* Put a tile that has run `turn_off` turns of its job back in the
 * continuation ring of class q.  Returns false if that ring is full. */
__device__ __forceinline__ bool serve_requeue(const AtbServeRing& ring, const AtbTile& tile,
                                              int turn_off, int q) {
    q = q < 0 ? 0 : (q >= ring.nring ? ring.nring - 1 : q);
    const int h = atomicAdd(ring.head + q, 0);
    const int t = atomicAdd(ring.tail + q, 0);
    if (t - h >= ring.cap - 64) return false;      /* leave room for racing producers */
    const int idx = atomicAdd(ring.tail + q, 1);
    AtbServeCont* e = ring.slots + (size_t)q * ring.cap + (idx & (ring.cap - 1));
    e->tile = tile;
    e->turn_off = turn_off;
    __threadfence();
    atomicExch(&e->seq, idx + 1);
    return true;
}

#ifndef ATB_NO_TRACK_KERNEL

/* lost-particle marking of one particle after an element (pyat/at.c:115-161) */
__device__ __forceinline__ void apply_loss_rule(const AtbJob& J, P6& r, bool& lost, bool active,
                                                long long p, int nturn, int ei) {
    if (J.losses) {
        if (!lost && is_bad(r)) {
            lost = true;
            if (active) {
                J.lturn[p] = (unsigned)nturn;
                J.lelem[p] = (unsigned)ei;
                store6(J.lcoord + 6 * p, r);
            }
            r.x = nan_d(); r.px = 0.0; r.y = 0.0; r.py = 0.0; r.dp = 0.0; r.ct = 0.0;
        }
    } else if (isfinite(r.x) && is_bad(r)) {
        r.x = nan_d(); r.px = 0.0; r.y = 0.0; r.py = 0.0; r.dp = 0.0; r.ct = 0.0;
    }
}

/* The persistent tile loop.  NP particles per thread: particle k of thread t
 * in a tile is tile.first + k * blockDim + t, so every k stays coalesced; the
 * element parameters read from shared memory serve all NP particles, whose
 * dependency chains interleave.
 *
 * Refill (NP = 1, a compaction scratch area and a job cursor given): a job
 * tracked over whole turns with no refpts snapshots and no per-turn
 * statistics hands out its particles through job_next[job] instead of fixed
 * tile ranges.  At the end of every turn a block retires the particles that
 * were lost or finished their turns (final state and loss flag stored), moves
 * the survivors to its lowest threads when that frees a warp, and takes
 * not-yet-started particles of the same job into its free lanes; each lane
 * counts its own turns (RF phase, loss turn and random kicks use the
 * particle's turn).  Blocks so stay full while their job has particles left
 * instead of running a few survivors for all remaining turns. */
template <int NP, bool GEN = false, bool SERVE = false>
__device__ __forceinline__ void track_tiles(const AtbJob* __restrict__ jobs,
                                            const AtbTile* __restrict__ tiles, int ntiles,
                                            int* __restrict__ tile_counter,
                                            unsigned long long* __restrict__ job_next,
                                            int* __restrict__ status, int smem_cap_words,
                                            double* __restrict__ scratch,
                                            AtbServeArgs sv = AtbServeArgs{}) {
    extern __shared__ __align__(128) double smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_tile;
    /* serving: the claimed tile, the turns of its job already run, the job's
       full turn count, and whether the block keeps its tile for the next
       chunk (continuation ring full) */
    __shared__ AtbTile s_ctile;
    __shared__ int s_toff, s_full, s_self;
    __shared__ unsigned long long s_first;
    __shared__ int s_warp[ATB_MAX_THREADS / 32];
    double* buf0 = smem;
    double* buf1 = smem + smem_cap_words;
    uint32_t use_count[2] = {0u, 0u};
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if constexpr (SERVE) {
        if (tid == 0) s_self = 0;
    }
    __syncthreads();

    int resident_job = -1;   /* job whose whole table sits in buf0 */

    while (true) {
        if (tid == 0) {
            if constexpr (SERVE) {
                if (s_self) s_tile = 1;            /* the same tile, next chunk */
                else s_tile = serve_claim(sv.ctl, tile_counter, tiles, sv.ring, sv.inflight,
                                          status, &s_ctile, &s_toff);
            } else {
                s_tile = atomicAdd(tile_counter, 1);
            }
        }
        __syncthreads();
        const int t = s_tile;
        __syncthreads();
        if constexpr (SERVE) {
            if (t <= 0) break;
        } else {
            if (t >= ntiles) break;
        }
        AtbTile tile;
        const AtbJob* jp;
        if constexpr (SERVE) {
            /* the host writes job records while the kernel runs: read the
               record past the L1 cache into shared memory (only the serving
               kernel has this buffer), then narrow it to this claim's chunk
               of turns, continuing the absolute turn counter */
            __shared__ __align__(16) AtbJob s_job;
            tile = s_ctile;
            const unsigned long long* src =
                reinterpret_cast<const unsigned long long*>(jobs + tile.job);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s_job);
            for (int w = tid; w < (int)(sizeof(AtbJob) / 8); w += nthr) dst[w] = __ldcg(src + w);
            __syncthreads();
            if (tid == 0) {
                const int full = s_job.nturns;
                const int rem = full - s_toff;
                s_full = full;
                s_job.turn0 += s_toff;
                s_job.nturns = (s_job.chunk > 0 && s_job.chunk < rem) ? s_job.chunk : rem;
            }
            __syncthreads();
            jp = &s_job;
        } else {
            tile = tiles[t];
            jp = jobs + tile.job;
        }
        const AtbJob& J = *jp;
        const bool refill =
            NP == 1 && scratch != nullptr && job_next != nullptr && atb_job_refills(&J);
        long long first = tile.first;
        int count = tile.count;
        if (refill) {
            if (tid == 0) s_first = atomicAdd(&job_next[tile.job], (unsigned long long)count);
            __syncthreads();
            first = (long long)s_first;
            const long long left = J.np - first;
            if (left < count) count = left > 0 ? (int)left : 0;
            if (count == 0) continue;   /* the job's particles are all taken */
        }
        long long taken = count;        /* particles this claim stores (serving) */
        long long p[NP];
        bool active[NP];
        int lt0[NP];                    /* turn of the block at which the lane's particle joined */
        int tt_end = J.nturns;          /* the block tracks until this turn */
        bool exhausted = false;         /* the job cursor has no particle left */
        const bool resident = (J.resident != 0);

        P6 r[NP];
        bool lost[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            p[k] = first + (long long)k * nthr + tid;
            active[k] = (k * nthr + tid) < count;
            if constexpr (SERVE) {
                if (J.pidx && active[k]) p[k] = __ldcg(J.pidx + p[k]);
            }
            lt0[k] = 0;
            lost[k] = false;
            if (active[k]) {
                if constexpr (SERVE) {
                    load6_cg(J.r + 6 * p[k], r[k]);
                    if (J.losses) lost[k] = __ldcg(J.lost + p[k]) != 0;
                } else {
                    load6(J.r + 6 * p[k], r[k]);
                    if (J.losses) lost[k] = J.lost[p[k]] != 0;
                }
            } else {
                r[k].x = nan_d(); r[k].px = r[k].py = r[k].y = r[k].dp = r[k].ct = 0.0;
                lost[k] = true;
            }
        }

        /* staging pipeline state for this tile */
        /* segments the tile visits; a refilling block runs until its lanes
           are empty and leaves through the drain below */
        const long long nq = (J.nturns <= 0) ? 0
                             : refill ? (1LL << 60)
                                      : (long long)J.nseg_first +
                                            (long long)(J.nturns - 1) * J.nseg_turn;
        bool timed_out = false;
        if (resident) {
            if (resident_job != tile.job) {
                if (tid == 0) {
                    const uint32_t bytes = (uint32_t)(J.segs[0].nwords * 8);
                    mbar_expect_tx(&bars[0], bytes);
                    bulk_g2s(buf0, J.table + J.segs[0].word0, bytes, &bars[0]);
                }
                bool ok = mbar_wait_bounded(&bars[0], use_count[0] & 1u);
                use_count[0]++;
                timed_out = __syncthreads_or(!ok);
                resident_job = tile.job;
            }
        } else {
            resident_job = -1;
            if (tid == 0) {
                for (int b = 0; b < 2 && b < nq; ++b) {
                    const AtbSeg sg = J.segs[seg_at(J, b)];
                    const uint32_t bytes = (uint32_t)(sg.nwords * 8);
                    mbar_expect_tx(&bars[b], bytes);
                    bulk_g2s(b ? buf1 : buf0, J.table + sg.word0, bytes, &bars[b]);
                }
            }
        }
        if (timed_out) {
            if (tid == 0) atomicOr(status, ATB_STATUS_WAIT_TIMEOUT);
            break;
        }

        long long slot = J.rout_slot0;
        long long q = 0;
        for (int tt = 0; tt < tt_end && !timed_out; ++tt) {
            int nturn[NP];
#pragma unroll
            for (int k = 0; k < NP; ++k) nturn[k] = J.turn0 + tt - lt0[k];
            const int estart = (tt == 0) ? J.start_elem : 0;
            const int eend = J.end_elem;
            int nri = 0;
            unsigned nextref = (nri < J.nref) ? J.refpts[nri++] : 0xffffffffu;
            const int nseg_this = (tt == 0) ? J.nseg_first : J.nseg_turn;
            for (int si = 0; si < nseg_this; ++si, ++q) {
                const int b = resident ? 0 : (int)(q & 1);
                const AtbSeg sg = J.segs[resident ? 0 : seg_at(J, q)];
                const double* base = b ? buf1 : buf0;
                if (!resident) {
                    bool ok = mbar_wait_bounded(&bars[b], use_count[b] & 1u);
                    use_count[b]++;
                    if (__syncthreads_or(!ok)) { timed_out = true; break; }
                }
                /* elements of this segment */
                int e_lo = resident ? estart : sg.first_elem;
                int e_hi = resident ? eend : sg.first_elem + sg.nelem;
                if (e_lo < estart) e_lo = estart;
                if (e_hi > eend) e_hi = eend;
                int w = 0;
                if (resident) {
                    w = J.elem_off[e_lo] - J.elem_off[0];
                } else {
                    w = J.elem_off[e_lo] - J.elem_off[sg.first_elem];
                }
                for (int ei = e_lo; ei < e_hi; ++ei) {
                    Rec e;
                    e.p = base + w;
                    const uint64_t* hp = reinterpret_cast<const uint64_t*>(e.p);
                    e.hdr = hp[0];
                    e.opt = hp[1];
                    if ((unsigned)ei == nextref) {
#pragma unroll
                        for (int k = 0; k < NP; ++k)
                            if (active[k]) store6(J.rout + 6 * (p[k] + J.np * slot), r[k]);
                        ++slot;
                        nextref = (nri < J.nref) ? J.refpts[nri++] : 0xffffffffu;
                    }
                    bool together = false;
                    if constexpr (NP > 1) together = track_together(r, e);
                    if (together) {
                        if constexpr (NP > 1) pass_multipoles_together(r, e);
                    } else {
#pragma unroll
                        for (int k = 0; k < NP; ++k)
                            track_element<GEN>(r[k], e, nturn[k], Param{-1, 0.0}, &J.rng,
                                               p[k], ei);
                    }
#pragma unroll
                    for (int k = 0; k < NP; ++k)
                        if (J.check_loss)
                            apply_loss_rule(J, r[k], lost[k], active[k], p[k], nturn[k], ei);
                    w += e.len();
                }
                if (!resident) {
                    __syncthreads();   /* every thread is done with buffer b */
                    if (tid == 0 && q + 2 < nq) {
                        const AtbSeg nx = J.segs[seg_at(J, q + 2)];
                        const uint32_t bytes = (uint32_t)(nx.nwords * 8);
                        mbar_expect_tx(&bars[b], bytes);
                        bulk_g2s(b ? buf1 : buf0, J.table + nx.word0, bytes, &bars[b]);
                    }
                }
            }
            if (timed_out) break;
            if ((unsigned)J.nelem == nextref) {
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    if (active[k]) store6(J.rout + 6 * (p[k] + J.np * slot), r[k]);
                ++slot;
            }
            if (J.alive) {
                /* per-turn survivors and first/second moments: warp ballot
                 * and shuffle reductions, one atomic per warp */
                unsigned cnt = 0;
                double v[12];
#pragma unroll
                for (int c = 0; c < 12; ++c) v[c] = 0.0;
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    const bool alive = active[k] && !isnan(r[k].x) && !(J.losses && lost[k]);
                    cnt += __popc(__ballot_sync(0xffffffffu, alive));
                    const double c6[6] = {r[k].x, r[k].px, r[k].y, r[k].py, r[k].dp, r[k].ct};
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        const double x = alive ? c6[c] : 0.0;
                        v[c] += x;
                        v[6 + c] += x * x;
                    }
                }
#pragma unroll
                for (int c = 0; c < 12; ++c) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
                }
                if ((tid & 31) == 0) {
                    atomicAdd(&J.alive[tt], cnt);
                    if (J.moments) {
#pragma unroll
                        for (int c = 0; c < 12; ++c) atomicAdd(&J.moments[12 * tt + c], v[c]);
                    }
                }
            }
            /* a tile whose particles are all lost stops early (nothing it
               would still compute is observable without refpts snapshots) */
            if (refill || (J.nref == 0 && tt + 1 < tt_end)) {
                if constexpr (NP == 1) {
                    if (refill && active[0]) {
                        /* retire a particle that is lost or has done its turns */
                        const bool done = tt + 1 - lt0[0] == J.nturns;
                        if (done || isnan(r[0].x) || (J.losses && lost[0])) {
                            store6(J.r + 6 * p[0], r[0]);
                            if (J.losses) J.lost[p[0]] = lost[0] ? 1 : 0;
                            active[0] = false;
                            r[0].x = nan_d(); r[0].px = 0.0; r[0].y = 0.0;
                            r[0].py = 0.0; r[0].dp = 0.0; r[0].ct = 0.0;
                            lost[0] = true;
                        }
                    }
                }
                bool any_live = false;
#pragma unroll
                for (int k = 0; k < NP; ++k)
                    any_live |= active[k] && !isnan(r[k].x) && !(J.losses && lost[k]);
                int nlive = __syncthreads_count(any_live);
                if constexpr (NP == 1) {
                    const bool live = any_live;
                    const unsigned ball = __ballot_sync(0xffffffffu, live);
                    const int lane = tid & 31, warp = tid >> 5;
                    /* warps that still hold a live particle */
                    const int held = __syncthreads_count(lane == 0 && ball != 0u);
                    if (scratch && nlive > 0 && (nlive + 31) / 32 < held) {
                        /* The survivors fit in fewer warps than hold them:
                           move them to the lowest threads, so that whole
                           warps fall idle instead of running with masked
                           lanes.  The lost ones are retired first (their
                           final state and loss flag are what the end of the
                           tile would store). */
                        if (active[0] && !live) {
                            store6(J.r + 6 * p[0], r[0]);
                            if (J.losses) J.lost[p[0]] = lost[0] ? 1 : 0;
                        }
                        if (lane == 0) s_warp[warp] = __popc(ball);
                        __syncthreads();
                        int dest = __popc(ball & ((1u << lane) - 1u));
                        for (int wv = 0; wv < warp; ++wv) dest += s_warp[wv];
                        double* sb = scratch + (size_t)blockIdx.x * ATB_COMPACT_WORDS * nthr;
                        if (live) {
                            sb[dest] = r[0].x;
                            sb[nthr + dest] = r[0].px;
                            sb[2 * nthr + dest] = r[0].y;
                            sb[3 * nthr + dest] = r[0].py;
                            sb[4 * nthr + dest] = r[0].dp;
                            sb[5 * nthr + dest] = r[0].ct;
                            sb[6 * nthr + dest] = __longlong_as_double(p[0]);
                            sb[7 * nthr + dest] = __longlong_as_double(lt0[0]);
                        }
                        __syncthreads();
                        active[0] = tid < nlive;
                        if (active[0]) {
                            r[0].x = sb[tid];
                            r[0].px = sb[nthr + tid];
                            r[0].y = sb[2 * nthr + tid];
                            r[0].py = sb[3 * nthr + tid];
                            r[0].dp = sb[4 * nthr + tid];
                            r[0].ct = sb[5 * nthr + tid];
                            p[0] = __double_as_longlong(sb[6 * nthr + tid]);
                            lt0[0] = (int)__double_as_longlong(sb[7 * nthr + tid]);
                            lost[0] = false;
                        } else {
                            r[0].x = nan_d(); r[0].px = 0.0; r[0].y = 0.0;
                            r[0].py = 0.0; r[0].dp = 0.0; r[0].ct = 0.0;
                            lost[0] = true;
                        }
                        __syncthreads();   /* scratch free for the next compaction */
                    }
                    if (refill && !exhausted) {
                        /* free lanes take the job's next particles */
                        const bool fr = !active[0];
                        const unsigned fb = __ballot_sync(0xffffffffu, fr);
                        if (lane == 0) s_warp[warp] = __popc(fb);
                        const int nfree = __syncthreads_count(fr);
                        if (nfree > 0) {
                            if (tid == 0)
                                s_first = atomicAdd(&job_next[tile.job],
                                                    (unsigned long long)nfree);
                            __syncthreads();
                            const long long c = (long long)s_first;
                            long long take = J.np - c;
                            if (take > nfree) take = nfree;
                            if (take < nfree) exhausted = true;
                            if (take > 0) {
                                int rank = __popc(fb & ((1u << lane) - 1u));
                                for (int wv = 0; wv < warp; ++wv) rank += s_warp[wv];
                                if (fr && rank < take) {
                                    p[0] = c + rank;
                                    active[0] = true;
                                    lt0[0] = tt + 1;
                                    load6(J.r + 6 * p[0], r[0]);
                                    lost[0] = J.losses ? J.lost[p[0]] != 0 : false;
                                }
                                nlive += (int)take;
                                taken += take;
                                if (tt + 1 + J.nturns > tt_end) tt_end = tt + 1 + J.nturns;
                            }
                            __syncthreads();   /* s_warp and s_first free again */
                        }
                    }
                }
                if (nlive == 0) {
                    if (!resident) {
                        /* wait for the copies this tile has in flight: after q
                           consumed segments, segments [0, min(nq, q + 2)) were
                           issued, buffer b holding the ones with index % 2 == b */
                        const long long issued = (q + 2 < nq) ? q + 2 : nq;
                        for (int b = 0; b < 2; ++b) {
                            long long pending = (issued - b + 1) / 2 - (q - b + 1) / 2;
                            for (; pending > 0; --pending) {
                                if (!mbar_wait_bounded(&bars[b], use_count[b] & 1u))
                                    timed_out = true;
                                use_count[b]++;
                            }
                        }
                        __syncthreads();
                    }
                    break;
                }
            }
        }
        if (timed_out) {
            /* drain our own copies still in flight before leaving */
            if (!resident) {
                const long long issued = (q + 2 < nq) ? q + 2 : nq;
                for (int b = 0; b < 2; ++b) {
                    if (use_count[b] < (uint32_t)((issued + 1 - b) / 2)) {
                        mbar_wait_bounded(&bars[b], use_count[b] & 1u);
                    }
                }
            }
            if (tid == 0) atomicOr(status, ATB_STATUS_WAIT_TIMEOUT);
            break;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            if (active[k]) {
                store6(J.r + 6 * p[k], r[k]);
                if (J.losses) J.lost[p[k]] = lost[k] ? 1 : 0;
            }
        }
        if constexpr (SERVE) {
            /* the chunk is stored and visible device-wide: a tile with live
               particles and turns left goes back to the continuation ring
               (or, if the ring is full, stays with this block); otherwise its
               particles count as done.  With a particle index (NP = 1) the
               tile keeps only its live particles, their indices packed at
               the front of its range, and the others count as done now. */
            __threadfence();
            bool live = false;
#pragma unroll
            for (int k = 0; k < NP; ++k)
                live |= active[k] && !isnan(r[k].x) && !(J.losses && lost[k]);
            const int nlive = __syncthreads_count(live);
            const bool more = nlive > 0 && s_toff + J.nturns < s_full;
            int keep_count = count;
            if (NP == 1 && J.pidx && more && nlive < count) {
                const unsigned ball = __ballot_sync(0xffffffffu, live);
                const int lane = tid & 31, warp = tid >> 5;
                if (lane == 0) s_warp[warp] = __popc(ball);
                __syncthreads();
                if (tid == 0) {
                    int acc = 0;
                    for (int w = 0; w < (nthr + 31) / 32; ++w) {
                        const int c = s_warp[w];
                        s_warp[w] = acc;
                        acc += c;
                    }
                }
                __syncthreads();
                if (live) {
                    const int rank = s_warp[warp] + __popc(ball & ((1u << lane) - 1u));
                    J.pidx[tile.first + rank] = (int32_t)p[0];
                }
                __threadfence();
                __syncthreads();
                keep_count = nlive;
            }
            if (tid == 0) {
                const int ran = s_toff + J.nturns;
                bool requeued = false, keep = false;
                if (more && !sv.ctl->stop) {
                    AtbTile nt = tile;
                    nt.count = keep_count;
                    /* class: decade of the tile's remaining time, so that
                       tiles near their end go first */
                    const double key = (double)(s_full - ran) * J.turn_cost;
                    const int q = key >= 1.0 ? (int)floor(log10(key)) : 0;
                    requeued = serve_requeue(sv.ring, nt, ran, q);
                    if (!requeued) {
                        atomicOr(status, ATB_STATUS_RING_FULL);
                        keep = true;
                        s_toff = ran;
                        s_ctile = nt;
                    }
                }
                if (requeued || keep) {
                    if (keep_count < taken)
                        atomicAdd(&sv.done[tile.job], (unsigned long long)(taken - keep_count));
                } else if (!more) {
                    atomicAdd(&sv.done[tile.job], (unsigned long long)taken);
                }
                if (!keep) atomicSub(sv.inflight, 1);
                s_self = keep ? 1 : 0;
            }
        }
        /* all threads must be past the last segment before the buffers are
           re-filled by the next tile */
        __syncthreads();
    }
}

extern "C" __global__ void __launch_bounds__(ATB_MAX_THREADS)
ATB_CAT(atb_track_kernel, ATB_KSUFFIX)(const AtbJob* __restrict__ jobs,
                                       const AtbTile* __restrict__ tiles, int ntiles,
                                       int* __restrict__ tile_counter,
                                       unsigned long long* __restrict__ job_next,
                                       int* __restrict__ status, int smem_cap_words,
                                       double* __restrict__ scratch) {
    track_tiles<1>(jobs, tiles, ntiles, tile_counter, job_next, status, smem_cap_words,
                   scratch);
}

/* with the other integrators of the GPU call (tables with ATB_F_INTEG) */
extern "C" __global__ void __launch_bounds__(ATB_MAX_THREADS)
ATB_CAT(ATB_CAT(atb_track_kernel, ATB_KSUFFIX), _gen)(const AtbJob* __restrict__ jobs,
                                                      const AtbTile* __restrict__ tiles,
                                                      int ntiles, int* __restrict__ tile_counter,
                                                      unsigned long long* __restrict__ job_next,
                                                      int* __restrict__ status,
                                                      int smem_cap_words,
                                                      double* __restrict__ scratch) {
    track_tiles<1, true>(jobs, tiles, ntiles, tile_counter, job_next, status, smem_cap_words,
                         scratch);
}

/* The serving loop's persistent kernel: new tiles come from a queue the host
   appends to while it runs (AtbServeCtl), continuations from the device-side
   ring; `done[job]` counts the particles of each job that have run all their
   turns (or were lost) and are back in memory.  No lane refill: a tile keeps
   its particles from chunk to chunk. */
extern "C" __global__ void __launch_bounds__(ATB_MAX_THREADS)
ATB_CAT(atb_serve_kernel, ATB_KSUFFIX)(const AtbJob* __restrict__ jobs,
                                       const AtbTile* __restrict__ tiles, AtbServeArgs sv,
                                       int* __restrict__ tile_counter, int* __restrict__ status,
                                       int smem_cap_words, double* __restrict__ scratch) {
    track_tiles<1, false, true>(jobs, tiles, 0, tile_counter, nullptr, status, smem_cap_words,
                                scratch, sv);
}

/* two particles per thread (the autotuner's particles-per-thread choice) */
extern "C" __global__ void __launch_bounds__(ATB_MAX_THREADS)
ATB_CAT(ATB_CAT(atb_track_kernel, ATB_KSUFFIX), _np2)(const AtbJob* __restrict__ jobs,
                                                      const AtbTile* __restrict__ tiles,
                                                      int ntiles, int* __restrict__ tile_counter,
                                                      unsigned long long* __restrict__ job_next,
                                                      int* __restrict__ status,
                                                      int smem_cap_words,
                                                      double* __restrict__ scratch) {
    track_tiles<2>(jobs, tiles, ntiles, tile_counter, job_next, status, smem_cap_words,
                   scratch);
}

#endif  // ATB_NO_TRACK_KERNEL

}  // namespace atb

#endif  // ATB_TRACK_KERNEL_CUH
