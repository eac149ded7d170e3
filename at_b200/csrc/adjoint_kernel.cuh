/*
 * The adjoint kernels: reverse-mode derivatives of multi-turn tracking.
 *
 * For a scalar function of the final coordinates, L = sum_p g_p . r_p(T),
 * one backward sweep gives dL/d r_p(0) for every particle and dL/dK_q for
 * every differentiated strength K_q = PolynomB[k_q] of an element, whatever
 * the number of strengths (the tangent kernel carries one derivative
 * direction per input instead).  This is the vector-Jacobian product that a
 * torch.autograd backward pass needs.
 *
 * Forward (atb_adjoint_forward_kernel): the particles are tracked with the
 * strengths substituted, by the same pass-method code as every other kernel
 * of this unit ("exact" arithmetic, so the values equal the exact tracking
 * kernel's), and the state entering every stride-th turn is stored.
 *
 * Backward (atb_adjoint_turn_kernel, one launch per turn, last turn first):
 * from the turn's entry state the turn is tracked again, every element's
 * entry state going to a scratch array ([element][particle][6], coalesced)
 * -- or, when the forward pass stored every turn's element-entry states
 * (memory permitting), those are read instead;
 * then the elements are walked backwards with lambda <- J_e^T lambda, J_e
 * the element's Jacobian at its stored entry state, and at an element that
 * carries K_q, dL/dK_q += (d r_out / d K_q) . lambda_out, summed over the
 * block's particles in shared memory and added to the global sum once per
 * block.
 *
 * Element adjoints:
 *  - DriftPass, IdentityPass, AperturePass, RFCavityPass, thin
 *    CorrectorPass, ThinMPolePass and the non-radiating StrMPole/BndMPole
 *    Symplectic4 passes (plain or bend-edge entrance/exit, misaligned or
 *    not): written out by hand.  In a thick magnet the
 *    (x, px, y, py) entering each integration step are recomputed from the
 *    element's entry state into a per-thread store in shared memory (every step up to
 *    ATB_ADJ_STEPS steps, every ceil(n / ATB_ADJ_STEPS)-th beyond, the rest
 *    recomputed from the nearest), each step is re-run with the inputs of its
 *    seven stages kept in registers, and the stages are reversed: the
 *    fastdrift (driftkick.c:37-48), and the kick (driftkick.c:51-115) with the
 *    field derivative F'(z) of F(z) = sum (B_n + i A_n) z^n from a second
 *    Horner recursion and dF/dB_k = z^k for the strength.
 *  - every other element (radiating magnets, quadrupole fringes, field
 *    scaling, thick correctors, bend edges of method 3): J_e from a forward-mode evaluation of the whole element on dual
 *    numbers (6 directions, 7 when the element carries a strength), out of
 *    line so that its registers do not weigh on the common path.
 * A particle that is lost (NaN, or lost during the turn) gets a NaN
 * cotangent and adds nothing to the strengths' gradient.
 */
#ifndef ATB_ADJOINT_KERNEL_CUH
#define ATB_ADJOINT_KERNEL_CUH

#include "track_kernel.cuh"

namespace atb {

/* integration-step entry states kept per thread, in shared memory */
#define ATB_ADJ_STEPS ATB_ADJ_STEPS_SMEM

/* A thread's step-entry store in the block's shared memory: entry c,
 * component k (x, px, y, py) at base[(4 c + k) * stride], stride the block
 * size, so a warp's accesses fall on consecutive words. */
struct StepStore {
    double* base;
    int stride;
    __device__ __forceinline__ double& at(int c, int k) const {
        return base[(4 * c + k) * stride];
    }
};
#ifndef ATB_ADJ_MIN_BLOCKS
#define ATB_ADJ_MIN_BLOCKS 4   /* 128 registers a thread: the dual-number
                                  fallback spills, the common path does not */
#endif

struct Lam6 {
    double v[6];
    double g;          /* the element's strength gradient contribution */
};

__device__ __forceinline__ Param adj_param(const AtbAdjoint& A, int ei) {
    Param pm{-1, 0.0};
    if (A.pelem) {
        const int q = A.pelem[ei];
        if (q >= 0) { pm.k = A.porder[q]; pm.v = A.pvalue[q]; }
    }
    return pm;
}

__device__ __forceinline__ Rec adj_rec(const AtbAdjoint& A, int ei) {
    Rec e;
    e.p = A.table + A.elem_off[ei];
    const uint64_t* hp = reinterpret_cast<const uint64_t*>(e.p);
    e.hdr = hp[0];
    e.opt = hp[1];
    return e;
}

/* ---- transposed linear maps --------------------------------------------- */

/* lambda <- R^T lambda for the misalignment rotation of mult_r */
__device__ __forceinline__ void adj_mult_r(double* lam, const double* m, bool dense) {
    if (dense) {
        double o[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < 6; ++i) s = fma(m[i + 6 * j], lam[i], s);
            o[j] = s;
        }
#pragma unroll
        for (int j = 0; j < 6; ++j) lam[j] = o[j];
    } else {
        /* x' = m0 x + m1 y, px' = m2 px + m3 py, y' = m4 x + m5 y,
           py' = m6 px + m7 py */
        const double lx = lam[0], lpx = lam[1], ly = lam[2], lpy = lam[3];
        lam[0] = fma(m[0], lx, m[4] * ly);
        lam[2] = fma(m[1], lx, m[5] * ly);
        lam[1] = fma(m[2], lpx, m[6] * lpy);
        lam[3] = fma(m[3], lpx, m[7] * lpy);
    }
}

__device__ __forceinline__ void adj_exit_misalign(double* lam, const Rec& e) {
    if (const double* r2 = e.blk(ATB_OPT_R2)) adj_mult_r(lam, r2, e.flags() & ATB_F_R2_DENSE);
}

__device__ __forceinline__ void adj_entrance_misalign(double* lam, const Rec& e) {
    if (const double* r1 = e.blk(ATB_OPT_R1)) adj_mult_r(lam, r1, e.flags() & ATB_F_R1_DENSE);
}

/* ---- drift --------------------------------------------------------------- */

/* drift6 at input s: x += nl px, y += nl py, ct += nl pn S / 2 with
 * pn = 1/(1+dp), nl = L pn, S = px^2 + py^2 */
__device__ __forceinline__ void adj_drift6(const P6& s, double* lam, double L) {
    const double pn = 1.0 / (1.0 + s.dp);
    const double nl = L * pn;
    const double lx = lam[0], ly = lam[2], lc = lam[5];
    const double S = fma(s.px, s.px, s.py * s.py);
    const double cp = lc * nl * pn;
    lam[1] += fma(lx, nl, cp * s.px);
    lam[3] += fma(ly, nl, cp * s.py);
    lam[4] -= L * pn * pn * fma(lx, s.px, fma(ly, s.py, lc * pn * S));
}

/* DriftPass.c:16-48 */
__device__ __forceinline__ void adj_pass_drift(const P6& s, double* lam, const Rec& e) {
    P6 r = s;
    entrance_misalign(r, e);
    adj_exit_misalign(lam, e);
    adj_drift6(r, lam, e.f(ATB_DR_LE));
    adj_entrance_misalign(lam, e);
}

/* ---- thick multipoles ---------------------------------------------------- */

/* The element's multipole coefficients for the reverse pass, B_sk replaced
 * by the differentiated strength kv: in registers for MaxOrder MO in 0..3,
 * read from the table for MO = -1 (any order).  field() is F(z) =
 * sum_n (B_n + i A_n) z^n by Horner's rule with fused multiply-adds (the
 * recomputed steps inside an element only feed derivatives, so they need not
 * round as the tracking does); prime() is F'(z) by the same recursion. */
template <int MO>
struct AdjCoef {
    double a[MO + 1], b[MO + 1];
    int sk;
    __device__ __forceinline__ void load(const double* A, const double* B, int, int k,
                                         double v) {
#pragma unroll
        for (int i = 0; i <= MO; ++i) {
            a[i] = A[i];
            b[i] = (i == k) ? v : B[i];
        }
        sk = k;
    }
    __device__ __forceinline__ void field(double x, double y, double& re, double& im) const {
        re = b[MO];
        im = a[MO];
#pragma unroll
        for (int i = MO - 1; i >= 0; --i) {
            const double t = fma(re, x, fma(-im, y, b[i]));
            im = fma(im, x, fma(re, y, a[i]));
            re = t;
        }
    }
    __device__ __forceinline__ void prime(double x, double y, double& dr, double& di) const {
        if constexpr (MO == 0) {
            dr = 0.0;
            di = 0.0;
        } else {
            dr = (double)MO * b[MO];
            di = (double)MO * a[MO];
#pragma unroll
            for (int n = MO - 1; n >= 1; --n) {
                const double t = fma(dr, x, fma(-di, y, (double)n * b[n]));
                di = fma(di, x, fma(dr, y, (double)n * a[n]));
                dr = t;
            }
        }
    }
};

template <>
struct AdjCoef<-1> {
    const double* a;
    const double* b;
    int mo;
    int sk;
    double kv;
    __device__ __forceinline__ void load(const double* A, const double* B, int m, int k,
                                         double v) {
        a = A; b = B; mo = m; sk = k; kv = v;
    }
    __device__ __forceinline__ double bk(int i) const { return (i == sk) ? kv : b[i]; }
    __device__ __forceinline__ void field(double x, double y, double& re, double& im) const {
        re = bk(mo);
        im = a[mo];
        for (int i = mo - 1; i >= 0; --i) {
            const double t = fma(re, x, fma(-im, y, bk(i)));
            im = fma(im, x, fma(re, y, a[i]));
            re = t;
        }
    }
    __device__ __forceinline__ void prime(double x, double y, double& dr, double& di) const {
        if (mo <= 0) {
            dr = 0.0;
            di = 0.0;
            return;
        }
        dr = (double)mo * bk(mo);
        di = (double)mo * a[mo];
        for (int n = mo - 1; n >= 1; --n) {
            const double t = fma(dr, x, fma(-di, y, (double)n * bk(n)));
            di = fma(di, x, fma(dr, y, (double)n * a[n]));
            dr = t;
        }
    }
};

/* (x + i y)^k */
__device__ __forceinline__ void zpow(double x, double y, int k, double& zr, double& zi) {
    zr = 1.0;
    zi = 0.0;
    for (int i = 0; i < k; ++i) {
        const double t = fma(zr, x, -zi * y);
        zi = fma(zr, y, zi * x);
        zr = t;
    }
}

/* strthinkick / bndthinkick of length L at input (x, y):
 * px -= L (Re F - [bend] (dp - x irho) irho), py += L Im F,
 * [bend] ct += lirho x */
template <bool BEND, int MO>
__device__ __forceinline__ void adj_kick(const AdjCoef<MO>& c, double x, double y, double L,
                                         double lirho, double irho, double* lam, double& g) {
    double dr, di;
    c.prime(x, y, dr, di);
    const double lpx = lam[1], lpy = lam[3];
    double ax = L * fma(-dr, lpx, di * lpy);
    const double ay = L * fma(di, lpx, dr * lpy);
    if (BEND) {
        ax = fma(-L * irho * irho, lpx, fma(lirho, lam[5], ax));
        lam[4] = fma(L * irho, lpx, lam[4]);
    }
    lam[0] += ax;
    lam[2] += ay;
    if (c.sk >= 0) {
        double zr, zi;
        zpow(x, y, c.sk, zr, zi);
        g = fma(L, fma(-zr, lpx, zi * lpy), g);
    }
}

/* fastdrift (exact form) at input (px, py): x += nl px, y += nl py,
 * ct += nl S h with h = 1/(2 (1 + dp)); nl = L/(1 + dp_entry) is a function
 * of the element's entry momentum, collected in lnl */
__device__ __forceinline__ void adj_fastdrift(double px, double py, double h, double nl,
                                              double* lam, double& lnl) {
    const double lx = lam[0], ly = lam[2], lc = lam[5];
    const double S = fma(px, px, py * py);
    const double c2 = 2.0 * lc * nl * h;
    lam[1] += fma(lx, nl, c2 * px);
    lam[3] += fma(ly, nl, c2 * py);
    lam[4] -= c2 * S * h;
    lnl += fma(lx, px, fma(ly, py, lc * S * h));
}

/* The transverse coordinates inside a non-radiating magnet, where dp is
 * constant and ct feeds nothing: what the recomputed steps carry. */
struct XY {
    double x, px, y, py;
};

__device__ __forceinline__ void xy_drift(XY& q, double nl) {
    q.x = fma(nl, q.px, q.x);
    q.y = fma(nl, q.py, q.y);
}

template <bool BEND, int MO>
__device__ __forceinline__ void xy_kick(XY& q, const AdjCoef<MO>& c, double L, double irho,
                                        double dp) {
    double re, im;
    c.field(q.x, q.y, re, im);
    if (BEND) re = fma(-fma(-q.x, irho, dp), irho, re);     /* re - (dp - x irho) irho */
    q.px = fma(-L, re, q.px);
    q.py = fma(L, im, q.py);
}

/* one Forest-Ruth step (StrMPoleSymplectic4Pass.c:73-93) on the transverse
 * coordinates */
template <bool BEND, int MO>
__device__ __forceinline__ void xy_step(XY& q, const AdjCoef<MO>& c, double nl1, double nl2,
                                        double K1, double K2, double irho, double dp) {
    xy_drift(q, nl1);
    xy_kick<BEND>(q, c, K1, irho, dp);
    xy_drift(q, nl2);
    xy_kick<BEND>(q, c, K2, irho, dp);
    xy_drift(q, nl2);
    xy_kick<BEND>(q, c, K1, irho, dp);
    xy_drift(q, nl1);
}

/* edge_fringe (methods other than 3, exact arithmetic) at input s:
 * px += x fx, py -= y fy(dp) with fy = tn or tn/(1+dp) (method 2),
 * tn = irho tan(edge - fc/(1+dp)) (fy_c when that argument is the edge) */
__device__ __forceinline__ void adj_edge(const P6& s, double* lam, double irho, double edge,
                                         double fc, double fx, double fy_c, int method) {
    const double opd = 1.0 + s.dp;
    const double t = edge - fc / opd;
    const double tn = (t == edge) ? fy_c : irho * tan(t);
    double dtn = 0.0;
    if (fc != 0.0) {
        const double tt = tan(t);
        dtn = irho * fma(tt, tt, 1.0) * fc / (opd * opd);
    }
    double fy = tn, dfy = dtn;
    if (method == ATB_BM_2) {
        fy = tn / opd;
        dfy = (dtn - fy) / opd;
    }
    lam[0] = fma(lam[1], fx, lam[0]);
    lam[4] = fma(-lam[3] * s.y, dfy, lam[4]);
    lam[2] = fma(-lam[3], fy, lam[2]);
}

/* the hand-written magnet path applies (flags and edge methods) */
__device__ __forceinline__ bool adj_by_hand(const Rec& e, bool bend) {
    const uint32_t fl = e.flags();
    if (fl & (ATB_F_SCALING | ATB_F_FQ_IN | ATB_F_FQ_OUT | ATB_F_INTEG)) return false;
    if (bend) {
        const int m_in = (int)((fl >> ATB_F_BM_IN_SHIFT) & ATB_F_BM_MASK);
        const int m_out = (int)((fl >> ATB_F_BM_OUT_SHIFT) & ATB_F_BM_MASK);
        if (m_in == ATB_BM_3 || m_out == ATB_BM_3) return false;
    }
    return true;
}

/* StrMPoleSymplectic4Pass.c:29-109 / BndMPoleSymplectic4Pass.c:38-129 in
 * reverse; `ss` is the thread's step-entry store.  The entry transforms run
 * in the tracking arithmetic from the stored entry state; the steps are
 * recomputed on the transverse coordinates. */
template <bool BEND, int MO>
__device__ __forceinline__ void adj_multipole_mo(const P6& s, double* lam, const Rec& e,
                                                 const Param& pm, double& g,
                                                 const StepStore& ss) {
    const uint32_t fl = e.flags();
    const double L1 = e.f(ATB_SM_L1), L2 = e.f(ATB_SM_L2);
    const double K1 = e.f(ATB_SM_K1), K2 = e.f(ATB_SM_K2);
    const int mo = e.mo();
    const double* A = e.p + (BEND ? ATB_BM_POLY : ATB_SM_POLY);
    AdjCoef<MO> c;
    c.load(A, A + mo + 1, mo, pm.k, pm.v);

    /* forward to every step entry */
    P6 r = s;
    const double pn0 = 1.0 / (1.0 + r.dp);
    const double nl1 = L1 * pn0, nl2 = L2 * pn0;
    entrance_misalign(r, e);
    const P6 s_in = r;                       /* entering the entrance edge */
    double irho = 0.0, k1i = 0.0, k2i = 0.0;
    int m_in = 0, m_out = 0;
    if (BEND) {
        irho = e.f(ATB_BM_IRHO);
        k1i = e.f(ATB_BM_K1IRHO);
        k2i = e.f(ATB_BM_K2IRHO);
        m_in = (int)((fl >> ATB_F_BM_IN_SHIFT) & ATB_F_BM_MASK);
        m_out = (int)((fl >> ATB_F_BM_OUT_SHIFT) & ATB_F_BM_MASK);
        edge_fringe<false>(r, irho, e.f(ATB_BM_EIN), e.f(ATB_BM_FCIN), e.f(ATB_BM_FXIN),
                           e.f(ATB_BM_FYIN), m_in, fl & ATB_F_FC0_IN, 1.0);
    }
    const double dp = r.dp;                  /* constant through the steps */
    const double h = 1.0 / (2.0 * (1.0 + dp));
    const int ns = e.nsteps();
    const int stride = ns > ATB_ADJ_STEPS ? (ns + ATB_ADJ_STEPS - 1) / ATB_ADJ_STEPS : 1;
    XY q{r.x, r.px, r.y, r.py};
    for (int m = 0; m < ns; ++m) {
        if (m % stride == 0) {
            const int c = m / stride;
            ss.at(c, 0) = q.x; ss.at(c, 1) = q.px; ss.at(c, 2) = q.y; ss.at(c, 3) = q.py;
        }
        xy_step<BEND>(q, c, nl1, nl2, K1, K2, irho, dp);
    }

    /* reverse */
    adj_exit_misalign(lam, e);
    if (BEND) {
        P6 so;
        so.x = q.x; so.px = q.px; so.y = q.y; so.py = q.py; so.dp = dp; so.ct = 0.0;
        adj_edge(so, lam, irho, e.f(ATB_BM_EOUT), e.f(ATB_BM_FCOUT), e.f(ATB_BM_FXOUT),
                 e.f(ATB_BM_FYOUT), m_out);
    }
    double lnl1 = 0.0, lnl2 = 0.0;
    for (int m = ns - 1; m >= 0; --m) {
        const int cb = m / stride;
        XY t{ss.at(cb, 0), ss.at(cb, 1), ss.at(cb, 2), ss.at(cb, 3)};
        for (int j = cb * stride; j < m; ++j) xy_step<BEND>(t, c, nl1, nl2, K1, K2, irho, dp);
        /* the step once more, keeping the input of every stage */
        const double px0 = t.px, py0 = t.py;
        xy_drift(t, nl1);
        const double x1 = t.x, y1 = t.y;
        xy_kick<BEND>(t, c, K1, irho, dp);
        const double px2 = t.px, py2 = t.py;
        xy_drift(t, nl2);
        const double x3 = t.x, y3 = t.y;
        xy_kick<BEND>(t, c, K2, irho, dp);
        const double px4 = t.px, py4 = t.py;
        xy_drift(t, nl2);
        const double x5 = t.x, y5 = t.y;
        xy_kick<BEND>(t, c, K1, irho, dp);
        const double px6 = t.px, py6 = t.py;
        adj_fastdrift(px6, py6, h, nl1, lam, lnl1);
        adj_kick<BEND>(c, x5, y5, K1, k1i, irho, lam, g);
        adj_fastdrift(px4, py4, h, nl2, lam, lnl2);
        adj_kick<BEND>(c, x3, y3, K2, k2i, irho, lam, g);
        adj_fastdrift(px2, py2, h, nl2, lam, lnl2);
        adj_kick<BEND>(c, x1, y1, K1, k1i, irho, lam, g);
        adj_fastdrift(px0, py0, h, nl1, lam, lnl1);
    }
    if (BEND)
        adj_edge(s_in, lam, irho, e.f(ATB_BM_EIN), e.f(ATB_BM_FCIN), e.f(ATB_BM_FXIN),
                 e.f(ATB_BM_FYIN), m_in);
    adj_entrance_misalign(lam, e);
    /* nl1, nl2 = L1, L2 / (1 + dp) of the entry momentum */
    lam[4] -= fma(lnl1, L1, lnl2 * L2) * pn0 * pn0;
}

template <bool BEND>
__device__ __forceinline__ void adj_pass_multipole(const P6& s, double* lam, const Rec& e,
                                                   const Param& pm, double& g,
                                                   const StepStore& ss) {
    switch (e.mo()) {
        case 0: adj_multipole_mo<BEND, 0>(s, lam, e, pm, g, ss); break;
        case 1: adj_multipole_mo<BEND, 1>(s, lam, e, pm, g, ss); break;
        case 2: adj_multipole_mo<BEND, 2>(s, lam, e, pm, g, ss); break;
        case 3: adj_multipole_mo<BEND, 3>(s, lam, e, pm, g, ss); break;
        default: adj_multipole_mo<BEND, -1>(s, lam, e, pm, g, ss); break;
    }
}

/* ---- thin elements -------------------------------------------------------- */

/* rf_kick at input s: dp -= nv sin(tf ((ct - lag)/c - ht nturn) - phi) */
__device__ __forceinline__ void adj_rf_kick(const P6& s, double* lam, const Rec& e, int nturn) {
    const double nv = e.f(ATB_RF_NV), tf = e.f(ATB_RF_TF), lag = e.f(ATB_RF_LAG);
    const double ht = e.f(ATB_RF_HT), phi = e.f(ATB_RF_PHI);
    const double a = tf * ((s.ct - lag) / ATB_C0 - ht * (double)nturn) - phi;
    lam[5] = fma(-nv * cos(a) * tf / ATB_C0, lam[4], lam[5]);
}

/* RFCavityPass.c:23-68 (trackRFCavity, attrackfunc.c:5-42) */
__device__ __forceinline__ void adj_pass_rfcavity(const P6& s, double* lam, const Rec& e,
                                                  int nturn) {
    const uint32_t fl = e.flags();
    if (!(fl & ATB_F_THICK)) {
        if (fl & ATB_F_NV) adj_rf_kick(s, lam, e, nturn);
        return;
    }
    const double half = e.f(ATB_RF_HALF);
    P6 r = s;
    drift6<false>(r, half);
    const P6 s1 = r;
    if (fl & ATB_F_NV) rf_kick(r, e, nturn);
    adj_drift6(r, lam, half);
    if (fl & ATB_F_NV) adj_rf_kick(s1, lam, e, nturn);
    adj_drift6(s, lam, half);
}

/* ThinMPolePass.c:28-70 without field scaling */
__device__ __forceinline__ void adj_pass_thinmpole(const P6& s, double* lam, const Rec& e,
                                                   const Param& pm, double& g) {
    const int mo = e.mo();
    const double* A = e.p + ATB_TM_POLY;
    const double* B = A + mo + 1;
    const double bax = e.f(ATB_TM_BAX), bay = e.f(ATB_TM_BAY);
    P6 r = s;
    entrance_misalign(r, e);
    adj_exit_misalign(lam, e);
    /* px += bax dp, py -= bay dp, ct -= bax x - bay y */
    lam[4] = fma(bax, lam[1], fma(-bay, lam[3], lam[4]));
    lam[0] = fma(-bax, lam[5], lam[0]);
    lam[2] = fma(bay, lam[5], lam[2]);
    AdjCoef<-1> c;
    c.load(A, B, mo, pm.k, pm.v);
    adj_kick<false>(c, r.x, r.y, 1.0, 0.0, 0.0, lam, g);
    adj_entrance_misalign(lam, e);
}

/* ---- any element: forward mode on dual numbers --------------------------- */

template <int K>
__device__ __forceinline__ Lam6 adj_dual(const P6& s, const Lam6& in, const Rec& e, int nturn,
                                         const Param& pm) {
    using D = Dual<K>;
    P6T<D> r;
    r.x = D(s.x); r.px = D(s.px); r.y = D(s.y);
    r.py = D(s.py); r.dp = D(s.dp); r.ct = D(s.ct);
    r.x.d[0] = 1.0; r.px.d[1] = 1.0; r.y.d[2] = 1.0;
    r.py.d[3] = 1.0; r.dp.d[4] = 1.0; r.ct.d[5] = 1.0;
    track_element(r, e, nturn, pm);
    const D* rows[6] = {&r.x, &r.px, &r.y, &r.py, &r.dp, &r.ct};
    Lam6 out;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double a = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) a = fma(in.v[i], rows[i]->d[j], a);
        out.v[j] = a;
    }
    out.g = 0.0;
    if constexpr (K == 7) {
#pragma unroll
        for (int i = 0; i < 6; ++i) out.g = fma(in.v[i], rows[i]->d[6], out.g);
    }
    return out;
}

__device__ __noinline__ Lam6 adj_dual6(P6 s, Lam6 in, Rec e, int nturn) {
    return adj_dual<6>(s, in, e, nturn, Param{-1, 0.0});
}

__device__ __noinline__ Lam6 adj_dual7(P6 s, Lam6 in, Rec e, int nturn, Param pm) {
    return adj_dual<7>(s, in, e, nturn, pm);
}

/* lambda <- J_e(s)^T lambda; g += the strength's term */
__device__ __forceinline__ void adj_element(const P6& s, double* lam, const Rec& e, int nturn,
                                            const Param& pm, double& g, const StepStore& ss) {
    switch (e.op()) {
        case ATB_OP_DRIFT: adj_pass_drift(s, lam, e); return;
        case ATB_OP_IDENTITY:
            adj_exit_misalign(lam, e);
            adj_entrance_misalign(lam, e);
            return;
        case ATB_OP_APERTURE:
        case ATB_OP_QUANTDIFF: return;      /* identity for a surviving particle */
        case ATB_OP_RFCAVITY: adj_pass_rfcavity(s, lam, e, nturn); return;
        case ATB_OP_CORRECTOR:
            if (!(e.flags() & (ATB_F_THICK | ATB_F_SCALING))) {   /* px += xk, py += yk */
                adj_exit_misalign(lam, e);
                adj_entrance_misalign(lam, e);
                return;
            }
            break;
        case ATB_OP_THINMPOLE:
            if (!(e.flags() & ATB_F_SCALING)) { adj_pass_thinmpole(s, lam, e, pm, g); return; }
            break;
        case ATB_OP_STRMPOLE:
            if (adj_by_hand(e, false)) { adj_pass_multipole<false>(s, lam, e, pm, g, ss); return; }
            break;
        case ATB_OP_BNDMPOLE:
            if (adj_by_hand(e, true)) { adj_pass_multipole<true>(s, lam, e, pm, g, ss); return; }
            break;
        default: break;
    }
    Lam6 in;
#pragma unroll
    for (int i = 0; i < 6; ++i) in.v[i] = lam[i];
    in.g = 0.0;
    const Lam6 out = pm.k >= 0 ? adj_dual7(s, in, e, nturn, pm) : adj_dual6(s, in, e, nturn);
#pragma unroll
    for (int i = 0; i < 6; ++i) lam[i] = out.v[i];
    g += out.g;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* ---- kernels ------------------------------------------------------------- */

extern "C" __global__ void __launch_bounds__(ATB_ADJ_THREADS)
atb_adjoint_forward_kernel(const AtbAdjoint A) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    P6 r;
    load6(A.r + 6 * p, r);
    bool lost = isnan(r.x);
    for (int tt = 0; tt < A.nturns; ++tt) {
        if (A.ckpt && tt % A.stride == 0)
            store6(A.ckpt + 6 * ((long long)(tt / A.stride) * A.ld + p), r);
        if (lost || (A.skip_last && tt == A.nturns - 1)) continue;
        const int nturn = A.turn0 + tt;
        for (int ei = 0; ei < A.nelem; ++ei) {
            if (A.scratch)
                store6(A.scratch + 6 * (((long long)tt * A.nelem + ei) * A.ld + p), r);
            track_element(r, adj_rec(A, ei), nturn, adj_param(A, ei));
            if (is_bad(r)) {                  /* pyat/at.c:115-139 */
                lost = true;
                break;
            }
        }
        if (lost) {
            r.x = nan_d(); r.px = 0.0; r.y = 0.0; r.py = 0.0; r.dp = 0.0; r.ct = 0.0;
        }
    }
    store6(A.r + 6 * p, r);
    if (A.lost) A.lost[p] = lost ? 1 : 0;
}

extern "C" __global__ void __launch_bounds__(ATB_ADJ_THREADS, ATB_ADJ_MIN_BLOCKS)
atb_adjoint_turn_kernel(const AtbAdjoint A) {
    /* the block's strength gradient (nparam words), then the threads' step
       stores (ATB_ADJ_STEPS x 4 x blockDim words) */
    extern __shared__ double sg[];
    for (int q = threadIdx.x; q < A.nparam; q += blockDim.x) sg[q] = 0.0;
    __syncthreads();
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = p < A.np;
    const long long np = A.np;
    P6 s;
    double lam[6];
    bool live = false;
    if (in) {
        load6(A.ckpt + 6 * p, s);
#pragma unroll
        for (int i = 0; i < 6; ++i) lam[i] = A.lam[6 * p + i];
        live = !isnan(s.x);
#pragma unroll
        for (int i = 0; i < 6; ++i) live &= isfinite(lam[i]);
    }
    if (A.next) {
        /* the forward pass stored this turn's element-entry states; a
           particle lost during the turn enters the next one as NaN */
        if (live) live = !isnan(__ldg(A.next + 6 * p));
    } else {
        /* the turn once more, every element's entry state to the scratch */
        for (int ei = 0; ei < A.nelem; ++ei) {
            if (live) {
                store6(A.scratch + 6 * ((long long)ei * np + p), s);
                track_element(s, adj_rec(A, ei), A.turn0, adj_param(A, ei));
                if (is_bad(s)) live = false;      /* lost in this turn */
            }
        }
    }
    const StepStore ss{sg + A.nparam + threadIdx.x, (int)blockDim.x};
    for (int ei = A.nelem - 1; ei >= 0; --ei) {
        const Param pm = adj_param(A, ei);
        double g = 0.0;
        if (live) {
            P6 se;
            load6(A.scratch + 6 * ((long long)ei * np + p), se);
            adj_element(se, lam, adj_rec(A, ei), A.turn0, pm, g, ss);
        }
        if (pm.k >= 0) {                      /* the same for the whole block */
            g = warp_sum(g);
            if ((threadIdx.x & 31) == 0) atomicAdd(&sg[A.pelem[ei]], g);
        }
    }
    if (in) {
        const double nan = nan_d();
#pragma unroll
        for (int i = 0; i < 6; ++i) A.lam[6 * p + i] = live ? lam[i] : nan;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < A.nparam; q += blockDim.x)
        if (sg[q] != 0.0) atomicAdd(&A.gparam[q], sg[q]);
}

}  // namespace atb

#endif  // ATB_ADJOINT_KERNEL_CUH
