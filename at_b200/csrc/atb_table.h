/*
 * Flat element table ("lattice program") shared by the host lattice compiler
 * (at_b200/lattice.py) and the tracking kernel (track_kernel.cuh).
 *
 * A compiled lattice is one array of 64-bit words.  Element i occupies the
 * words [offset[i], offset[i] + len_i).  Every record starts with two integer
 * words (stored bit-cast in the double array):
 *
 *   word 0  : opcode (bits 0-5) | max_order (6-11) | flags (12-31)
 *             | num_int_steps (32-47) | record length in words (48-63)
 *   word 1  : word offsets, relative to the record start, of the optional
 *             blocks T1, R1, RApertures, EApertures, R2, T2, FRINGE
 *             (9 bits each, 0 = absent)
 *   word 2+ : opcode-specific doubles at the fixed positions below, then the
 *             PolynomA[0..max_order] and PolynomB[0..max_order] coefficients
 *             (multipole opcodes), then the optional blocks.
 *
 * Per-element invariants are folded on the host with the same IEEE double
 * operations, in the same order, as the reference integrators evaluate them
 * (e.g. atintegrators/StrMPoleSymplectic4Pass.c:39-52), so the per-particle
 * arithmetic left on the device sees bit-identical constants.  Records are
 * padded to an even number of words so each starts on a 16-byte boundary.
 */
#ifndef ATB_TABLE_H
#define ATB_TABLE_H

/* ---- opcodes (one per supported PassMethod) ---------------------------- */
#define ATB_OP_IDENTITY      0   /* IdentityPass.c                        */
#define ATB_OP_DRIFT         1   /* DriftPass.c                           */
#define ATB_OP_STRMPOLE      2   /* StrMPoleSymplectic4Pass.c             */
#define ATB_OP_STRMPOLE_RAD  3   /* StrMPoleSymplectic4RadPass.c          */
#define ATB_OP_BNDMPOLE      4   /* BndMPoleSymplectic4Pass.c             */
#define ATB_OP_BNDMPOLE_RAD  5   /* BndMPoleSymplectic4RadPass.c          */
#define ATB_OP_THINMPOLE     6   /* ThinMPolePass.c                       */
#define ATB_OP_RFCAVITY      7   /* RFCavityPass.c / attrackfunc.c        */
#define ATB_OP_CORRECTOR     8   /* CorrectorPass.c                       */
#define ATB_OP_APERTURE      9   /* AperturePass.c                        */
#define ATB_OP_QUANTDIFF    10   /* QuantDiffPass.c                       */
#define ATB_NUM_OPS         11

/* ---- header word 0 packing --------------------------------------------- */
#define ATB_H_OP_SHIFT     0
#define ATB_H_OP_MASK      63u
#define ATB_H_MO_SHIFT     6
#define ATB_H_MO_MASK      63u
#define ATB_H_FL_SHIFT     12
#define ATB_H_FL_MASK      0xfffffu
#define ATB_H_NS_SHIFT     32
#define ATB_H_NS_MASK      0xffffu
#define ATB_H_LEN_SHIFT    48
#define ATB_H_LEN_MASK     0xffffu

/* ---- flag bits ---------------------------------------------------------- */
#define ATB_F_SCALING      (1u << 0)   /* FieldScaling != 1.0              */
#define ATB_F_R1_DENSE     (1u << 1)   /* R1 is a general 6x6              */
#define ATB_F_R2_DENSE     (1u << 2)   /* R2 is a general 6x6              */
#define ATB_F_FQ_IN        (1u << 3)   /* quad fringe at entrance          */
#define ATB_F_FQ_IN_LIN    (1u << 4)   /*   ... with the linear elegant maps */
#define ATB_F_FQ_OUT       (1u << 5)   /* quad fringe at exit              */
#define ATB_F_FQ_OUT_LIN   (1u << 6)
#define ATB_F_THICK        (1u << 7)   /* Corrector / RFCavity length != 0 */
#define ATB_F_NV           (1u << 8)   /* RFCavity voltage != 0            */
#define ATB_F_FC0_IN       (1u << 9)   /* bend entrance fringecorr == 0    */
#define ATB_F_FC0_OUT      (1u << 10)  /* bend exit fringecorr == 0        */
#define ATB_F_BM_IN_SHIFT  11          /* bend entrance method, 2 bits     */
#define ATB_F_BM_OUT_SHIFT 13          /* bend exit method, 2 bits         */
#define ATB_F_BM_MASK      3u
#define ATB_F_FINT_IN      (1u << 15)  /* bend entrance FringeInt1 > 0 and FullGap > 0
                                          (the diffusion-matrix edge term)  */
#define ATB_F_FINT_OUT     (1u << 16)  /* bend exit FringeInt2 > 0 and FullGap > 0 */
#define ATB_F_NOSKEW       (1u << 17)  /* thick multipole: every PolynomA
                                          coefficient (KickAngle folded) is 0 */
#define ATB_F_INTEG        (1u << 18)  /* thick multipole integrated by the
                                          integrator whose id (1-6) is stored at
                                          ATB_SM_INTEG, with step ATB_SM_SL */
/* bend fringe "method" codes after host normalisation (atphyslib.c:15-79) */
#define ATB_BM_LEGACY      0   /* method 0 or any value other than 1,2,3   */
#define ATB_BM_1           1
#define ATB_BM_2           2
#define ATB_BM_3           3

/* ---- word-1 optional block slots --------------------------------------- */
#define ATB_OPT_T1      0
#define ATB_OPT_R1      1
#define ATB_OPT_RAP     2
#define ATB_OPT_EAP     3
#define ATB_OPT_R2      4
#define ATB_OPT_T2      5
#define ATB_OPT_FRINGE  6   /* 32 words: entrance maps M1, M2; exit M1, M2   */
#define ATB_NUM_OPT     7
#define ATB_OPT_BITS    9
#define ATB_OPT_MASK    511u

/* a rotation-only ("tilt") R block holds R[0,0],R[0,2],R[1,1],R[1,3],
   R[2,0],R[2,2],R[3,1],R[3,3]; every other entry is 0 except R[4,4]=R[5,5]=1 */
#define ATB_R_TILT_WORDS  8
#define ATB_R_DENSE_WORDS 36
/* each linear quad-fringe map: x-plane 2x2 (m00,m01,m10,m11), y-plane 2x2   */
#define ATB_FRINGE_WORDS  32

/* ---- fixed field positions (word index inside the record) -------------- */
#define ATB_W_HDR   0
#define ATB_W_OPT   1

/* DRIFT */
#define ATB_DR_LE      2

/* STRMPOLE / STRMPOLE_RAD */
#define ATB_SM_L1      2
#define ATB_SM_L2      3
#define ATB_SM_K1      4
#define ATB_SM_K2      5
#define ATB_SM_SCALE   6   /* FieldScaling                                   */
#define ATB_SM_ISCALE  7   /* 1.0/FieldScaling                               */
#define ATB_SM_B1      8   /* PolynomB[1] as seen by the quad fringe         */
#define ATB_SM_RADC    9   /* RAD_CONST*gamma^3 (Rad variants)               */
#define ATB_SM_POLY   10   /* A[0..n], then B[0..n]                          */
/* with ATB_F_INTEG set, the Forest-Ruth words carry the step and the id */
#define ATB_SM_SL     ATB_SM_L1   /* Length/NumIntSteps                     */
#define ATB_SM_ONE    ATB_SM_L2   /* 1.0: the entrance L2 x 1/(1+delta) is then
                                     1/(1+delta) itself                     */
#define ATB_SM_INTEG  ATB_SM_K1   /* integrator id, as a double             */

/* BNDMPOLE / BNDMPOLE_RAD share words 2-9 with STRMPOLE                     */
#define ATB_BM_IRHO    10
#define ATB_BM_K1IRHO  11  /* K1*irho                                        */
#define ATB_BM_K2IRHO  12  /* K2*irho                                        */
#define ATB_BM_EIN     13  /* entrance edge angle                            */
#define ATB_BM_FCIN    14  /* entrance fringecorr (psi for the Rad variant)  */
#define ATB_BM_FXIN    15  /* irho*tan(edge)                                 */
#define ATB_BM_FYIN    16  /* irho*tan(edge) (used when fringecorr == 0)     */
#define ATB_BM_EOUT    17
#define ATB_BM_FCOUT   18
#define ATB_BM_FXOUT   19
#define ATB_BM_FYOUT   20
#define ATB_BM_POLY    22  /* keeps A/B 16-byte aligned                      */

/* THINMPOLE */
#define ATB_TM_BAX     2
#define ATB_TM_BAY     3
#define ATB_TM_SCALE   4
#define ATB_TM_ISCALE  5
#define ATB_TM_POLY    6

/* RFCAVITY */
#define ATB_RF_LE      2
#define ATB_RF_NV      3   /* Voltage/Energy                                 */
#define ATB_RF_TF      4   /* TWOPI*Frequency                                */
#define ATB_RF_LAG     5   /* TimeLag                                        */
#define ATB_RF_HT      6   /* HarmNumber/Frequency - T0                      */
#define ATB_RF_PHI     7   /* PhaseLag                                       */
#define ATB_RF_HALF    8   /* Length/2                                       */

/* CORRECTOR */
#define ATB_CO_XK      2
#define ATB_CO_YK      3
#define ATB_CO_LE      4
#define ATB_CO_SCALE   5
#define ATB_CO_ISCALE  6
#define ATB_CO_K2      7   /* xkick*xkick/3 + ykick*ykick/3                  */
#define ATB_CO_HX      8   /* xkick/2                                        */
#define ATB_CO_HY      9   /* ykick/2                                        */

/* APERTURE */
#define ATB_AP_LIM     2   /* 4 limits                                       */

/* QuantDiffPass: the 6x6 Lmatp, column-major ([i][j] at i + 6 j) */
#define ATB_QD_L       2

#define ATB_MAX_RECORD_WORDS 511
#define ATB_MAX_ORDER 40

#endif /* ATB_TABLE_H */
