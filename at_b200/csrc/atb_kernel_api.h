/*
 * Launch-side data structures of the tracking kernel (device and host).
 *
 * A launch processes a list of tiles; each tile is a contiguous run of at
 * most blockDim particles of one job.  A job is one (lattice, particle set,
 * turn range) triple with its output buffers, so the same kernel serves the
 * plain drop-in call (one job), batched lattice variants (one job per
 * variant) and the serving loop (one job per admitted request).
 */
#ifndef ATB_KERNEL_API_H
#define ATB_KERNEL_API_H

#include <stdint.h>

#define ATB_MAX_THREADS 512
/* doubles per thread in the survivor-compaction scratch area: the six
   coordinates, the particle index and the turn at which it joined */
#define ATB_COMPACT_WORDS 8
/* bounded mbarrier wait: 1 s, then the kernel reports and returns */
#define ATB_WAIT_NS 1000000000ULL
#define ATB_STATUS_WAIT_TIMEOUT 1
#define ATB_STATUS_INTEGRATOR 2   /* an element compiled for another integrator
                                     reached a kernel built without them */
#define ATB_STATUS_IDLE 4         /* the serving kernel left after waiting
                                     ATB_SERVE_IDLE_NS without new work */
/* the serving kernel waits this long for new work, then leaves (the host
   launches it again when work arrives) */
#define ATB_SERVE_IDLE_NS 200000000ULL

/* Control words of the serving loop, in host memory mapped into the device's
 * address space.  The host writes job and tile records into device memory,
 * waits for those copies, then raises `published` (the number of tiles the
 * kernel may claim); it sets `stop` to let the kernel leave once every
 * published tile is claimed. */
typedef struct AtbServeCtl {
    volatile int32_t published;
    volatile int32_t stop;
} AtbServeCtl;

typedef struct AtbTile {
    int32_t job;
    int32_t count;
    int64_t first;
} AtbTile;

/* A tile that has run one chunk of its job's turns and waits for the next:
   written by the block that ran it into the serving loop's continuation ring
   (device memory), `seq` (its ring index + 1) last, after a fence.  32 bytes,
   so that every entry's tile is 16-byte aligned for its vector load. */
typedef struct AtbServeCont {
    AtbTile tile;
    int32_t turn_off;           /* turns of the job already run             */
    int32_t seq;
    int64_t pad;
} AtbServeCont;

/* The serving loop's device-side queue: one continuation ring per priority
   class (class 0 first) and their cursors (device memory). */
#define ATB_SERVE_CLASSES 8

typedef struct AtbServeRing {
    AtbServeCont* slots;        /* nring rings of cap entries               */
    int32_t cap;                /* entries per ring (power of two)          */
    int32_t nring;
    int* head;                  /* per ring: next entry to claim            */
    int* tail;                  /* per ring: next entry to write            */
} AtbServeRing;

#define ATB_STATUS_RING_FULL 8    /* a continuation found the ring full and
                                     ran its remaining turns in place */

/* Everything the serving kernel shares with the host besides the tile and
   job arrays. */
typedef struct AtbServeArgs {
    const AtbServeCtl* ctl;     /* mapped host memory                       */
    AtbServeRing ring;
    int* inflight;              /* tiles claimed and not yet finished       */
    unsigned long long* done;   /* per job: particles finished              */
} AtbServeArgs;

/* one staged lattice segment: consecutive element records */
typedef struct AtbSeg {
    int32_t first_elem;
    int32_t nelem;
    int64_t word0;     /* first word in the table (16-byte aligned)        */
    int32_t nwords;    /* words copied (even)                              */
    int32_t pad;
} AtbSeg;

/* The quantum-diffusion kicks of a job: the normals of its particle p are
 * a function of (key, pbase + p, turn, element), pbase placing the job's
 * particles in a larger set that the host tracks in parts. */
typedef struct AtbRng {
    uint64_t key;
    int64_t pbase;
} AtbRng;

typedef struct AtbJob {
    const double* table;        /* element table words                      */
    const AtbSeg* segs;         /* segment list                             */
    const uint32_t* elem_off;   /* word offset of every element (+ end)     */
    int32_t nelem;
    int32_t resident;           /* whole table in one buffer                */
    int32_t seg_first0;         /* first segment of the first turn          */
    int32_t nseg_first;         /* segments visited in the first turn       */
    int32_t nseg_turn;          /* segments visited in later turns          */
    int32_t check_loss;         /* 0 for single-element tracking            */
    double* r;                  /* (6, np) Fortran-order state              */
    int64_t np;
    int32_t turn0;              /* absolute turn number of the first turn   */
    int32_t nturns;
    int32_t start_elem;         /* first element of the first turn          */
    int32_t end_elem;           /* one past the last element of every turn  */
    const uint32_t* refpts;
    int32_t nref;
    int32_t losses;             /* 1: loss map (checkiflost), 0: setlost    */
    double* rout;               /* (6, np, slots) snapshots                 */
    int64_t rout_slot0;
    uint8_t* lost;              /* loss map (losses == 1)                   */
    uint32_t* lturn;
    uint32_t* lelem;
    double* lcoord;
    uint32_t* alive;            /* optional: survivors after each turn     */
    double* moments;            /* optional: 12 sums per turn              */
    AtbRng rng;                 /* quantum-diffusion kicks                  */
    int32_t chunk;              /* serving: turns per claim, 0 all (a tile
                                   re-enqueues itself for the rest)         */
    int32_t pad_serve;
    double turn_cost;           /* serving: relative cost of one turn; a
                                   continuation's class is the decade of
                                   (turns left) x turn_cost, 0: one class   */
    int32_t* pidx;              /* serving, optional: the particle at each
                                   tile position; a re-enqueued tile keeps
                                   only its live particles, packed first    */
} AtbJob;

/* Whether a job's particles may be handed out through a per-job cursor with
 * lanes refilled at turn boundaries (the tracking kernel's refill, used with
 * one particle per thread when the launch provides compaction scratch and
 * job cursors): whole turns, no refpts snapshots, no per-turn statistics,
 * loss checks on, at least one table segment per turn.  Shared by the kernel
 * and the host, which may then issue fewer claims than tiles for the job. */
#ifdef __CUDACC__
__host__ __device__
#endif
static inline int atb_job_refills(const AtbJob* J) {
    return J->nref == 0 && J->alive == 0 && J->check_loss && J->start_elem == 0 &&
           J->end_elem == J->nelem && J->nturns > 0 && J->nturns < (1 << 30) &&
           J->nseg_turn > 0 && J->nseg_first == J->nseg_turn;
}

/* Tangent (forward-mode) tracking: one launch over np particles of one
 * lattice, with the Jacobian of the final coordinates with respect to the
 * initial ones and to nparam multipole strengths. */
#define ATB_TANGENT_THREADS 128

typedef struct AtbTangent {
    const double* table;        /* element table words                      */
    const uint32_t* elem_off;   /* word offset of every element (+ end)     */
    int32_t nelem;
    int32_t nturns;
    int32_t turn0;
    int32_t nparam;
    double* r;                  /* (6, np) state, updated in place          */
    int64_t np;
    const int32_t* pelem;       /* per element: parameter index or -1       */
    const int32_t* porder;      /* per parameter: PolynomB order            */
    const double* pvalue;       /* per parameter: strength used             */
    double* jac;                /* (np, 6, 6): d r_i / d r0_j               */
    double* grad;               /* (nparam, 6, np): d r_i / d K_q           */
    uint8_t* lost;              /* optional (np): 1 if the particle was lost */
} AtbTangent;

/* Adjoint (reverse-mode) tracking, one thread per particle.  The forward
 * kernel tracks `nturns` turns with the differentiated strengths substituted
 * and stores the state entering every `stride`-th turn in `ckpt`
 * ((turns / stride, ld, 6) slabs).  The turn kernel runs the adjoint of one
 * turn (absolute number turn0) from its entry states `ckpt` ((np, 6)): it
 * re-tracks the turn storing every element's entry state in `scratch`
 * ((nelem, np, 6)), then maps the cotangent `lam` ((np, 6), in place) from
 * the turn's exit to its entry and adds the strengths' gradient to
 * `gparam`. */
#define ATB_ADJ_THREADS 128
#define ATB_ADJ_STEPS_SMEM 10      /* step entries a thread keeps in shared memory */

typedef struct AtbAdjoint {
    const double* table;        /* element table words                      */
    const uint32_t* elem_off;   /* word offset of every element (+ end)     */
    int32_t nelem;
    int32_t nturns;             /* forward: turns tracked                   */
    int32_t turn0;              /* absolute number of the first turn        */
    int32_t stride;             /* forward: a checkpoint every stride turns */
    const int32_t* pelem;       /* per element: parameter index or -1       */
    const int32_t* porder;      /* per parameter: PolynomB order            */
    const double* pvalue;       /* per parameter: strength used             */
    int32_t nparam;
    int32_t skip_last;          /* forward: store the last turn's entry, do
                                   not track it                             */
    int64_t np;
    int64_t ld;                 /* forward: particles per checkpoint slab   */
    double* r;                  /* forward: (np, 6) state, in place         */
    double* ckpt;               /* forward: out; turn kernel: entry states  */
    uint8_t* lost;              /* forward: optional loss flags (np)        */
    double* lam;                /* turn kernel: (np, 6) cotangent           */
    double* scratch;            /* turn kernel: (nelem, np, 6) element-entry
                                   states; forward, optional: every turn's
                                   ((nturns, nelem, ld, 6)), stored as the
                                   particles pass                          */
    double* gparam;             /* turn kernel: (nparam), added to          */
    const double* next;         /* turn kernel, states stored by the forward
                                   pass: the (np, 6) states entering the next
                                   turn (NaN: lost in this one); NULL: the
                                   kernel tracks the turn again itself      */
} AtbAdjoint;

/* Per-element transfer and diffusion matrices for a particle entering each
 * element at orbits[6 * i]: one thread per element. */
typedef struct AtbElemMaps {
    const double* table;
    const uint32_t* elem_off;
    int32_t nelem;
    int32_t pad;
    const double* orbits;       /* (nelem, 6)                               */
    double* m66;                /* (nelem, 6, 6) row-major: d out_i / d in_j */
    double* b66;                /* (nelem, 6, 6) row-major diffusion matrix */
    double diff_const;          /* DIF_CONST * gamma^5                      */
    double* exits;              /* (nelem, 6) exit coordinates, or NULL     */
} AtbElemMaps;

#endif /* ATB_KERNEL_API_H */
