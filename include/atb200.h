/*
 * atb200 -- C ABI of the B200 particle-tracking engine.
 *
 * Plain C types only (pointers, sizes, status codes); no Python, NumPy or
 * torch types cross this boundary.  Every entry point returns ATB_OK (0) or a
 * negative ATB_ERR_* code and never aborts; atb_last_error() gives the
 * message of the calling thread's last failure.
 *
 * What each entry point replaces in the reference (atcollab/at):
 *   atb_lattice_upload   the lattice cache that pyat/at.c builds on a
 *                        non-reuse call (pyat/at.c:445-512) and the per-element
 *                        `struct elem` set-up of every trackFunction
 *                        (atintegrators/atelem.c:373-374, e.g.
 *                        StrMPoleSymplectic4Pass.c:112-166): the host compiles
 *                        the elements into one flat table (atb_table.h) and
 *                        this call makes it device-resident.
 *   atb_track            at_atpass (pyat/at.c:340-681) / at_gpupass
 *                        (atgpu/PyInterface.cpp:132-402): multi-turn tracking
 *                        of a 6xN Fortran-ordered particle array, in place,
 *                        with refpts snapshots (6,N,R,T) and the loss map.
 *                        With ATB_FLAG_ELEMENT it is at_elempass
 *                        (pyat/at.c:683-753): one pass, no loss marking.
 *   atb_device_count /   at_gpuinfo (atgpu/PyInterface.cpp:95-129).
 *   atb_device_info
 */
#ifndef ATB200_H
#define ATB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATB_OK 0
#define ATB_ERR_ARG (-1)      /* invalid argument                          */
#define ATB_ERR_CUDA (-2)     /* CUDA runtime error                        */
#define ATB_ERR_TIMEOUT (-3)  /* a bounded in-kernel wait gave up          */
#define ATB_ERR_NOMEM (-4)    /* device memory budget exceeded             */
#define ATB_ERR_NOLAT (-5)    /* unknown lattice id                        */

#define ATB_MODE_EXACT 0      /* reference operation order, no FMA (the
                                 Python layer's default)                  */
#define ATB_MODE_FAST 1       /* FMA + reciprocal reuse                    */

#define ATB_FLAG_ELEMENT 1    /* single-element pass: no loss marking      */

typedef struct atb_handle atb_handle;

/* One job of a batched launch (lattice variant x particle set). Device
 * pointers.  rout/refpts are not supported in batches. */
typedef struct atb_job_desc {
    int32_t lattice_id;
    int32_t nturns;
    int32_t turn0;
    int32_t losses;
    double* r;            /* (6, np) Fortran order, device                */
    int64_t np;
    uint8_t* islost;      /* device, np (losses == 1)                      */
    uint32_t* lturn;
    uint32_t* lelem;
    double* lcoord;       /* device, 6*np                                  */
} atb_job_desc;

/* library version (major*10000 + minor*100 + patch) */
int atb_version(void);

/* message of the calling thread's last failing call ("" if none) */
const char* atb_last_error(void);

/* at_gpuinfo (atgpu/PyInterface.cpp:95-129): device count and properties */
int atb_device_count(int* count);
int atb_device_info(int device, char* name, int name_len, int* cc_major, int* cc_minor,
                    int* sm_count, uint64_t* total_mem);

/* An engine bound to one device, with its own stream and buffers.  Not
 * re-entrant: one host thread at a time per handle (the reference's atpass
 * keeps static state too, pyat/at.c:62-75). */
int atb_create(int device, atb_handle** out);
int atb_destroy(atb_handle* h);

/* Refill factor of prepared batches (atb_batch_prepare), 1..64, default 8:
 * a job tracked over whole turns without refpts snapshots or per-turn
 * statistics starts on one block per k tiles' worth of its particles, and
 * each block takes the job's remaining particles into the lanes that lost or
 * finished particles free at turn boundaries (halved until the launch has
 * two claims per resident block).  It pays where many particles are lost
 * early (dynamic-aperture studies over lattice variants) and costs where
 * they survive, so atb_track_batch keeps one claim per tile.  Results do not
 * depend on it.  Refused while prepared batches exist.  No reference
 * counterpart (launch tuning). */
int atb_set_refill_factor(atb_handle* h, int32_t k);

/* Particles per thread of the tracking kernel (1 or 2): with 2, each thread
 * carries two particles through every element, reusing the element's
 * parameters and interleaving two dependency chains; the autotuner picks it.
 * Small particle sets that would not fill the SMs use 1.  Refused while
 * prepared batches exist.  No reference counterpart (launch tuning). */
int atb_set_particles_per_thread(atb_handle* h, int32_t ppt);

/* Launch tuning: threads per block (32..512, multiple of 32), shared-memory
 * segment capacity in 8-byte words, largest table kept resident in shared
 * memory, and the device-memory budget for refpts snapshots.  0 keeps the
 * current value. */
int atb_set_launch(atb_handle* h, int threads_per_block, int seg_cap_words,
                   int resident_max_words, int64_t rout_budget_bytes);

/* Make a compiled lattice (flat table of atb_table.h: `nwords` words, element
 * i at words [elem_off[i], elem_off[i+1])) device-resident.  Replaces the
 * reference's lattice cache (pyat/at.c:445-512). */
int atb_lattice_upload(atb_handle* h, const double* words, int64_t nwords,
                       const uint32_t* elem_off, int32_t nelem, int32_t* lattice_id);

/* Overwrite the words of an uploaded lattice (same layout), e.g. after the
 * energy-dependent fields were refreshed for a new ring energy. */
int atb_lattice_update(atb_handle* h, int32_t lattice_id, const double* words, int64_t nwords);

int atb_lattice_free(atb_handle* h, int32_t lattice_id);

/* at_atpass / at_gpupass.  All pointers are HOST memory:
 *   rin     (6, np) Fortran order, updated in place (pyat/at.c:555,633)
 *   refpts  nref uint32 element indices (sorted, as get_uint32_index gives)
 *   rout    (6, np, nref, nturns) Fortran order, or NULL when nref == 0
 *   losses  1: fill islost/lturn/lelem/lcoord (pyat/at.c:574-594,664-677)
 *   alive   optional (nturns) survivors after each turn, or NULL
 *   moments optional (nturns, 12): sums of the 6 coordinates and of their
 *           squares over survivors after each turn, or NULL
 * turn0 is the reference's param.nturn at the first turn (the `turn` or kept
 * counter, pyat/at.c:428-431); start_elem/end_elem as pyat/at.c:514-536.
 * The snapshots pass through a device buffer of at most the handle's
 * snapshot budget (atb_set_launch, 4 GB by default): the turns are tracked
 * in chunks whose snapshots fit it, and when one turn of all particles' does
 * not, the particles in groups (same results; ATB_ERR_NOMEM only if one
 * particle's turn exceeds the budget).  Blocks until the results are back in
 * host memory. */
int atb_track(atb_handle* h, int32_t lattice_id, double* rin, int64_t np, int32_t nturns,
              int32_t turn0, int32_t start_elem, int32_t end_elem, const uint32_t* refpts,
              int32_t nref, double* rout, int32_t losses, uint8_t* islost, uint32_t* lturn,
              uint32_t* lelem, double* lcoord, uint32_t* alive, double* moments, int32_t mode,
              int32_t flags);

/* The same with DEVICE pointers (particles already resident in HBM), enqueued
 * on `stream` (NULL: the handle's stream) without host synchronisation; no
 * refpts.  Kernel status is reported by the next atb_sync(). */
int atb_track_device(atb_handle* h, int32_t lattice_id, double* r, int64_t np, int32_t nturns,
                     int32_t turn0, int32_t losses, uint8_t* islost, uint32_t* lturn,
                     uint32_t* lelem, double* lcoord, uint32_t* alive, double* moments,
                     int32_t mode, void* stream);

/* Tangent tracking (device pointers, enqueued on `stream`, NULL: the
 * handle's stream): tracks the (6, np) particles `r` in place for `nturns`
 * whole turns in the exact arithmetic and writes the exact derivatives of
 * the final coordinates, jac (np, 6, 6) = d r_i / d r0_j and grad
 * (nparam, 6, np) = d r_i / d K_q, for nparam multipole strengths
 * K_q = PolynomB[param_order[q]] of element param_elem[q] (host arrays; one
 * strength per element, order in [1, MaxOrder]).  The strengths used are
 * read from param_value (device, nparam), which replaces the table's values
 * for those coefficients, so a caller can move them without re-uploading the
 * lattice.  Lost particles come back NaN in r, jac and grad (islost, optional,
 * marks them).  The lattice must be compiled for the default integrator
 * (ATB_ERR_ARG otherwise).  Replaces the finite-difference Jacobian of
 * pyat/at/physics/matrix.py:105-165 (find_m66) and the finite differences a
 * caller of lattice_pass would take for strength sensitivities; the
 * reference has no exact-derivative tracking. */
int atb_tangent_device(atb_handle* h, int32_t lattice_id, double* r, int64_t np, int32_t nturns,
                       int32_t turn0, const int32_t* param_elem, const int32_t* param_order,
                       const double* param_value, int32_t nparam, double* jac, double* grad,
                       uint8_t* islost, void* stream);

/* Adjoint (reverse-mode) tracking, device pointers, enqueued on `stream`
 * (NULL: the handle's stream); strengths as for atb_tangent_device.
 *   atb_adjoint_forward   tracks the (6, np) particles `r` in place for
 *       `nturns` whole turns (exact arithmetic, the strengths param_value
 *       substituted) and, when ckpt is not NULL, stores the state entering
 *       turns 0, stride, 2 stride, ... in ckpt ((ceil(nturns / stride), np, 6)).
 *       Lost particles come back NaN (islost, optional, marks them).  With
 *       estates (device, nturns x nelem x np x 6 doubles; stride must be 1)
 *       it also stores every element's entry state of every turn, which
 *       spares the backward sweep its re-tracking.
 *   atb_adjoint_backward  from those checkpoints (same np, nturns, turn0,
 *       stride and strengths) and the cotangent lam = dL/d r_final
 *       ((6, np), in place), writes lam = dL/d r_initial and
 *       gparam (nparam) = dL/dK_q = sum over particles, for any scalar L of
 *       the final coordinates: one backward sweep, one launch per turn, whose
 *       cost does not grow with the number of strengths.  With stride > 1
 *       each block of turns is tracked again from its checkpoint.  With the
 *       forward pass's estates (and rfinal, its final states) nothing is
 *       tracked again; NULL: each turn is tracked again from its checkpoint.  Lost
 *       particles get NaN in lam and add nothing to gparam.
 * Work buffers live on the handle: calls on one handle from different
 * streams must be ordered by the caller.  Replaces, for a scalar objective,
 * the finite differences a caller of lattice_pass would take; the reference's
 * own diff_* routines (atintegrators/diff_*.c) propagate diffusion matrices,
 * not gradients. */
int atb_adjoint_forward(atb_handle* h, int32_t lattice_id, double* r, int64_t np,
                        int32_t nturns, int32_t turn0, const int32_t* param_elem,
                        const int32_t* param_order, const double* param_value, int32_t nparam,
                        double* ckpt, int32_t stride, double* estates, uint8_t* islost,
                        void* stream);
int atb_adjoint_backward(atb_handle* h, int32_t lattice_id, const double* ckpt, int64_t np,
                         int32_t nturns, int32_t turn0, int32_t stride, const double* estates,
                         const double* rfinal, const int32_t* param_elem,
                         const int32_t* param_order, const double* param_value, int32_t nparam,
                         double* lam, double* gparam, void* stream);

/* Element maps for Ohmi's envelope (device pointers, enqueued on `stream`):
 * for a particle entering element i at orbits[6 i .. 6 i + 5], its transfer
 * matrix m66[i] (exact derivatives, row-major d out / d in) and its radiation
 * diffusion matrix b66[i] (row-major; zero for non-radiating pass methods),
 * with `diff_const` = DIF_CONST gamma^5, all elements in one launch (the
 * lattice compiled for the default integrator, ATB_ERR_ARG otherwise).  Replaces
 * the per-element loop of pyat/at/physics/radiation.py:76-148 (_dmatr), i.e.
 * find_elem_m66 and pyat/at.c:755-831 (diffusion_matrix) per element. */
int atb_element_maps(atb_handle* h, int32_t lattice_id, const double* orbits, double* m66,
                     double* b66, double diff_const, void* stream);

/* Every element alone on its own particle (device pointers, enqueued on
 * `stream`): element i tracks r_in[6 i .. 6 i + 5] once, in the exact
 * arithmetic at turn 0, and writes its exit coordinates to r_out (nelem, 6)
 * and, when m66 is not NULL, its transfer matrix (nelem, 6, 6, row-major,
 * exact derivatives), all elements in one launch (the lattice compiled for
 * the default integrator, ATB_ERR_ARG otherwise).  Replaces a loop of
 * at_elempass calls, one per element (pyat/at.c:683-753), such as the
 * radiation energy loss of pyat/at/physics/energy_loss.py:80-89 (method
 * TRACKING: each radiating element entered at zero). */
int atb_element_pass(atb_handle* h, int32_t lattice_id, const double* r_in, double* r_out,
                     double* m66, void* stream);

/* Many lattice variants and particle sets in one persistent launch (device
 * pointers); the tiles of the longest jobs are scheduled first. */
int atb_track_batch(atb_handle* h, const atb_job_desc* jobs, int32_t njobs, int32_t mode,
                    void* stream);

/* Prepared batches: the same jobs as atb_track_batch, with the launch lists
 * built and uploaded once, so a launch is one memset and one persistent
 * kernel; atb_batch_capture records that launch as a CUDA graph (on the
 * handle's stream) and later launches replay the graph.  The job descriptors'
 * device buffers are used in place at every launch (the particles continue
 * from where the previous launch left them).  The reference runs each lattice
 * and particle set as a separate atpass call (pyat/at.c:340-681). */
int atb_batch_prepare(atb_handle* h, const atb_job_desc* jobs, int32_t njobs, int32_t mode,
                      int32_t* batch_id);
int atb_batch_capture(atb_handle* h, int32_t batch_id);
int atb_batch_launch(atb_handle* h, int32_t batch_id, void* stream);
int atb_batch_free(atb_handle* h, int32_t batch_id);

/* Measurement helper with no counterpart in the reference: the FP64 FMA
 * throughput of `device` (TFLOP/s, one FMA = 2 flops) from independent DFMA
 * chains in registers, the denominator of the tracking kernel's roofline. */
int atb_fp64_peak(int device, double* tflops, double* seconds);

/* No counterpart in the reference.  Tracking for callers that cannot
 * allocate device memory on their call path: real-time loops (an online model
 * in an orbit or tune feedback, where cudaMalloc/cudaFree would synchronise
 * the device and add unbounded latency) and applications whose HBM is owned
 * by another allocator (a pool that reserved it up front, where an extra
 * cudaMalloc fails or fragments it).  Same tracking as atb_track_device (whole
 * turns from element 0, no refpts), on caller-owned device buffers only:
 * `table` (nwords words) and `elem_off` (nelem+1 offsets) are the compiled
 * lattice on the device, `elem_off_host` the same offsets in host memory (to
 * plan the shared-memory segments), `r` the (6, np) particles, and the four
 * loss-map arrays when `losses` is 1.  Nothing is allocated: the launch lists
 * live in one fixed array of ATB_NOALLOC_SCRATCH_BYTES inside the library,
 * held by every GPU that loads it until the process exits.  Limits: at most
 * ATB_NOALLOC_MAX_PARTICLES particles and ATB_NOALLOC_MAX_SEGS segments of 48 KB
 * (a lattice table of up to about 48 MB); larger requests return ATB_ERR_ARG.
 * Alignment (checked, ATB_ERR_ARG otherwise; buffers from cudaMalloc always
 * satisfy it, a caller's own sub-allocator must): `table`, `r` and `lcoord`
 * 16-byte aligned, `elem_off`, `lturn` and `lelem` 4-byte aligned, `nwords`
 * and every element offset even (records on 16-byte boundaries, as the
 * lattice compiler writes them).  A table compiled for another integrator
 * than the default is refused (ATB_ERR_ARG) before anything is tracked.
 * The first call on a device looks up the array's device address and sets the
 * kernels' shared-memory limit, so make it before any stream capture.  All
 * calls share the array: calls that overlap on the GPU (two host threads, or
 * two streams) race, so serialise them.  Enqueued on `stream` (NULL: the
 * legacy default stream); returns after the launch completed, with
 * ATB_ERR_TIMEOUT if a bounded in-kernel wait gave up. */
#define ATB_NOALLOC_SCRATCH_BYTES (576 * 1024)
#define ATB_NOALLOC_MAX_TILES 32768
#define ATB_NOALLOC_MAX_PARTICLES (ATB_NOALLOC_MAX_TILES * 256)
#define ATB_NOALLOC_MAX_SEGS 1024
int atb_track_noalloc(int32_t device, const double* table, int64_t nwords,
                      const uint32_t* elem_off_host, const uint32_t* elem_off, int32_t nelem,
                      double* r, int64_t np, int32_t nturns, int32_t turn0, int32_t losses,
                      uint8_t* islost, uint32_t* lturn, uint32_t* lelem, double* lcoord,
                      int32_t mode, void* stream);

/* The serving loop (no reference counterpart: the reference runs each
 * request as one blocking atpass call, pyat/at.c:340-681).  A persistent
 * kernel claims tiles of jobs from a queue that the host appends to while it
 * runs, so a request admitted while others are on the GPU joins the running
 * launch at once instead of waiting for it to end.
 *   atb_serve_open    a queue of up to max_jobs jobs and max_tiles tiles for
 *                     jobs on the given lattices (uploaded on h), run in
 *                     `mode`.  The kernel is launched by the first submit.
 *   atb_serve_submit  append a job (device buffers as in atb_track_batch:
 *                     whole turns from turn0, loss map when losses is 1) and
 *                     publish its tiles; returns its slot.  With chunk_turns
 *                     > 0 a tile runs that many turns per claim and then goes
 *                     back to a device-side queue, so long jobs share the GPU
 *                     with later ones tile by tile (0: all turns in one
 *                     claim).  Re-enqueued tiles wait in one of 8 queues, the
 *                     decade of (turns left) x turn_cost (clamped to 0-7;
 *                     turn_cost <= 0: queue 0 only); blocks take new tiles
 *                     first, then queue 0, 1, ..., so tiles near their end
 *                     go ahead of long ones chunk by chunk.
 *                     With pidx (device, np int32 holding 0, 1,
 *                     ..., np - 1; NULL: none) a re-enqueued tile keeps
 *                     only its live particles, their indices packed at the
 *                     front of its range (pidx is overwritten), and counts
 *                     the others as done at once, so lost particles stop
 *                     costing lanes.  ATB_ERR_NOMEM when the queue is full
 *                     (atb_serve_reset it once every job has finished).
 *   atb_serve_poll    the particles of slots [first, first + nslots) that are done and
 *                     back in memory after all their turns (a job is
 *                     finished when its count equals its particle count; its
 *                     buffers may then be read), and
 *                     whether the kernel is running.  The kernel leaves after
 *                     ATB_SERVE_IDLE (0.2 s) without new work (a block also
 *                     after 40 s in one claim); poll and submit launch it
 *                     again while published or re-enqueued work waits.
 *   atb_serve_counters  tiles published and claimed from the host queue, and
 *                     continuations written to and taken from the device
 *                     queue since the last reset (out[4]).
 *   atb_serve_reset   leave the kernel and empty the queue.
 *   atb_serve_close   leave the kernel (after the claimed work) and free.
 * A job's result is the same as tracking it alone: each particle runs the
 * same operations with the same absolute turn counter. */
typedef struct atb_server atb_server;
int atb_serve_open(atb_handle* h, const int32_t* lattice_ids, int32_t nlat, int32_t mode,
                   int32_t max_jobs, int32_t max_tiles, atb_server** out);
int atb_serve_submit(atb_server* s, const atb_job_desc* job, int32_t chunk_turns,
                     double turn_cost, int32_t* pidx, int32_t* slot);
int atb_serve_poll(atb_server* s, int32_t first, int32_t nslots, uint64_t* done,
                   int32_t* running);
int atb_serve_counters(atb_server* s, int32_t* out);
int atb_serve_reset(atb_server* s);
int atb_serve_close(atb_server* s);

/* Key of the random kicks of QuantDiffPass elements in the launches that
 * follow on this handle.  The reference draws them from one sequential
 * PCG32 stream (atintegrators/atrandom.c, reset by pyat/at.c:833-852
 * reset_rng); here the kicks of particle p at element e in turn n are a
 * function of (key, job, p, n, e), so they are reproducible for a given key
 * whatever the launch shape, and statistically equivalent to the
 * reference's.  atb_track_noalloc uses key 0. */
int atb_set_rng(atb_handle* h, uint64_t key);

/* Wait for all work enqueued by this handle and return the kernels' status
 * (ATB_ERR_TIMEOUT if a bounded wait gave up). */
int atb_sync(atb_handle* h, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ATB200_H */
