/*
 * Host runtime of the C ABI declared in include/atb200.h: device buffers,
 * lattice tables, segment planning, launch configuration and the
 * refpts-snapshot streaming of at_atpass (pyat/at.c:340-681).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/atb200.h"
#include "atb_kernel_api.h"
#include "atb_table.h"

/* FP64 roofline probe: independent DFMA chains, no memory traffic */
__global__ void atb_dfma_probe(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
    double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[0] = s;   /* keeps the chains live */
}

extern "C" __global__ void atb_track_kernel_exact(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_fast(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_exact_gen(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_fast_gen(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_exact_np2(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_fast_np2(const AtbJob*, const AtbTile*, int, int*,
                                       unsigned long long*, int*, int, double*);

/* the tracking kernel for an arithmetic mode and a number of particles per
   thread (1 or 2); gen: the kernels with the other integrators of the GPU
   call (one particle per thread) */
static const void* track_fn(int mode, int ppt, bool gen = false) {
    if (gen)
        return mode == ATB_MODE_EXACT ? (const void*)atb_track_kernel_exact_gen
                                      : (const void*)atb_track_kernel_fast_gen;
    if (mode == ATB_MODE_EXACT)
        return ppt == 2 ? (const void*)atb_track_kernel_exact_np2
                        : (const void*)atb_track_kernel_exact;
    return ppt == 2 ? (const void*)atb_track_kernel_fast_np2 : (const void*)atb_track_kernel_fast;
}
extern "C" __global__ void atb_serve_kernel_exact(const AtbJob*, const AtbTile*, AtbServeArgs,
                                                  int*, int*, int, double*);
extern "C" __global__ void atb_serve_kernel_fast(const AtbJob*, const AtbTile*, AtbServeArgs, int*,
                                                 int*, int, double*);
extern "C" __global__ void atb_tangent_kernel(const AtbTangent);
extern "C" __global__ void atb_adjoint_forward_kernel(const AtbAdjoint);
extern "C" __global__ void atb_adjoint_turn_kernel(const AtbAdjoint);
extern "C" __global__ void atb_element_maps_kernel(const AtbElemMaps);

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define ATB_CUDA(call)                                                                 \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(ATB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

/* A growable device allocation. */
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

/* A prepared batch: its launch lists stay on the device, so launching it is
   one memset and one kernel, which can be captured in a CUDA graph. */
struct Batch {
    bool used = false;
    int mode = 1;
    int threads = 256;      /* launch shape fixed when the batch is prepared */
    int ppt = 1;            /* particles per thread                             */
    bool gen = false;       /* the kernels with the other integrators           */
    int seg_cap = 6144;
    int smem = 0;
    int grid = 0;
    int ntiles = 0;
    int njobs = 0;
    DevBuf jobs, tiles, counter, scratch, jobnext;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

struct Lattice {
    bool used = false;
    int nelem = 0;
    int64_t nwords = 0;
    std::vector<uint32_t> off;
    std::vector<uint64_t> hdr;  /* every element's header word              */
    std::vector<AtbSeg> segs;   /* pipelined segments (empty when resident) */
    bool resident = false;
    bool integ = false;         /* some element needs another integrator    */
    int plan_cap = 0;           /* seg capacity used to build the plan      */
    DevBuf words, doff, dsegs;
};

}  // namespace

struct atb_handle {
    int device = 0;
    uint64_t rng_key = 0;              /* quantum-diffusion kicks (atb_set_rng) */
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    int smem_optin = 0;
    int threads = 256;
    int ppt = 1;                       /* particles per thread (1 or 2)     */
    int refill_k = 8;                  /* prepared batches: tiles per initial claim */
    int seg_cap_words = 6144;          /* 48 KB per buffer, two buffers    */
    int resident_max_words = 14336;    /* tables up to 112 KB stay resident */
    int64_t rout_budget = 4LL << 30;
    std::vector<Lattice> lats;
    DevBuf r, rout, lost, lturn, lelem, lcoord, refpts, jobs, tiles, counter, status, alive,
        moments, tan_pelem, tan_porder, compact, jobnext, adj_pelem, adj_porder, adj_scratch,
        adj_block, adj_state;
    std::vector<int32_t> h_pelem;
    std::vector<AtbTile> h_tiles;
    std::vector<struct Batch> batches;
    char* stage[2] = {nullptr, nullptr};            /* pinned snapshot staging */
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
};

/* The serving loop: a persistent kernel that claims tiles from a queue the
   host appends to while it runs.  Job and tile records live in device memory
   (append-only within a session), the control words in mapped host memory. */
struct atb_server {
    atb_handle* h = nullptr;
    int mode = 0;
    int max_jobs = 0, max_tiles = 0;
    int njobs = 0, ntiles = 0;          /* appended so far                       */
    int smem = 0, grid = 0, threads = 256, seg_cap = 6144;
    std::vector<int32_t> lattice_ids;   /* the lattices jobs may use             */
    AtbServeCtl* ctl = nullptr;         /* host view of the mapped control words */
    AtbServeCtl* dctl = nullptr;        /* its device address                    */
    DevBuf jobs, tiles, counter, status, jobnext, done, compact;
    DevBuf ring, ring_ctr;              /* continuation rings; heads, tails, inflight */
    int ring_cap = 0;
    unsigned long long* h_done = nullptr;   /* pinned: done counters, claim counter,
                                               ring cursors                       */
    AtbJob* h_job = nullptr;            /* pinned staging of one job record      */
    unsigned long long* h_zero = nullptr;   /* pinned zeros for the job counters */
    AtbTile* h_tiles = nullptr;         /* pinned staging of one job's tiles     */
    int h_tiles_cap = 0;
    cudaStream_t kstream = nullptr;     /* the persistent kernel                 */
    cudaStream_t cstream = nullptr;     /* record copies and polls               */
    bool launched = false;
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

/* greedy segmentation of the element records, each segment <= cap words */
int plan_segments(Lattice& L, int cap) {
    L.segs.clear();
    int i = 0;
    while (i < L.nelem) {
        int j = i;
        while (j < L.nelem && (int64_t)(L.off[j + 1] - L.off[i]) <= cap) ++j;
        if (j == i)
            return fail(ATB_ERR_ARG, "element record longer than the shared-memory segment");
        AtbSeg s;
        s.first_elem = i;
        s.nelem = j - i;
        s.word0 = L.off[i];
        int nw = (int)(L.off[j] - L.off[i]);
        s.nwords = nw + (nw & 1);
        s.pad = 0;
        L.segs.push_back(s);
        i = j;
    }
    L.plan_cap = cap;
    return ATB_OK;
}

int seg_of(const Lattice& L, int elem) {
    /* index of the segment holding element `elem` */
    int lo = 0, hi = (int)L.segs.size() - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (L.segs[mid].first_elem <= elem) lo = mid; else hi = mid - 1;
    }
    return lo;
}

int upload_plan(atb_handle* h, Lattice& L) {
    L.resident = (L.nelem > 0) && (L.nwords <= h->resident_max_words);
    if (L.resident) {
        L.segs.clear();
        AtbSeg s;
        s.first_elem = 0;
        s.nelem = L.nelem;
        s.word0 = 0;
        s.nwords = (int)(L.nwords + (L.nwords & 1));
        s.pad = 0;
        L.segs.push_back(s);
        L.plan_cap = h->seg_cap_words;
    } else {
        int rc = plan_segments(L, h->seg_cap_words);
        if (rc) return rc;
    }
    if (!L.segs.empty()) {
        if (L.dsegs.ensure(L.segs.size() * sizeof(AtbSeg)) != cudaSuccess)
            return fail(ATB_ERR_CUDA, "cudaMalloc(segments) failed");
        ATB_CUDA(cudaMemcpy(L.dsegs.p, L.segs.data(), L.segs.size() * sizeof(AtbSeg),
                            cudaMemcpyHostToDevice));
    }
    return ATB_OK;
}

/* at.c refpts walk (pyat/at.c:618-651): snapshots taken in one turn */
int64_t count_records(const uint32_t* refpts, int nref, int start, int end, int nelem) {
    const uint32_t kNone = 0x7fffffffu; /* INT_MAX as at.c assigns it */
    int nri = 0;
    uint32_t nextref = (nri < nref) ? refpts[nri++] : kNone;
    int64_t cnt = 0;
    for (int e = start; e < end; ++e) {
        if ((uint32_t)e == nextref) {
            ++cnt;
            nextref = (nri < nref) ? refpts[nri++] : kNone;
        }
    }
    if ((uint32_t)nelem == nextref) ++cnt;
    return cnt;
}

/* the random-kick key of job j: distinct per job, so batched particle sets
   that share a lattice draw independent kicks */
uint64_t job_key(const atb_handle* h, int j) {
    return h->rng_key ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(j + 1));
}

void fill_job_lattice(AtbJob& J, const Lattice& L, int start_elem, int end_elem) {
    J.table = L.words.as<double>();
    J.segs = L.dsegs.as<AtbSeg>();
    J.elem_off = L.doff.as<uint32_t>();
    J.nelem = L.nelem;
    J.resident = L.resident ? 1 : 0;
    J.start_elem = start_elem;
    J.end_elem = end_elem;
    if (L.nelem == 0 || L.segs.empty()) {
        J.resident = 0;
        J.seg_first0 = 0;
        J.nseg_first = 0;
        J.nseg_turn = 0;
    } else if (L.resident) {
        J.seg_first0 = 0;
        J.nseg_first = 1;
        J.nseg_turn = 1;
    } else {
        if (start_elem >= end_elem) {
            J.seg_first0 = 0;
            J.nseg_first = 0;
        } else {
            J.seg_first0 = seg_of(L, start_elem);
            J.nseg_first = seg_of(L, end_elem - 1) - J.seg_first0 + 1;
        }
        J.nseg_turn = (end_elem > 0) ? seg_of(L, end_elem - 1) + 1 : 0;
    }
}

int kernel_config(atb_handle* h, const std::vector<const Lattice*>& lats, int mode,
                  int* smem_bytes, int* grid_max, bool* gen) {
    bool any_pipe = false;
    int64_t res_words = 0;
    *gen = false;
    for (const Lattice* L : lats) {
        if (L->integ) *gen = true;
        if (L->resident) res_words = std::max<int64_t>(res_words, L->nwords + (L->nwords & 1));
        else if (!L->segs.empty()) any_pipe = true;
    }
    int64_t words = any_pipe ? 2LL * h->seg_cap_words : 0;
    words = std::max<int64_t>(words, res_words);
    int bytes = (int)(words * 8);
    if (bytes > h->smem_optin)
        return fail(ATB_ERR_ARG, "shared-memory plan exceeds the per-block limit");
    *smem_bytes = bytes;
    const void* fn = track_fn(mode, *gen ? 1 : h->ppt, *gen);
    int per_sm = 0;
    ATB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, h->threads, bytes));
    if (per_sm < 1) return fail(ATB_ERR_ARG, "launch configuration does not fit on an SM");
    *grid_max = per_sm * h->sm_count;
    return ATB_OK;
}

int launch(atb_handle* h, const std::vector<AtbJob>& jobs, const std::vector<AtbTile>& tiles,
           int smem_bytes, int grid_max, int mode, cudaStream_t st, int threads, int ppt,
           bool gen) {
    if (tiles.empty()) return ATB_OK;
    if (h->jobs.ensure(jobs.size() * sizeof(AtbJob)) != cudaSuccess ||
        h->tiles.ensure(tiles.size() * sizeof(AtbTile)) != cudaSuccess)
        return fail(ATB_ERR_CUDA, "cudaMalloc(launch lists) failed");
    ATB_CUDA(cudaMemcpyAsync(h->jobs.p, jobs.data(), jobs.size() * sizeof(AtbJob),
                             cudaMemcpyHostToDevice, st));
    ATB_CUDA(cudaMemcpyAsync(h->tiles.p, tiles.data(), tiles.size() * sizeof(AtbTile),
                             cudaMemcpyHostToDevice, st));
    ATB_CUDA(cudaMemsetAsync(h->counter.p, 0, sizeof(int), st));
    /* per-job particle cursors of the refilling tile loop */
    if (h->jobnext.ensure(jobs.size() * sizeof(unsigned long long)) != cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(job cursors) failed");
    ATB_CUDA(cudaMemsetAsync(h->jobnext.p, 0, jobs.size() * sizeof(unsigned long long), st));
    int grid = std::min<int64_t>((int64_t)tiles.size(), grid_max);
    int cap = h->seg_cap_words;
    /* survivor-compaction scratch: ATB_COMPACT_WORDS doubles per thread of the grid */
    if (h->compact.ensure((size_t)grid * threads * ATB_COMPACT_WORDS * sizeof(double)) !=
        cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(compaction scratch) failed");
    const AtbJob* dj = h->jobs.as<AtbJob>();
    const AtbTile* dt = h->tiles.as<AtbTile>();
    const int nt = (int)tiles.size();
    int* cnt = h->counter.as<int>();
    unsigned long long* jn = h->jobnext.as<unsigned long long>();
    int* sts = h->status.as<int>();
    double* scr = h->compact.as<double>();
    if (gen && mode == ATB_MODE_EXACT)
        atb_track_kernel_exact_gen<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts,
                                                                      cap, scr);
    else if (gen)
        atb_track_kernel_fast_gen<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts,
                                                                     cap, scr);
    else if (mode == ATB_MODE_EXACT && ppt == 2)
        atb_track_kernel_exact_np2<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts,
                                                                      cap, scr);
    else if (mode == ATB_MODE_EXACT)
        atb_track_kernel_exact<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts, cap,
                                                                  scr);
    else if (ppt == 2)
        atb_track_kernel_fast_np2<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts,
                                                                     cap, scr);
    else
        atb_track_kernel_fast<<<grid, threads, smem_bytes, st>>>(dj, dt, nt, cnt, jn, sts, cap,
                                                                 scr);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

/* Threads per block for a single particle set: the handle's value, reduced
   (to a multiple of 32) when the set is too small to give every SM a tile,
   so that a few hundred particles run on many SMs rather than queue on a
   few.  Results do not depend on it: particles are independent. */
int threads_for(const atb_handle* h, int64_t np) {
    const int64_t per_sm = (np + h->sm_count - 1) / std::max(h->sm_count, 1);
    const int64_t want = std::max<int64_t>(32, ((per_sm + 31) / 32) * 32);
    return (int)std::min<int64_t>(h->threads, want);
}

/* particles per thread for a single set: the handle's choice when the set
   fills every SM with full tiles, else one */
int ppt_for(const atb_handle* h, int64_t np) {
    return np >= (int64_t)h->sm_count * h->threads * h->ppt ? h->ppt : 1;
}

void make_tiles(std::vector<AtbTile>& tiles, int job, int64_t np, int threads) {
    for (int64_t f = 0; f < np; f += threads) {
        AtbTile t;
        t.job = job;
        t.first = f;
        t.count = (int32_t)std::min<int64_t>(threads, np - f);
        tiles.push_back(t);
    }
}

/* The claims of a multi-job launch.  With factor k > 1 a job whose lanes
   refill (one particle per thread) gets one claim per k tiles: each claim
   starts a block on a tile's worth of the job's particles and the block takes
   the rest of the job through its freed lanes, so blocks stay full while
   particles are lost; other jobs get one claim per tile.  The factor is
   halved until the launch has at least two claims per resident block. */
void make_claims(const atb_handle* h, std::vector<AtbTile>& tiles,
                 const std::vector<AtbJob>& J, const std::vector<int>& order, int grid_max,
                 int refill_k, int ppt) {
    const int size = h->threads * ppt;
    int k = ppt == 1 ? std::max(1, refill_k) : 1;
    for (;; k /= 2) {
        tiles.clear();
        for (int j : order) {
            if (J[j].nturns <= 0) continue;
            if (k > 1 && atb_job_refills(&J[j])) {
                const int64_t n = std::max<int64_t>(1, (J[j].np + (int64_t)size * k - 1) /
                                                           ((int64_t)size * k));
                for (int64_t i = 0; i < n; ++i) {
                    AtbTile t;
                    t.job = j;
                    t.first = 0;   /* refilling jobs take particles from their cursor */
                    t.count = (int32_t)std::min<int64_t>(size, J[j].np);
                    if (t.count > 0) tiles.push_back(t);
                }
            } else {
                make_tiles(tiles, j, J[j].np, size);
            }
        }
        if (k <= 1 || (int64_t)tiles.size() >= 2LL * grid_max) break;
    }
}

Lattice* get_lat(atb_handle* h, int id) {
    if (id < 0 || id >= (int)h->lats.size() || !h->lats[id].used) return nullptr;
    return &h->lats[id];
}

int check_status(atb_handle* h, cudaStream_t st) {
    int s = 0;
    ATB_CUDA(cudaMemcpyAsync(&s, h->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    ATB_CUDA(cudaStreamSynchronize(st));
    if (s & ATB_STATUS_WAIT_TIMEOUT) {
        cudaMemsetAsync(h->status.p, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return fail(ATB_ERR_TIMEOUT, "a bounded shared-memory staging wait timed out");
    }
    if (s & ATB_STATUS_INTEGRATOR) {
        cudaMemsetAsync(h->status.p, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return fail(ATB_ERR_ARG, "an element compiled for another integrator reached a kernel "
                                 "built without them");
    }
    return ATB_OK;
}

}  // namespace

/* lets the other translation units of the library report through
   atb_last_error() */
void atb_set_error_message(const char* msg) { g_err = msg ? msg : ""; }

extern "C" {

int atb_version(void) { return 10000; }

const char* atb_last_error(void) { return g_err.c_str(); }

int atb_device_count(int* count) {
    if (!count) return fail(ATB_ERR_ARG, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(ATB_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    }
    *count = n;
    return ATB_OK;
}

int atb_device_info(int device, char* name, int name_len, int* cc_major, int* cc_minor,
                    int* sm_count, uint64_t* total_mem) {
    cudaDeviceProp p;
    ATB_CUDA(cudaGetDeviceProperties(&p, device));
    if (name && name_len > 0) {
        std::strncpy(name, p.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (total_mem) *total_mem = p.totalGlobalMem;
    return ATB_OK;
}

int atb_create(int device, atb_handle** out) {
    if (!out) return fail(ATB_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    ATB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(ATB_ERR_ARG, "invalid device id");
    DeviceGuard g(device);
    std::unique_ptr<atb_handle> h(new atb_handle());
    h->device = device;
    cudaDeviceProp p;
    ATB_CUDA(cudaGetDeviceProperties(&p, device));
    if (p.major < 10)
        return fail(ATB_ERR_ARG, "this build targets sm_100a (B200); device is sm_" +
                                     std::to_string(p.major) + std::to_string(p.minor));
    h->sm_count = p.multiProcessorCount;
    ATB_CUDA(cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                    device));
    /* leave room for the kernel's static shared memory */
    h->smem_optin -= 1024;
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_exact,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_fast,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_exact_np2,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_exact_gen,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_fast_gen,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaFuncSetAttribute(atb_track_kernel_fast_np2,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    ATB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    if (h->counter.ensure(sizeof(int)) != cudaSuccess || h->status.ensure(sizeof(int)) != cudaSuccess)
        return fail(ATB_ERR_CUDA, "cudaMalloc failed");
    ATB_CUDA(cudaMemset(h->status.p, 0, sizeof(int)));
    *out = h.release();
    return ATB_OK;
}

int atb_destroy(atb_handle* h) {
    if (!h) return ATB_OK;
    {
        DeviceGuard g(h->device);
        if (h->stream) cudaStreamSynchronize(h->stream);
        for (Lattice& L : h->lats) {
            L.words.release();
            L.doff.release();
            L.dsegs.release();
        }
        for (Batch& B : h->batches) {
            if (B.exec) cudaGraphExecDestroy(B.exec);
            if (B.graph) cudaGraphDestroy(B.graph);
            B.jobs.release();
            B.tiles.release();
            B.counter.release();
            B.scratch.release();
            B.jobnext.release();
        }
        for (DevBuf* b : {&h->r, &h->rout, &h->lost, &h->lturn, &h->lelem, &h->lcoord,
                          &h->refpts, &h->jobs, &h->tiles, &h->counter, &h->status, &h->alive,
                          &h->moments, &h->tan_pelem, &h->tan_porder, &h->compact,
                          &h->adj_pelem, &h->adj_porder, &h->adj_scratch, &h->adj_block,
                          &h->adj_state,
                          &h->jobnext})
            b->release();
        for (int i = 0; i < 2; ++i) {
            if (h->stage[i]) cudaFreeHost(h->stage[i]);
            if (h->stage_ev[i]) cudaEventDestroy(h->stage_ev[i]);
        }
        if (h->stream) cudaStreamDestroy(h->stream);
    }
    delete h;
    return ATB_OK;
}

int atb_set_refill_factor(atb_handle* h, int32_t k) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    if (k < 1 || k > 64) return fail(ATB_ERR_ARG, "refill factor must be in [1, 64]");
    for (const Batch& B : h->batches)
        if (B.used) return fail(ATB_ERR_ARG, "free the prepared batches before changing the launch shape");
    h->refill_k = k;
    return ATB_OK;
}

int atb_set_particles_per_thread(atb_handle* h, int32_t ppt) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    if (ppt != 1 && ppt != 2) return fail(ATB_ERR_ARG, "particles per thread must be 1 or 2");
    for (const Batch& B : h->batches)
        if (B.used) return fail(ATB_ERR_ARG, "free the prepared batches before changing the launch shape");
    h->ppt = ppt;
    return ATB_OK;
}

int atb_set_launch(atb_handle* h, int threads, int seg_cap_words, int resident_max_words,
                   int64_t rout_budget_bytes) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    for (const Batch& B : h->batches)
        if (B.used) return fail(ATB_ERR_ARG, "free the prepared batches before changing the launch shape");
    if (threads) {
        if (threads < 32 || threads > ATB_MAX_THREADS || threads % 32)
            return fail(ATB_ERR_ARG, "threads per block must be a multiple of 32 in [32, 512]");
        h->threads = threads;
    }
    if (seg_cap_words) {
        if (seg_cap_words < ATB_MAX_RECORD_WORDS + 1 || seg_cap_words % 2 ||
            (int64_t)seg_cap_words * 16 > h->smem_optin)
            return fail(ATB_ERR_ARG, "segment capacity out of range");
        h->seg_cap_words = seg_cap_words;
    }
    if (resident_max_words) {
        if ((int64_t)resident_max_words * 8 > h->smem_optin)
            return fail(ATB_ERR_ARG, "resident table limit exceeds shared memory");
        h->resident_max_words = resident_max_words;
    }
    if (rout_budget_bytes > 0) h->rout_budget = rout_budget_bytes;
    /* re-plan every lattice for the new capacities; prepared batches hold
       launch lists built on the current plans, so they must be freed first */
    for (const Batch& B : h->batches)
        if (B.used) return fail(ATB_ERR_ARG, "free the prepared batches before changing the launch shape");
    DeviceGuard g(h->device);
    ATB_CUDA(cudaDeviceSynchronize());   /* no launch may still read the old plans */
    for (Lattice& L : h->lats)
        if (L.used) {
            int rc = upload_plan(h, L);
            if (rc) return rc;
        }
    return ATB_OK;
}

int atb_lattice_upload(atb_handle* h, const double* words, int64_t nwords,
                       const uint32_t* elem_off, int32_t nelem, int32_t* lattice_id) {
    if (!h || !lattice_id) return fail(ATB_ERR_ARG, "NULL argument");
    if (nelem < 0 || nwords < 0 || (nelem > 0 && (!words || !elem_off)))
        return fail(ATB_ERR_ARG, "invalid lattice table");
    if (nelem > 0 && (elem_off[0] != 0 || (int64_t)elem_off[nelem] != nwords))
        return fail(ATB_ERR_ARG, "element offsets do not span the table");
    for (int i = 0; i < nelem; ++i) {
        uint32_t a = elem_off[i], b = elem_off[i + 1];
        if (b <= a || (a & 1u) || (b - a) > ATB_MAX_RECORD_WORDS)
            return fail(ATB_ERR_ARG, "invalid element record bounds");
        uint64_t hdr;
        std::memcpy(&hdr, words + a, 8);
        uint32_t len = (uint32_t)((hdr >> ATB_H_LEN_SHIFT) & ATB_H_LEN_MASK);
        uint32_t op = (uint32_t)((hdr >> ATB_H_OP_SHIFT) & ATB_H_OP_MASK);
        if (len != b - a || op >= ATB_NUM_OPS)
            return fail(ATB_ERR_ARG, "corrupt element record header");
    }
    DeviceGuard g(h->device);
    int id = -1;
    for (int i = 0; i < (int)h->lats.size(); ++i)
        if (!h->lats[i].used) { id = i; break; }
    if (id < 0) {
        h->lats.emplace_back();
        id = (int)h->lats.size() - 1;
    }
    Lattice& L = h->lats[id];
    L.used = true;
    L.nelem = nelem;
    L.nwords = nwords;
    L.off.assign(elem_off, elem_off + nelem + 1);
    if (nelem == 0) L.off.assign(1, 0u);
    L.hdr.resize(nelem);
    for (int i = 0; i < nelem; ++i) std::memcpy(&L.hdr[i], words + elem_off[i], 8);
    L.integ = false;
    for (int i = 0; i < nelem; ++i)
        if ((L.hdr[i] >> ATB_H_FL_SHIFT) & ATB_F_INTEG) L.integ = true;
    size_t wbytes = (size_t)(nwords + 2) * 8;
    if (L.words.ensure(wbytes) != cudaSuccess || L.doff.ensure(L.off.size() * 4) != cudaSuccess) {
        L.used = false;
        return fail(ATB_ERR_CUDA, "cudaMalloc(lattice) failed");
    }
    ATB_CUDA(cudaMemset(L.words.p, 0, wbytes));
    if (nwords) ATB_CUDA(cudaMemcpy(L.words.p, words, nwords * 8, cudaMemcpyHostToDevice));
    ATB_CUDA(cudaMemcpy(L.doff.p, L.off.data(), L.off.size() * 4, cudaMemcpyHostToDevice));
    int rc = upload_plan(h, L);
    if (rc) {
        L.used = false;
        return rc;
    }
    *lattice_id = id;
    return ATB_OK;
}

int atb_lattice_update(atb_handle* h, int32_t id, const double* words, int64_t nwords) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (nwords != L->nwords) return fail(ATB_ERR_ARG, "table size changed");
    DeviceGuard g(h->device);
    ATB_CUDA(cudaStreamSynchronize(h->stream));
    if (nwords) ATB_CUDA(cudaMemcpy(L->words.p, words, nwords * 8, cudaMemcpyHostToDevice));
    for (int i = 0; i < L->nelem; ++i) std::memcpy(&L->hdr[i], words + L->off[i], 8);
    L->integ = false;
    for (int i = 0; i < L->nelem; ++i)
        if ((L->hdr[i] >> ATB_H_FL_SHIFT) & ATB_F_INTEG) L->integ = true;
    return ATB_OK;
}

int atb_lattice_free(atb_handle* h, int32_t id) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    DeviceGuard g(h->device);
    cudaStreamSynchronize(h->stream);
    L->words.release();
    L->doff.release();
    L->dsegs.release();
    L->used = false;
    return ATB_OK;
}

namespace {

constexpr int64_t kStageBytes = 64LL << 20;   /* each of the two staging buffers */
constexpr int64_t kStageDirect = 8LL << 20;   /* smaller copies go directly      */

/* The snapshots of one chunk -- `slots` slots of gn particles, gn * 48 bytes
   each, contiguous on the device -- to slots [slot0, slot0 + slots) of the
   caller's rout (np particles a slot), columns [a, a + gn).  Small copies go
   directly; large ones through two pinned staging buffers: the GPU fills one
   while host threads place the other, so the copy is not held to one
   thread's pace through the caller's fresh (not yet touched) pages. */
int copy_snapshots(atb_handle* h, cudaStream_t st, const double* dev, int64_t slots, int64_t gn,
                   double* rout, int64_t np, int64_t a, int64_t slot0) {
    const int64_t row = gn * 48, pitch = np * 48, total = slots * row;
    char* dst = reinterpret_cast<char*>(rout + (slot0 * np + a) * 6);
    if (total <= kStageDirect) {
        if (gn == np)
            ATB_CUDA(cudaMemcpyAsync(dst, dev, (size_t)total, cudaMemcpyDeviceToHost, st));
        else
            ATB_CUDA(cudaMemcpy2DAsync(dst, (size_t)pitch, dev, (size_t)row, (size_t)row,
                                       (size_t)slots, cudaMemcpyDeviceToHost, st));
        return ATB_OK;
    }
    for (int i = 0; i < 2; ++i) {
        if (!h->stage[i])
            ATB_CUDA(cudaHostAlloc((void**)&h->stage[i], (size_t)kStageBytes, cudaHostAllocDefault));
        if (!h->stage_ev[i])
            ATB_CUDA(cudaEventCreateWithFlags(&h->stage_ev[i], cudaEventDisableTiming));
    }
    const char* src = reinterpret_cast<const char*>(dev);
    const int64_t npieces = (total + kStageBytes - 1) / kStageBytes;
    auto issue = [&](int64_t p) {
        const int64_t off = p * kStageBytes, len = std::min(kStageBytes, total - off);
        cudaError_t e = cudaMemcpyAsync(h->stage[p & 1], src + off, (size_t)len,
                                        cudaMemcpyDeviceToHost, st);
        return e == cudaSuccess ? cudaEventRecord(h->stage_ev[p & 1], st) : e;
    };
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (int64_t p = 0; p < std::min<int64_t>(2, npieces); ++p) ATB_CUDA(issue(p));
    for (int64_t p = 0; p < npieces; ++p) {
        ATB_CUDA(cudaEventSynchronize(h->stage_ev[p & 1]));
        const int64_t off = p * kStageBytes, len = std::min(kStageBytes, total - off);
        const char* stage = h->stage[p & 1];
        /* device bytes [b0, b1) of this piece to their rows of rout */
        auto place = [=](int64_t b0, int64_t b1) {
            if (pitch == row) {              /* all particles: one block */
                std::memcpy(dst + b0, stage + (b0 - off), (size_t)(b1 - b0));
                return;
            }
            while (b0 < b1) {
                const int64_t slot = b0 / row, within = b0 - slot * row;
                const int64_t n = std::min(b1 - b0, row - within);
                std::memcpy(dst + slot * pitch + within, stage + (b0 - off), (size_t)n);
                b0 += n;
            }
        };
        const int64_t part = (len + nthr - 1) / nthr;
        std::vector<std::thread> th;
        for (int t = 1; t < nthr; ++t) {
            const int64_t b0 = off + std::min<int64_t>(len, t * part);
            const int64_t b1 = off + std::min<int64_t>(len, (t + 1) * part);
            if (b0 >= b1) continue;
            try {
                th.emplace_back(place, b0, b1);
            } catch (...) {
                place(b0, b1);     /* no thread to be had: this one does it */
            }
        }
        place(off, off + std::min<int64_t>(len, part));
        for (std::thread& x : th) x.join();
        if (p + 2 < npieces) ATB_CUDA(issue(p + 2));   /* into the buffer just placed */
    }
    return ATB_OK;
}

}  // namespace

int atb_track(atb_handle* h, int32_t id, double* rin, int64_t np, int32_t nturns, int32_t turn0,
              int32_t start_elem, int32_t end_elem, const uint32_t* refpts, int32_t nref,
              double* rout, int32_t losses, uint8_t* islost, uint32_t* lturn, uint32_t* lelem,
              double* lcoord, uint32_t* alive, double* moments, int32_t mode, int32_t flags) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (np < 0 || nturns < 0 || nref < 0) return fail(ATB_ERR_ARG, "negative size");
    if (np > 0 && !rin) return fail(ATB_ERR_ARG, "rin is NULL");
    if (nref > 0 && (!refpts || (!rout && np > 0))) return fail(ATB_ERR_ARG, "refpts/rout missing");
    if (losses && np > 0 && (!islost || !lturn || !lelem || !lcoord))
        return fail(ATB_ERR_ARG, "loss map buffers missing");
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return fail(ATB_ERR_ARG, "bad mode");
    const int nelem = L->nelem;
    if (nelem > 0) {
        if (start_elem < 0 || start_elem >= nelem || end_elem < 0 || end_elem > nelem ||
            start_elem > end_elem)
            return fail(ATB_ERR_ARG, "start_elem/end_elem out of range");
    } else {
        start_elem = end_elem = 0;
    }
    if (np == 0 || nturns == 0) return ATB_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = h->stream;

    /* device buffers */
    const size_t rbytes = (size_t)np * 48;
    if (h->r.ensure(rbytes) != cudaSuccess) return fail(ATB_ERR_NOMEM, "cudaMalloc(particles) failed");
    ATB_CUDA(cudaMemcpyAsync(h->r.p, rin, rbytes, cudaMemcpyHostToDevice, st));
    if (losses) {
        if (h->lost.ensure(np) != cudaSuccess || h->lturn.ensure(np * 4) != cudaSuccess ||
            h->lelem.ensure(np * 4) != cudaSuccess || h->lcoord.ensure(rbytes) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(loss map) failed");
        ATB_CUDA(cudaMemsetAsync(h->lost.p, 0, np, st));
        ATB_CUDA(cudaMemsetAsync(h->lturn.p, 0, np * 4, st));
        ATB_CUDA(cudaMemsetAsync(h->lelem.p, 0, np * 4, st));
        ATB_CUDA(cudaMemsetAsync(h->lcoord.p, 0, rbytes, st));
    }
    if (alive || moments) {
        if (h->alive.ensure((size_t)nturns * 4) != cudaSuccess ||
            h->moments.ensure((size_t)nturns * 96) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(statistics) failed");
        ATB_CUDA(cudaMemsetAsync(h->alive.p, 0, (size_t)nturns * 4, st));
        ATB_CUDA(cudaMemsetAsync(h->moments.p, 0, (size_t)nturns * 96, st));
    }
    if (nref > 0) {
        if (h->refpts.ensure((size_t)nref * 4) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(refpts) failed");
        ATB_CUDA(cudaMemcpyAsync(h->refpts.p, refpts, (size_t)nref * 4, cudaMemcpyHostToDevice, st));
    }

    /* Snapshots bounded by the device budget: turns in chunks, and when one
       turn of snapshots of all particles does not fit, particles in groups
       whose snapshots go to their columns of every slot of rout (the
       particles are independent, so a group sees exactly what it would in one
       launch; per-turn statistics add up over the groups). */
    const int64_t rec_first = nref ? count_records(refpts, nref, start_elem, end_elem, nelem) : 0;
    const int64_t rec_turn = nref ? count_records(refpts, nref, 0, end_elem, nelem) : 0;
    const int64_t rec_max = std::max(rec_first, rec_turn);
    int64_t group = np;
    if (nref > 0 && rec_max > 0) {
        group = std::min<int64_t>(np, h->rout_budget / (rec_max * 48));
        if (group < 1)
            return fail(ATB_ERR_NOMEM, "one turn of refpts snapshots of one particle exceeds the device budget");
    }
    const int64_t slot_bytes = group * 48;
    int64_t turns_per_chunk = nturns;
    if (nref > 0 && rec_turn > 0)
        turns_per_chunk = std::max<int64_t>(1, h->rout_budget / (rec_turn * slot_bytes));
    /* the first chunk holds rec_first + (nt - 1) rec_turn slots, the others
       nt rec_turn, nt <= turns_per_chunk: within the budget */
    const int64_t max_slots =
        nref ? std::max<int64_t>(
                   rec_first + (std::min<int64_t>(turns_per_chunk, nturns) - 1) * rec_turn,
                   turns_per_chunk * rec_turn)
             : 0;
    if (nref > 0 && max_slots > 0) {
        if (h->rout.ensure((size_t)(max_slots * slot_bytes)) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(refpts snapshots) failed");
    }

    std::vector<const Lattice*> lats{L};
    int smem = 0, grid_max = 0;
    bool gen = false;
    int rc = kernel_config(h, lats, mode, &smem, &grid_max, &gen);
    if (rc) return rc;

    for (int64_t a = 0; a < np; a += group) {
        const int64_t gn = std::min<int64_t>(group, np - a);
        int64_t slot_done = 0;
        for (int64_t t0 = 0; t0 < nturns; t0 += turns_per_chunk) {
            const int nt = (int)std::min<int64_t>(turns_per_chunk, nturns - t0);
            AtbJob J;
            std::memset(&J, 0, sizeof(J));
            fill_job_lattice(J, *L, t0 == 0 ? start_elem : 0, end_elem);
            J.rng.key = job_key(h, 0);
            J.check_loss = (flags & ATB_FLAG_ELEMENT) ? 0 : 1;
            J.rng.pbase = a;
            J.r = h->r.as<double>() + 6 * a;
            J.np = gn;
            J.turn0 = turn0 + (int32_t)t0;
            J.nturns = nt;
            J.refpts = h->refpts.as<uint32_t>();
            J.nref = nref;
            J.losses = losses ? 1 : 0;
            J.rout = nref ? h->rout.as<double>() : nullptr;
            J.rout_slot0 = 0;
            J.lost = losses ? h->lost.as<uint8_t>() + a : nullptr;
            J.lturn = losses ? h->lturn.as<uint32_t>() + a : nullptr;
            J.lelem = losses ? h->lelem.as<uint32_t>() + a : nullptr;
            J.lcoord = losses ? h->lcoord.as<double>() + 6 * a : nullptr;
            J.alive = (alive || moments) ? h->alive.as<uint32_t>() + t0 : nullptr;
            J.moments = (alive || moments) ? h->moments.as<double>() + 12 * t0 : nullptr;
            std::vector<AtbJob> jobs{J};
            h->h_tiles.clear();
            const int pp = gen ? 1 : ppt_for(h, gn);
            const int thr = pp > 1 ? h->threads : threads_for(h, gn);
            make_tiles(h->h_tiles, 0, gn, thr * pp);
            rc = launch(h, jobs, h->h_tiles, smem, grid_max, mode, st, thr, pp, gen);
            if (rc) return rc;
            if (nref) {
                int64_t slots = (t0 == 0 ? rec_first : rec_turn) + (int64_t)(nt - 1) * rec_turn;
                if (slots > 0) {
                    rc = copy_snapshots(h, st, h->rout.as<double>(), slots, gn, rout, np, a,
                                        slot_done);
                    if (rc) return rc;
                }
                slot_done += slots;
            }
            /* the job/tile lists are host vectors reused next chunk: make sure
               the copies above have consumed them */
            ATB_CUDA(cudaStreamSynchronize(st));
        }
    }
    ATB_CUDA(cudaMemcpyAsync(rin, h->r.p, rbytes, cudaMemcpyDeviceToHost, st));
    if (losses) {
        ATB_CUDA(cudaMemcpyAsync(islost, h->lost.p, np, cudaMemcpyDeviceToHost, st));
        ATB_CUDA(cudaMemcpyAsync(lturn, h->lturn.p, np * 4, cudaMemcpyDeviceToHost, st));
        ATB_CUDA(cudaMemcpyAsync(lelem, h->lelem.p, np * 4, cudaMemcpyDeviceToHost, st));
        ATB_CUDA(cudaMemcpyAsync(lcoord, h->lcoord.p, rbytes, cudaMemcpyDeviceToHost, st));
    }
    if (alive) ATB_CUDA(cudaMemcpyAsync(alive, h->alive.p, (size_t)nturns * 4, cudaMemcpyDeviceToHost, st));
    if (moments)
        ATB_CUDA(cudaMemcpyAsync(moments, h->moments.p, (size_t)nturns * 96, cudaMemcpyDeviceToHost, st));
    return check_status(h, st);
}

int atb_track_device(atb_handle* h, int32_t id, double* r, int64_t np, int32_t nturns,
                     int32_t turn0, int32_t losses, uint8_t* islost, uint32_t* lturn,
                     uint32_t* lelem, double* lcoord, uint32_t* alive, double* moments,
                     int32_t mode, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (np < 0 || nturns < 0) return fail(ATB_ERR_ARG, "negative size");
    if (np > 0 && !r) return fail(ATB_ERR_ARG, "r is NULL");
    if (losses && np > 0 && (!islost || !lturn || !lelem || !lcoord))
        return fail(ATB_ERR_ARG, "loss map buffers missing");
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return fail(ATB_ERR_ARG, "bad mode");
    if (np == 0 || nturns == 0) return ATB_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    std::vector<const Lattice*> lats{L};
    int smem = 0, grid_max = 0;
    bool gen = false;
    int rc = kernel_config(h, lats, mode, &smem, &grid_max, &gen);
    if (rc) return rc;
    AtbJob J;
    std::memset(&J, 0, sizeof(J));
    fill_job_lattice(J, *L, 0, L->nelem);
    J.rng.key = job_key(h, 0);
    J.check_loss = 1;
    J.r = r;
    J.np = np;
    J.turn0 = turn0;
    J.nturns = nturns;
    J.losses = losses ? 1 : 0;
    J.lost = islost;
    J.lturn = lturn;
    J.lelem = lelem;
    J.lcoord = lcoord;
    J.alive = alive;
    J.moments = moments;
    std::vector<AtbJob> jobs{J};
    h->h_tiles.clear();
    const int pp = gen ? 1 : ppt_for(h, np);
    const int thr = pp > 1 ? h->threads : threads_for(h, np);
    make_tiles(h->h_tiles, 0, np, thr * pp);
    /* pageable-source copies of the launch lists are staged before
       cudaMemcpyAsync returns, so the host vectors may be reused at once */
    return launch(h, jobs, h->h_tiles, smem, grid_max, mode, st, thr, pp, gen);
}

int atb_element_maps(atb_handle* h, int32_t id, const double* orbits, double* m66,
                     double* b66, double diff_const, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (L->nelem == 0) return ATB_OK;
    if (!orbits || !m66 || !b66) return fail(ATB_ERR_ARG, "NULL buffer");
    for (int e = 0; e < L->nelem; ++e)
        if ((L->hdr[e] >> ATB_H_FL_SHIFT) & ATB_F_INTEG)
            return fail(ATB_ERR_ARG, "element maps need a lattice compiled for the default "
                                     "integrator (4)");
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    AtbElemMaps A;
    std::memset(&A, 0, sizeof(A));
    A.table = L->words.as<double>();
    A.elem_off = L->doff.as<uint32_t>();
    A.nelem = L->nelem;
    A.orbits = orbits;
    A.m66 = m66;
    A.b66 = b66;
    A.diff_const = diff_const;
    const int blocks = (L->nelem + ATB_TANGENT_THREADS - 1) / ATB_TANGENT_THREADS;
    atb_element_maps_kernel<<<blocks, ATB_TANGENT_THREADS, 0, st>>>(A);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

int atb_element_pass(atb_handle* h, int32_t id, const double* r_in, double* r_out, double* m66,
                     void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (L->nelem == 0) return ATB_OK;
    if (!r_in || !r_out) return fail(ATB_ERR_ARG, "NULL buffer");
    for (int e = 0; e < L->nelem; ++e)
        if ((L->hdr[e] >> ATB_H_FL_SHIFT) & ATB_F_INTEG)
            return fail(ATB_ERR_ARG, "element passes need a lattice compiled for the default "
                                     "integrator (4)");
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    AtbElemMaps A;
    std::memset(&A, 0, sizeof(A));
    A.table = L->words.as<double>();
    A.elem_off = L->doff.as<uint32_t>();
    A.nelem = L->nelem;
    A.orbits = r_in;
    A.m66 = m66;
    A.exits = r_out;
    const int blocks = (L->nelem + ATB_TANGENT_THREADS - 1) / ATB_TANGENT_THREADS;
    atb_element_maps_kernel<<<blocks, ATB_TANGENT_THREADS, 0, st>>>(A);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

/* Checks shared by the derivative kernels: the lattice uses the default
   integrator (the kernels integrate with the CPU engine's Forest-Ruth steps),
   and each differentiated strength is PolynomB[k], k in [1, MaxOrder], of a
   multipole element carrying no other strength.  Builds the per-element
   parameter index in h->h_pelem. */
int strength_map(atb_handle* h, const Lattice* L, const int32_t* param_elem,
                 const int32_t* param_order, int32_t nparam, const char* who) {
    for (int e = 0; e < L->nelem; ++e)
        if ((L->hdr[e] >> ATB_H_FL_SHIFT) & ATB_F_INTEG)
            return fail(ATB_ERR_ARG, std::string("the ") + who +
                                         " kernel needs a lattice compiled for the "
                                         "default integrator (4)");
    h->h_pelem.assign((size_t)std::max(L->nelem, 1), -1);
    for (int q = 0; q < nparam; ++q) {
        const int e = param_elem[q];
        const int k = param_order[q];
        if (e < 0 || e >= L->nelem) return fail(ATB_ERR_ARG, "parameter element out of range");
        if (h->h_pelem[e] >= 0)
            return fail(ATB_ERR_ARG, "element " + std::to_string(e) + " has two parameters");
        const uint64_t hd = L->hdr[e];
        const int op = (int)((hd >> ATB_H_OP_SHIFT) & ATB_H_OP_MASK);
        const int mo = (int)((hd >> ATB_H_MO_SHIFT) & ATB_H_MO_MASK);
        const uint32_t fl = (uint32_t)((hd >> ATB_H_FL_SHIFT) & ATB_H_FL_MASK);
        if (op != ATB_OP_STRMPOLE && op != ATB_OP_STRMPOLE_RAD && op != ATB_OP_BNDMPOLE &&
            op != ATB_OP_BNDMPOLE_RAD && op != ATB_OP_THINMPOLE)
            return fail(ATB_ERR_ARG, "element " + std::to_string(e) + " has no PolynomB");
        if (k < 1 || k > mo)
            return fail(ATB_ERR_ARG, "PolynomB order " + std::to_string(k) +
                                         " outside [1, MaxOrder] of element " +
                                         std::to_string(e));
        if (k == 1 && (fl & (ATB_F_FQ_IN_LIN | ATB_F_FQ_OUT_LIN)))
            return fail(ATB_ERR_ARG, "element " + std::to_string(e) +
                                         ": linear quadrupole-fringe maps are not differentiated");
        h->h_pelem[e] = q;
    }
    return ATB_OK;
}

int atb_tangent_device(atb_handle* h, int32_t id, double* r, int64_t np, int32_t nturns,
                       int32_t turn0, const int32_t* param_elem, const int32_t* param_order,
                       const double* param_value, int32_t nparam, double* jac, double* grad,
                       uint8_t* islost, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (np < 0 || nturns < 0 || nparam < 0) return fail(ATB_ERR_ARG, "negative size");
    if (np > 0 && (!r || !jac)) return fail(ATB_ERR_ARG, "r or jac is NULL");
    if (nparam > 0 && (!param_elem || !param_order || !param_value || (np > 0 && !grad)))
        return fail(ATB_ERR_ARG, "parameter arrays missing");
    const int rc = strength_map(h, L, param_elem, param_order, nparam, "tangent");
    if (rc != ATB_OK) return rc;
    if (np == 0) return ATB_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    AtbTangent A;
    std::memset(&A, 0, sizeof(A));
    A.table = L->words.as<double>();
    A.elem_off = L->doff.as<uint32_t>();
    A.nelem = L->nelem;
    A.nturns = nturns;
    A.turn0 = turn0;
    A.nparam = nparam;
    A.r = r;
    A.np = np;
    if (nparam > 0) {
        if (h->tan_pelem.ensure(h->h_pelem.size() * 4) != cudaSuccess ||
            h->tan_porder.ensure((size_t)nparam * 4) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(parameter map) failed");
        /* pageable sources are staged before cudaMemcpyAsync returns */
        ATB_CUDA(cudaMemcpyAsync(h->tan_pelem.p, h->h_pelem.data(), h->h_pelem.size() * 4,
                                 cudaMemcpyHostToDevice, st));
        ATB_CUDA(cudaMemcpyAsync(h->tan_porder.p, param_order, (size_t)nparam * 4,
                                 cudaMemcpyHostToDevice, st));
        A.pelem = h->tan_pelem.as<int32_t>();
        A.porder = h->tan_porder.as<int32_t>();
        A.pvalue = param_value;
    }
    A.jac = jac;
    A.grad = grad;
    A.lost = islost;
    const long long blocks = (np + ATB_TANGENT_THREADS - 1) / ATB_TANGENT_THREADS;
    if (blocks > 0x7fffffffLL) return fail(ATB_ERR_ARG, "too many particles");
    atb_tangent_kernel<<<(unsigned)blocks, ATB_TANGENT_THREADS, 0, st>>>(A);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

/* the adjoint kernels' descriptor with the lattice and the strength map
   (uploaded on st) */
int adjoint_setup(atb_handle* h, const Lattice* L, const int32_t* param_order,
                  const double* param_value, int32_t nparam, cudaStream_t st, AtbAdjoint& A) {
    std::memset(&A, 0, sizeof(A));
    A.table = L->words.as<double>();
    A.elem_off = L->doff.as<uint32_t>();
    A.nelem = L->nelem;
    A.nparam = nparam;
    if (nparam > 0) {
        if (h->adj_pelem.ensure(h->h_pelem.size() * 4) != cudaSuccess ||
            h->adj_porder.ensure((size_t)nparam * 4) != cudaSuccess)
            return fail(ATB_ERR_NOMEM, "cudaMalloc(parameter map) failed");
        /* pageable sources are staged before cudaMemcpyAsync returns */
        ATB_CUDA(cudaMemcpyAsync(h->adj_pelem.p, h->h_pelem.data(), h->h_pelem.size() * 4,
                                 cudaMemcpyHostToDevice, st));
        ATB_CUDA(cudaMemcpyAsync(h->adj_porder.p, param_order, (size_t)nparam * 4,
                                 cudaMemcpyHostToDevice, st));
        A.pelem = h->adj_pelem.as<int32_t>();
        A.porder = h->adj_porder.as<int32_t>();
        A.pvalue = param_value;
    }
    return ATB_OK;
}

unsigned adjoint_blocks(int64_t n) {
    return (unsigned)((n + ATB_ADJ_THREADS - 1) / ATB_ADJ_THREADS);
}

int atb_adjoint_forward(atb_handle* h, int32_t id, double* r, int64_t np, int32_t nturns,
                        int32_t turn0, const int32_t* param_elem, const int32_t* param_order,
                        const double* param_value, int32_t nparam, double* ckpt,
                        int32_t stride, double* estates, uint8_t* islost, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (np < 0 || nturns < 0 || nparam < 0) return fail(ATB_ERR_ARG, "negative size");
    if (stride < 1) return fail(ATB_ERR_ARG, "checkpoint stride must be at least 1");
    if (np > 0 && !r) return fail(ATB_ERR_ARG, "r is NULL");
    if (nparam > 0 && (!param_elem || !param_order || !param_value))
        return fail(ATB_ERR_ARG, "parameter arrays missing");
    if (np > (int64_t)ATB_ADJ_THREADS * 0x7fffffffLL) return fail(ATB_ERR_ARG, "too many particles");
    if (estates && (stride != 1 || !ckpt))
        return fail(ATB_ERR_ARG, "element states need a checkpoint every turn");
    const int rc = strength_map(h, L, param_elem, param_order, nparam, "adjoint");
    if (rc != ATB_OK) return rc;
    if (np == 0) return ATB_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    AtbAdjoint A;
    const int rs = adjoint_setup(h, L, param_order, param_value, nparam, st, A);
    if (rs != ATB_OK) return rs;
    A.nturns = nturns;
    A.turn0 = turn0;
    A.stride = stride;
    A.np = np;
    A.ld = np;
    A.r = r;
    A.ckpt = ckpt;
    A.lost = islost;
    A.scratch = estates;
    atb_adjoint_forward_kernel<<<adjoint_blocks(np), ATB_ADJ_THREADS, 0, st>>>(A);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

int atb_adjoint_backward(atb_handle* h, int32_t id, const double* ckpt, int64_t np,
                         int32_t nturns, int32_t turn0, int32_t stride, const double* estates,
                         const double* rfinal, const int32_t* param_elem,
                         const int32_t* param_order, const double* param_value, int32_t nparam,
                         double* lam, double* gparam, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Lattice* L = get_lat(h, id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (np < 0 || nturns < 0 || nparam < 0) return fail(ATB_ERR_ARG, "negative size");
    if (stride < 1) return fail(ATB_ERR_ARG, "checkpoint stride must be at least 1");
    if (np > 0 && nturns > 0 && (!ckpt || !lam)) return fail(ATB_ERR_ARG, "ckpt or lam is NULL");
    if (nparam > 0 && (!param_elem || !param_order || !param_value || !gparam))
        return fail(ATB_ERR_ARG, "parameter arrays missing");
    if (estates && (stride != 1 || !rfinal))
        return fail(ATB_ERR_ARG, "element states need a checkpoint every turn and the final "
                                 "states");
    if (((size_t)nparam + (size_t)ATB_ADJ_STEPS_SMEM * 4 * ATB_ADJ_THREADS) * sizeof(double) >
        48 * 1024)
        return fail(ATB_ERR_ARG, "at most 1024 strengths");
    if (np > (int64_t)ATB_ADJ_THREADS * 0x7fffffffLL) return fail(ATB_ERR_ARG, "too many particles");
    const int rc = strength_map(h, L, param_elem, param_order, nparam, "adjoint");
    if (rc != ATB_OK) return rc;
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    if (nparam > 0) ATB_CUDA(cudaMemsetAsync(gparam, 0, (size_t)nparam * sizeof(double), st));
    if (np == 0 || nturns == 0) return ATB_OK;
    AtbAdjoint A;
    const int rs = adjoint_setup(h, L, param_order, param_value, nparam, st, A);
    if (rs != ATB_OK) return rs;
    const size_t smem_e =
        ((size_t)nparam + (size_t)ATB_ADJ_STEPS_SMEM * 4 * ATB_ADJ_THREADS) * sizeof(double);
    if (estates) {
        /* every turn's element-entry states were stored by the forward pass:
           no tracking here, all particles in one launch per turn */
        A.gparam = gparam;
        for (int t = nturns - 1; t >= 0; --t) {
            AtbAdjoint T = A;
            T.np = np;
            T.ckpt = const_cast<double*>(ckpt + 6 * ((int64_t)t * np));
            T.lam = lam;
            T.turn0 = turn0 + t;
            T.scratch = const_cast<double*>(estates) + 6 * ((int64_t)t * L->nelem * np);
            T.next = (t + 1 < nturns) ? ckpt + 6 * ((int64_t)(t + 1) * np) : rfinal;
            atb_adjoint_turn_kernel<<<adjoint_blocks(np), ATB_ADJ_THREADS, smem_e, st>>>(T);
        }
        ATB_CUDA(cudaGetLastError());
        return ATB_OK;
    }
    /* particles in chunks whose element-entry scratch fits 8 GiB */
    const int64_t per = (int64_t)std::max(L->nelem, 1) * 6 * sizeof(double);
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(np, (8LL << 30) / per));
    if (h->adj_scratch.ensure((size_t)(chunk * per)) != cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(adjoint scratch) failed");
    if (stride > 1 &&
        (h->adj_block.ensure((size_t)stride * chunk * 6 * sizeof(double)) != cudaSuccess ||
         h->adj_state.ensure((size_t)chunk * 6 * sizeof(double)) != cudaSuccess))
        return fail(ATB_ERR_NOMEM, "cudaMalloc(adjoint checkpoints) failed");
    const int nck = (nturns + stride - 1) / stride;
    const size_t smem =
        ((size_t)nparam + (size_t)ATB_ADJ_STEPS_SMEM * 4 * ATB_ADJ_THREADS) * sizeof(double);
    A.gparam = gparam;
    A.scratch = h->adj_scratch.as<double>();
    for (int64_t p0 = 0; p0 < np; p0 += chunk) {
        const int64_t n = std::min(chunk, np - p0);
        double* lp = lam + 6 * p0;
        for (int b = nck - 1; b >= 0; --b) {
            const int t0 = b * stride;
            const int nt = std::min(stride, nturns - t0);
            const double* slab = ckpt + 6 * ((int64_t)b * np + p0);
            if (stride == 1) {
                AtbAdjoint T = A;
                T.np = n;
                T.ckpt = const_cast<double*>(slab);
                T.lam = lp;
                T.turn0 = turn0 + t0;
                atb_adjoint_turn_kernel<<<adjoint_blocks(n), ATB_ADJ_THREADS, smem, st>>>(T);
                continue;
            }
            /* the block's turn entries, tracked again from its checkpoint */
            double* tmp = h->adj_state.as<double>();
            double* blk = h->adj_block.as<double>();
            ATB_CUDA(cudaMemcpyAsync(tmp, slab, (size_t)n * 6 * sizeof(double),
                                     cudaMemcpyDeviceToDevice, st));
            AtbAdjoint F = A;
            F.np = n;
            F.ld = n;
            F.r = tmp;
            F.ckpt = blk;
            F.nturns = nt;
            F.turn0 = turn0 + t0;
            F.stride = 1;
            F.skip_last = 1;
            F.scratch = nullptr;       /* no element states from this re-tracking */
            atb_adjoint_forward_kernel<<<adjoint_blocks(n), ATB_ADJ_THREADS, 0, st>>>(F);
            for (int t = nt - 1; t >= 0; --t) {
                AtbAdjoint T = A;
                T.np = n;
                T.ckpt = blk + 6 * ((int64_t)t * n);
                T.lam = lp;
                T.turn0 = turn0 + t0 + t;
                atb_adjoint_turn_kernel<<<adjoint_blocks(n), ATB_ADJ_THREADS, smem, st>>>(T);
            }
        }
    }
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

int atb_track_batch(atb_handle* h, const atb_job_desc* jobs, int32_t njobs, int32_t mode,
                    void* stream) {
    if (!h || (njobs > 0 && !jobs)) return fail(ATB_ERR_ARG, "NULL argument");
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return fail(ATB_ERR_ARG, "bad mode");
    if (njobs <= 0) return ATB_OK;
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    std::vector<const Lattice*> lats;
    std::vector<AtbJob> J(njobs);
    for (int j = 0; j < njobs; ++j) {
        const atb_job_desc& d = jobs[j];
        Lattice* L = get_lat(h, d.lattice_id);
        if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id in batch");
        if (d.np < 0 || d.nturns < 0 || (d.np > 0 && !d.r))
            return fail(ATB_ERR_ARG, "invalid batch job");
        if (d.losses && d.np > 0 && (!d.islost || !d.lturn || !d.lelem || !d.lcoord))
            return fail(ATB_ERR_ARG, "loss map buffers missing in batch job");
        lats.push_back(L);
        std::memset(&J[j], 0, sizeof(AtbJob));
        fill_job_lattice(J[j], *L, 0, L->nelem);
        J[j].rng.key = job_key(h, j);
        J[j].check_loss = 1;
        J[j].r = d.r;
        J[j].np = d.np;
        J[j].turn0 = d.turn0;
        J[j].nturns = d.nturns;
        J[j].losses = d.losses ? 1 : 0;
        J[j].lost = d.islost;
        J[j].lturn = d.lturn;
        J[j].lelem = d.lelem;
        J[j].lcoord = d.lcoord;
    }
    int smem = 0, grid_max = 0;
    bool gen = false;
    int rc = kernel_config(h, lats, mode, &smem, &grid_max, &gen);
    if (rc) return rc;
    /* longest-processing-time first: order jobs by turns x elements */
    std::vector<int> order(njobs);
    for (int j = 0; j < njobs; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        double ca = (double)J[a].nturns * (lats[a]->nwords + 1);
        double cb = (double)J[b].nturns * (lats[b]->nwords + 1);
        return ca > cb;
    });
    const int pp = gen ? 1 : h->ppt;
    make_claims(h, h->h_tiles, J, order, grid_max, 1, pp);
    return launch(h, J, h->h_tiles, smem, grid_max, mode, st, h->threads, pp, gen);
}

int atb_batch_prepare(atb_handle* h, const atb_job_desc* jobs, int32_t njobs, int32_t mode,
                      int32_t* batch_id) {
    if (!h || !batch_id || (njobs > 0 && !jobs)) return fail(ATB_ERR_ARG, "NULL argument");
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return fail(ATB_ERR_ARG, "bad mode");
    DeviceGuard g(h->device);
    std::vector<const Lattice*> lats;
    std::vector<AtbJob> J(njobs > 0 ? njobs : 0);
    for (int j = 0; j < njobs; ++j) {
        const atb_job_desc& d = jobs[j];
        Lattice* L = get_lat(h, d.lattice_id);
        if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id in batch");
        if (d.np < 0 || d.nturns < 0 || (d.np > 0 && !d.r))
            return fail(ATB_ERR_ARG, "invalid batch job");
        if (d.losses && d.np > 0 && (!d.islost || !d.lturn || !d.lelem || !d.lcoord))
            return fail(ATB_ERR_ARG, "loss map buffers missing in batch job");
        lats.push_back(L);
        std::memset(&J[j], 0, sizeof(AtbJob));
        fill_job_lattice(J[j], *L, 0, L->nelem);
        J[j].rng.key = job_key(h, j);
        J[j].check_loss = 1;
        J[j].r = d.r;
        J[j].np = d.np;
        J[j].turn0 = d.turn0;
        J[j].nturns = d.nturns;
        J[j].losses = d.losses ? 1 : 0;
        J[j].lost = d.islost;
        J[j].lturn = d.lturn;
        J[j].lelem = d.lelem;
        J[j].lcoord = d.lcoord;
    }
    int smem = 0, grid_max = 0;
    bool gen = false;
    if (!lats.empty()) {
        int rc = kernel_config(h, lats, mode, &smem, &grid_max, &gen);
        if (rc) return rc;
    }
    std::vector<int> order(J.size());
    for (size_t j = 0; j < J.size(); ++j) order[j] = (int)j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)J[a].nturns * (lats[a]->nwords + 1) * 1.0 >
               (double)J[b].nturns * (lats[b]->nwords + 1) * 1.0;
    });
    std::vector<AtbTile> tiles;
    make_claims(h, tiles, J, order, grid_max, h->refill_k, gen ? 1 : h->ppt);
    int id = -1;
    for (int i = 0; i < (int)h->batches.size(); ++i)
        if (!h->batches[i].used) { id = i; break; }
    if (id < 0) {
        h->batches.emplace_back();
        id = (int)h->batches.size() - 1;
    }
    Batch& B = h->batches[id];
    if (B.jobs.ensure(std::max<size_t>(1, J.size()) * sizeof(AtbJob)) != cudaSuccess ||
        B.tiles.ensure(std::max<size_t>(1, tiles.size()) * sizeof(AtbTile)) != cudaSuccess ||
        B.counter.ensure(sizeof(int)) != cudaSuccess ||
        B.jobnext.ensure(std::max<size_t>(1, J.size()) * sizeof(unsigned long long)) !=
            cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(batch lists) failed");
    if (!J.empty())
        ATB_CUDA(cudaMemcpy(B.jobs.p, J.data(), J.size() * sizeof(AtbJob), cudaMemcpyHostToDevice));
    if (!tiles.empty())
        ATB_CUDA(cudaMemcpy(B.tiles.p, tiles.data(), tiles.size() * sizeof(AtbTile),
                            cudaMemcpyHostToDevice));
    B.used = true;
    B.mode = mode;
    B.threads = h->threads;
    B.ppt = gen ? 1 : h->ppt;
    B.gen = gen;
    B.seg_cap = h->seg_cap_words;
    B.smem = smem;
    B.ntiles = (int)tiles.size();
    B.njobs = (int)J.size();
    B.grid = std::min<int64_t>((int64_t)tiles.size(), std::max(grid_max, 1));
    if (B.scratch.ensure((size_t)B.grid * B.threads * ATB_COMPACT_WORDS * sizeof(double)) !=
        cudaSuccess) {
        B.used = false;
        return fail(ATB_ERR_NOMEM, "cudaMalloc(compaction scratch) failed");
    }
    *batch_id = id;
    return ATB_OK;
}

static Batch* get_batch(atb_handle* h, int id) {
    if (id < 0 || id >= (int)h->batches.size() || !h->batches[id].used) return nullptr;
    return &h->batches[id];
}

static int batch_enqueue(atb_handle* h, Batch& B, cudaStream_t st) {
    ATB_CUDA(cudaMemsetAsync(B.counter.p, 0, sizeof(int), st));
    if (B.ntiles == 0) return ATB_OK;
    ATB_CUDA(cudaMemsetAsync(B.jobnext.p, 0, (size_t)B.njobs * sizeof(unsigned long long), st));
    const AtbJob* dj = B.jobs.as<AtbJob>();
    const AtbTile* dt = B.tiles.as<AtbTile>();
    int* cnt = B.counter.as<int>();
    unsigned long long* jn = B.jobnext.as<unsigned long long>();
    int* sts = h->status.as<int>();
    double* scr = B.scratch.as<double>();
    if (B.gen && B.mode == ATB_MODE_EXACT)
        atb_track_kernel_exact_gen<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn,
                                                                      sts, B.seg_cap, scr);
    else if (B.gen)
        atb_track_kernel_fast_gen<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn,
                                                                     sts, B.seg_cap, scr);
    else if (B.mode == ATB_MODE_EXACT && B.ppt == 2)
        atb_track_kernel_exact_np2<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn,
                                                                      sts, B.seg_cap, scr);
    else if (B.mode == ATB_MODE_EXACT)
        atb_track_kernel_exact<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn, sts,
                                                                  B.seg_cap, scr);
    else if (B.ppt == 2)
        atb_track_kernel_fast_np2<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn,
                                                                     sts, B.seg_cap, scr);
    else
        atb_track_kernel_fast<<<B.grid, B.threads, B.smem, st>>>(dj, dt, B.ntiles, cnt, jn, sts,
                                                                 B.seg_cap, scr);
    ATB_CUDA(cudaGetLastError());
    return ATB_OK;
}

int atb_batch_capture(atb_handle* h, int32_t batch_id) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Batch* B = get_batch(h, batch_id);
    if (!B) return fail(ATB_ERR_ARG, "unknown batch id");
    DeviceGuard g(h->device);
    if (B->exec) {
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    if (B->graph) {
        cudaGraphDestroy(B->graph);
        B->graph = nullptr;
    }
    ATB_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = batch_enqueue(h, *B, h->stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(ATB_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    B->graph = graph;
    ATB_CUDA(cudaGraphInstantiate(&B->exec, graph, 0));
    return ATB_OK;
}

int atb_batch_launch(atb_handle* h, int32_t batch_id, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Batch* B = get_batch(h, batch_id);
    if (!B) return fail(ATB_ERR_ARG, "unknown batch id");
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    if (B->exec) {
        ATB_CUDA(cudaGraphLaunch(B->exec, st));
        return ATB_OK;
    }
    return batch_enqueue(h, *B, st);
}

int atb_batch_free(atb_handle* h, int32_t batch_id) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    Batch* B = get_batch(h, batch_id);
    if (!B) return fail(ATB_ERR_ARG, "unknown batch id");
    DeviceGuard g(h->device);
    cudaStreamSynchronize(h->stream);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
    B->jobs.release();
    B->tiles.release();
    B->counter.release();
    B->scratch.release();
    B->jobnext.release();
    B->used = false;
    return ATB_OK;
}

int atb_fp64_peak(int device, double* tflops, double* seconds) {
    if (!tflops) return fail(ATB_ERR_ARG, "tflops is NULL");
    DeviceGuard g(device);
    cudaDeviceProp p;
    ATB_CUDA(cudaGetDeviceProperties(&p, device));
    const int threads = 256, blocks = p.multiProcessorCount * 8, iters = 4096;
    double* out = nullptr;
    ATB_CUDA(cudaMalloc(&out, sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    atb_dfma_probe<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);   /* warm-up */
    cudaEventRecord(e0);
    atb_dfma_probe<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return fail(ATB_ERR_CUDA, cudaGetErrorString(err));
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *tflops = flops / (ms * 1e-3) / 1e12;
    if (seconds) *seconds = ms * 1e-3;
    return ATB_OK;
}

int atb_set_rng(atb_handle* h, uint64_t key) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    h->rng_key = key;
    return ATB_OK;
}

int atb_sync(atb_handle* h, void* stream) {
    if (!h) return fail(ATB_ERR_ARG, "handle is NULL");
    DeviceGuard g(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    return check_status(h, st);
}

/* ---------------- the serving loop ------------------------------------------ */

namespace {

static_assert(sizeof(AtbTile) == 16 && sizeof(AtbServeCont) == 32,
              "the serving kernel reads tiles with 16-byte vector loads");

/* the ring cursors: ATB_SERVE_CLASSES heads, as many tails, the in-flight
   count (and one spare) */
constexpr int kRingCtr = 2 * ATB_SERVE_CLASSES + 2;

/* The continuation rings' cursors, read through pinned memory: whether any
   ring holds work, and the entries written and taken over all rings. */
int ring_cursors(atb_server* s, bool* pending, long long* written, long long* taken) {
    int* hc = reinterpret_cast<int*>(&s->h_done[s->max_jobs + 2]);
    ATB_CUDA(cudaMemcpyAsync(hc, s->ring_ctr.p, 2 * ATB_SERVE_CLASSES * sizeof(int),
                             cudaMemcpyDeviceToHost, s->cstream));
    ATB_CUDA(cudaStreamSynchronize(s->cstream));
    bool p = false;
    long long w = 0, t = 0;
    for (int q = 0; q < ATB_SERVE_CLASSES; ++q) {
        const int h = hc[q], tl = hc[ATB_SERVE_CLASSES + q];
        p |= h < tl;
        w += tl;
        t += h;
    }
    if (pending) *pending = p;
    if (written) *written = w;
    if (taken) *taken = t;
    return ATB_OK;
}

AtbServeArgs serve_args(atb_server* s) {
    AtbServeArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ctl = s->dctl;
    a.ring.slots = s->ring.as<AtbServeCont>();
    a.ring.cap = s->ring_cap;
    a.ring.nring = ATB_SERVE_CLASSES;
    a.ring.head = s->ring_ctr.as<int>();
    a.ring.tail = s->ring_ctr.as<int>() + ATB_SERVE_CLASSES;
    a.inflight = s->ring_ctr.as<int>() + 2 * ATB_SERVE_CLASSES;
    a.done = s->done.as<unsigned long long>();
    return a;
}

int serve_launch(atb_server* s) {
    const AtbJob* dj = s->jobs.as<AtbJob>();
    const AtbTile* dt = s->tiles.as<AtbTile>();
    int* cnt = s->counter.as<int>();
    int* sts = s->status.as<int>();
    double* scr = s->compact.as<double>();
    const AtbServeArgs a = serve_args(s);
    if (s->mode == ATB_MODE_EXACT)
        atb_serve_kernel_exact<<<s->grid, s->threads, s->smem, s->kstream>>>(
            dj, dt, a, cnt, sts, s->seg_cap, scr);
    else
        atb_serve_kernel_fast<<<s->grid, s->threads, s->smem, s->kstream>>>(
            dj, dt, a, cnt, sts, s->seg_cap, scr);
    ATB_CUDA(cudaGetLastError());
    s->launched = true;
    return ATB_OK;
}

/* the kernel left (stop, idle, or a failed wait): 1, still running: 0 */
int serve_finished(atb_server* s) {
    if (!s->launched) return 1;
    cudaError_t e = cudaStreamQuery(s->kstream);
    if (e == cudaErrorNotReady) return 0;
    s->launched = false;
    return 1;
}

}  // namespace

int atb_serve_open(atb_handle* h, const int32_t* lattice_ids, int32_t nlat, int32_t mode,
                   int32_t max_jobs, int32_t max_tiles, atb_server** out) {
    if (!h || !out || (nlat > 0 && !lattice_ids)) return fail(ATB_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return fail(ATB_ERR_ARG, "bad mode");
    if (nlat <= 0 || max_jobs <= 0 || max_tiles <= 0)
        return fail(ATB_ERR_ARG, "a server needs lattices and positive capacities");
    DeviceGuard g(h->device);
    std::vector<const Lattice*> lats;
    for (int i = 0; i < nlat; ++i) {
        Lattice* L = get_lat(h, lattice_ids[i]);
        if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
        if (L->integ)
            return fail(ATB_ERR_ARG, "the serving loop runs the default integrator (4) only");
        lats.push_back(L);
    }
    std::unique_ptr<atb_server> s(new atb_server());
    s->h = h;
    s->mode = mode;
    s->max_jobs = max_jobs;
    s->max_tiles = max_tiles;
    s->threads = h->threads;
    s->seg_cap = h->seg_cap_words;
    s->lattice_ids.assign(lattice_ids, lattice_ids + nlat);
    int per_sm = 0;
    {
        /* shared memory for the largest table of the pool; one particle per
           thread */
        bool any_pipe = false;
        int64_t res_words = 0;
        for (const Lattice* L : lats) {
            if (L->resident) res_words = std::max<int64_t>(res_words, L->nwords + (L->nwords & 1));
            else if (!L->segs.empty()) any_pipe = true;
        }
        int64_t words = std::max<int64_t>(any_pipe ? 2LL * s->seg_cap : 0, res_words);
        s->smem = (int)(words * 8);
        if (s->smem > h->smem_optin) return fail(ATB_ERR_ARG, "shared-memory plan too large");
        const void* fn = mode == ATB_MODE_EXACT ? (const void*)atb_serve_kernel_exact
                                                : (const void*)atb_serve_kernel_fast;
        ATB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      h->smem_optin));
        ATB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, s->threads, s->smem));
        if (per_sm < 1) return fail(ATB_ERR_ARG, "launch configuration does not fit on an SM");
    }
    s->grid = per_sm * h->sm_count;
    if (s->jobs.ensure((size_t)max_jobs * sizeof(AtbJob)) != cudaSuccess ||
        s->tiles.ensure((size_t)max_tiles * sizeof(AtbTile)) != cudaSuccess ||
        s->counter.ensure(sizeof(int)) != cudaSuccess ||
        s->status.ensure(sizeof(int)) != cudaSuccess ||
        s->jobnext.ensure((size_t)max_jobs * sizeof(unsigned long long)) != cudaSuccess ||
        s->done.ensure((size_t)max_jobs * sizeof(unsigned long long)) != cudaSuccess ||
        s->compact.ensure((size_t)s->grid * s->threads * ATB_COMPACT_WORDS * sizeof(double)) !=
            cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(serving queue) failed");
    /* continuation ring: a power of two at least the tile capacity (every
       live tile has at most one entry) */
    s->ring_cap = 1;
    while (s->ring_cap < max_tiles + 128) s->ring_cap <<= 1;
    if (s->ring.ensure((size_t)ATB_SERVE_CLASSES * s->ring_cap * sizeof(AtbServeCont)) !=
            cudaSuccess ||
        s->ring_ctr.ensure(kRingCtr * sizeof(int)) != cudaSuccess)
        return fail(ATB_ERR_NOMEM, "cudaMalloc(continuation ring) failed");
    ATB_CUDA(cudaHostAlloc((void**)&s->ctl, sizeof(AtbServeCtl), cudaHostAllocMapped));
    ATB_CUDA(cudaHostGetDevicePointer((void**)&s->dctl, s->ctl, 0));
    s->ctl->published = 0;
    s->ctl->stop = 0;
    ATB_CUDA(cudaHostAlloc((void**)&s->h_done, ((size_t)max_jobs + 2 + ATB_SERVE_CLASSES) * sizeof(unsigned long long),
                           cudaHostAllocDefault));
    ATB_CUDA(cudaHostAlloc((void**)&s->h_job, sizeof(AtbJob), cudaHostAllocDefault));
    ATB_CUDA(cudaHostAlloc((void**)&s->h_zero, 2 * sizeof(unsigned long long),
                           cudaHostAllocDefault));
    s->h_zero[0] = s->h_zero[1] = 0ULL;
    ATB_CUDA(cudaStreamCreateWithFlags(&s->kstream, cudaStreamNonBlocking));
    ATB_CUDA(cudaStreamCreateWithFlags(&s->cstream, cudaStreamNonBlocking));
    ATB_CUDA(cudaMemsetAsync(s->counter.p, 0, sizeof(int), s->cstream));
    ATB_CUDA(cudaMemsetAsync(s->status.p, 0, sizeof(int), s->cstream));
    ATB_CUDA(cudaMemsetAsync(s->ring_ctr.p, 0, kRingCtr * sizeof(int), s->cstream));
    ATB_CUDA(cudaMemsetAsync(s->ring.p, 0,
                             (size_t)ATB_SERVE_CLASSES * s->ring_cap * sizeof(AtbServeCont),
                             s->cstream));
    ATB_CUDA(cudaStreamSynchronize(s->cstream));
    *out = s.release();
    return ATB_OK;
}

int atb_serve_submit(atb_server* s, const atb_job_desc* d, int32_t chunk_turns,
                     double turn_cost, int32_t* pidx, int32_t* slot) {
    if (!s || !d || !slot) return fail(ATB_ERR_ARG, "NULL argument");
    if (chunk_turns < 0) return fail(ATB_ERR_ARG, "negative chunk");
    atb_handle* h = s->h;
    if (std::find(s->lattice_ids.begin(), s->lattice_ids.end(), d->lattice_id) ==
        s->lattice_ids.end())
        return fail(ATB_ERR_ARG, "the job's lattice is not in this server's pool");
    Lattice* L = get_lat(h, d->lattice_id);
    if (!L) return fail(ATB_ERR_NOLAT, "unknown lattice id");
    if (d->np <= 0 || d->nturns <= 0 || !d->r) return fail(ATB_ERR_ARG, "invalid job");
    if (d->losses && (!d->islost || !d->lturn || !d->lelem || !d->lcoord))
        return fail(ATB_ERR_ARG, "loss map buffers missing");
    const int64_t ntl = (d->np + s->threads - 1) / s->threads;
    if (s->njobs >= s->max_jobs || s->ntiles + ntl > s->max_tiles)
        return fail(ATB_ERR_NOMEM, "serving queue full: wait for the published jobs and reset");
    DeviceGuard g(h->device);
    AtbJob& J = *s->h_job;
    std::memset(&J, 0, sizeof(AtbJob));
    fill_job_lattice(J, *L, 0, L->nelem);
    J.rng.key = job_key(h, s->njobs);
    J.check_loss = 1;
    J.r = d->r;
    J.np = d->np;
    J.turn0 = d->turn0;
    J.nturns = d->nturns;
    J.losses = d->losses ? 1 : 0;
    J.lost = d->islost;
    J.lturn = d->lturn;
    J.lelem = d->lelem;
    J.lcoord = d->lcoord;
    J.chunk = chunk_turns;
    J.turn_cost = turn_cost > 0.0 && std::isfinite(turn_cost) ? turn_cost : 0.0;
    J.pidx = pidx;
    if (ntl > s->h_tiles_cap) {
        if (s->h_tiles) cudaFreeHost(s->h_tiles);
        s->h_tiles = nullptr;
        s->h_tiles_cap = 0;
        ATB_CUDA(cudaHostAlloc((void**)&s->h_tiles, (size_t)ntl * sizeof(AtbTile),
                               cudaHostAllocDefault));
        s->h_tiles_cap = (int)ntl;
    }
    const int j = s->njobs;
    for (int64_t k = 0; k < ntl; ++k) {
        AtbTile& t = s->h_tiles[k];
        t.job = j;
        t.first = k * s->threads;
        t.count = (int32_t)std::min<int64_t>(s->threads, d->np - t.first);
    }
    /* records first; the kernel may see them only after these copies end.
       Everything here is a copy (copy engine): the persistent kernel holds
       the SMs, so a kernel-based memset would wait for it to leave. */
    ATB_CUDA(cudaMemcpyAsync(s->jobs.as<AtbJob>() + j, &J, sizeof(AtbJob),
                             cudaMemcpyHostToDevice, s->cstream));
    ATB_CUDA(cudaMemcpyAsync(s->tiles.as<AtbTile>() + s->ntiles, s->h_tiles,
                             (size_t)ntl * sizeof(AtbTile), cudaMemcpyHostToDevice, s->cstream));
    ATB_CUDA(cudaMemcpyAsync(s->jobnext.as<unsigned long long>() + j, s->h_zero,
                             sizeof(unsigned long long), cudaMemcpyHostToDevice, s->cstream));
    ATB_CUDA(cudaMemcpyAsync(s->done.as<unsigned long long>() + j, s->h_zero + 1,
                             sizeof(unsigned long long), cudaMemcpyHostToDevice, s->cstream));
    ATB_CUDA(cudaStreamSynchronize(s->cstream));
    s->njobs = j + 1;
    s->ntiles += (int)ntl;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    s->ctl->published = s->ntiles;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    *slot = j;
    if (serve_finished(s)) return serve_launch(s);
    return ATB_OK;
}

int atb_serve_poll(atb_server* s, int32_t first, int32_t nslots, uint64_t* done,
                   int32_t* running) {
    if (!s || (nslots > 0 && !done)) return fail(ATB_ERR_ARG, "NULL argument");
    if (first < 0 || nslots < 0 || first + nslots > s->njobs)
        return fail(ATB_ERR_ARG, "poll outside the submitted jobs");
    DeviceGuard g(s->h->device);
    if (nslots > 0)
        ATB_CUDA(cudaMemcpyAsync(s->h_done, s->done.as<unsigned long long>() + first,
                                 (size_t)nslots * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s->cstream));
    int claimed = 0, status = 0;
    ATB_CUDA(cudaMemcpyAsync(&s->h_done[s->max_jobs], s->counter.p, sizeof(int),
                             cudaMemcpyDeviceToHost, s->cstream));
    ATB_CUDA(cudaStreamSynchronize(s->cstream));
    std::memcpy(&claimed, &s->h_done[s->max_jobs], sizeof(int));
    for (int i = 0; i < nslots; ++i) done[i] = s->h_done[i];
    if (serve_finished(s)) {
        /* the kernel left: a failed wait is an error; after an idle exit it
           is launched again while published or re-enqueued work waits */
        bool pending = false;
        ATB_CUDA(cudaMemcpy(&status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost));
        const int rr = ring_cursors(s, &pending, nullptr, nullptr);
        if (rr) return rr;
        if (status & ATB_STATUS_WAIT_TIMEOUT)
            return fail(ATB_ERR_TIMEOUT, "a bounded shared-memory staging wait timed out");
        if ((claimed < s->ntiles || pending) && !s->ctl->stop) {
            int rc = serve_launch(s);
            if (rc) return rc;
        }
    }
    if (running) *running = s->launched ? 1 : 0;
    return ATB_OK;
}

int atb_serve_counters(atb_server* s, int32_t* out) {
    if (!s || !out) return fail(ATB_ERR_ARG, "NULL argument");
    DeviceGuard g(s->h->device);
    int c = 0;
    ATB_CUDA(cudaMemcpyAsync(&s->h_done[s->max_jobs], s->counter.p, sizeof(int),
                             cudaMemcpyDeviceToHost, s->cstream));
    ATB_CUDA(cudaStreamSynchronize(s->cstream));
    std::memcpy(&c, &s->h_done[s->max_jobs], sizeof(int));
    long long w = 0, t = 0;
    const int rr = ring_cursors(s, nullptr, &w, &t);
    if (rr) return rr;
    out[0] = s->ntiles;
    out[1] = c;
    out[2] = (int32_t)std::min<long long>(w, INT32_MAX);
    out[3] = (int32_t)std::min<long long>(t, INT32_MAX);
    return ATB_OK;
}

int atb_serve_reset(atb_server* s) {
    if (!s) return fail(ATB_ERR_ARG, "NULL argument");
    DeviceGuard g(s->h->device);
    s->ctl->stop = 1;
    ATB_CUDA(cudaStreamSynchronize(s->kstream));
    s->launched = false;
    int claimed = 0;
    ATB_CUDA(cudaMemcpy(&claimed, s->counter.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (claimed < s->ntiles)
        return fail(ATB_ERR_ARG, "reset with published work unclaimed");
    bool pending = false;
    const int rr = ring_cursors(s, &pending, nullptr, nullptr);
    if (rr) return rr;
    if (pending) return fail(ATB_ERR_ARG, "reset with continuations pending");
    ATB_CUDA(cudaMemset(s->counter.p, 0, sizeof(int)));
    ATB_CUDA(cudaMemset(s->status.p, 0, sizeof(int)));
    ATB_CUDA(cudaMemset(s->ring_ctr.p, 0, kRingCtr * sizeof(int)));
    ATB_CUDA(cudaMemset(s->ring.p, 0,
                        (size_t)ATB_SERVE_CLASSES * s->ring_cap * sizeof(AtbServeCont)));
    s->njobs = 0;
    s->ntiles = 0;
    s->ctl->published = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    s->ctl->stop = 0;
    return ATB_OK;
}

int atb_serve_close(atb_server* s) {
    if (!s) return ATB_OK;
    int rc = ATB_OK;
    {
        DeviceGuard g(s->h->device);
        if (s->ctl) s->ctl->stop = 1;
        if (s->kstream && cudaStreamSynchronize(s->kstream) != cudaSuccess)
            rc = fail(ATB_ERR_CUDA, "the serving kernel failed");
        int status = 0;
        if (s->status.p) cudaMemcpy(&status, s->status.p, sizeof(int), cudaMemcpyDeviceToHost);
        if (rc == ATB_OK && (status & ATB_STATUS_WAIT_TIMEOUT))
            rc = fail(ATB_ERR_TIMEOUT, "a bounded shared-memory staging wait timed out");
        for (DevBuf* b : {&s->jobs, &s->tiles, &s->counter, &s->status, &s->jobnext, &s->done,
                          &s->compact, &s->ring, &s->ring_ctr})
            b->release();
        if (s->ctl) cudaFreeHost(s->ctl);
        if (s->h_done) cudaFreeHost(s->h_done);
        if (s->h_job) cudaFreeHost(s->h_job);
        if (s->h_zero) cudaFreeHost(s->h_zero);
        if (s->h_tiles) cudaFreeHost(s->h_tiles);
        if (s->kstream) cudaStreamDestroy(s->kstream);
        if (s->cstream) cudaStreamDestroy(s->cstream);
    }
    delete s;
    return rc;
}

}  // extern "C"
