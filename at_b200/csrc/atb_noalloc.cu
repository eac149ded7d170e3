/*
 * atb_track_noalloc: multi-turn tracking of device-resident particles that
 * allocates no memory.
 *
 * Some callers cannot call cudaMalloc on their call path: a real-time loop
 * (for example an online model inside an accelerator's orbit or tune
 * feedback) must not, because cudaMalloc/cudaFree implicitly synchronise the
 * device and take an unbounded time; and an application whose device memory
 * is owned by another allocator (a framework pool that reserved the HBM up
 * front) cannot, because an extra cudaMalloc fails or fragments that pool.
 * The handle-based entry points of atb200.h allocate their launch lists on
 * first use, so these callers get this one entry point instead.  They pass
 * every input and output already on the device; the launch lists (one job,
 * the segment list, the tile list, the tile counter and the status word) live
 * in the fixed-size array below, which is part of the library image: every
 * GPU that loads the library holds ATB_NOALLOC_SCRATCH_BYTES of it until the
 * process exits.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/atb200.h"
#include "atb_kernel_api.h"
#include "atb_table.h"

extern "C" __global__ void atb_track_kernel_exact(const AtbJob*, const AtbTile*, int, int*,
                                                  unsigned long long*, int*, int, double*);
extern "C" __global__ void atb_track_kernel_fast(const AtbJob*, const AtbTile*, int, int*,
                                                 unsigned long long*, int*, int, double*);
extern "C" const char* atb_last_error(void);
void atb_set_error_message(const char* msg);

/* layout of the scratch array (byte offsets) */
#define NA_JOB 0
#define NA_COUNTER 256
#define NA_STATUS 260
#define NA_SEGS 512
#define NA_TILES (NA_SEGS + ATB_NOALLOC_MAX_SEGS * 24)
#define NA_THREADS 256
#define NA_SEG_CAP_WORDS 6144
#define NA_RESIDENT_MAX_WORDS 14336

static_assert(sizeof(AtbJob) <= NA_COUNTER, "job record does not fit its slot");
static_assert(sizeof(AtbSeg) == 24, "segment record size");
static_assert(sizeof(AtbTile) == 16, "tile record size");
static_assert(NA_TILES + ATB_NOALLOC_MAX_TILES * 16 <= ATB_NOALLOC_SCRATCH_BYTES,
              "scratch array too small for its layout");

/* The launch lists of atb_track_noalloc.  Host code must not use this name
 * as an address: it is a host-side stand-in.  The device address comes from
 * cudaGetSymbolAddress at set-up. */
static __device__ __align__(256) unsigned char atb_noalloc_scratch[ATB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_na_lock;
unsigned char* g_na_ptr[kMaxDevices] = {nullptr};

int na_fail(int code, const std::string& msg) {
    atb_set_error_message(msg.c_str());
    return code;
}

/* tile t covers particles [t*threads, min(np, (t+1)*threads)) */
__global__ void atb_noalloc_tiles(AtbTile* tiles, int ntiles, int64_t np, int threads) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int64_t first = (int64_t)t * threads;
    tiles[t].job = 0;
    tiles[t].first = first;
    tiles[t].count = (int32_t)((np - first) < threads ? (np - first) : threads);
}

/* Per-device set-up (first call on each device): the device address of the
 * scratch array and the kernels' shared-memory limit.  The limit is raised to
 * the device's opt-in maximum (less 1 KiB for the kernels' static shared
 * memory), the value atb_create sets: it is a process-wide property of the
 * kernel, so setting anything smaller here would shrink what handles set up
 * earlier rely on. */
int na_setup(int device, unsigned char** out) {
    std::lock_guard<std::mutex> g(g_na_lock);
    if (g_na_ptr[device]) {
        *out = g_na_ptr[device];
        return ATB_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, atb_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return na_fail(ATB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                         cudaGetErrorString(e));
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
    const int want = std::max(2 * NA_SEG_CAP_WORDS, NA_RESIDENT_MAX_WORDS) * 8;
    const int limit = optin - 1024;
    if (want > limit) return na_fail(ATB_ERR_ARG, "device shared memory too small");
    e = cudaFuncSetAttribute(atb_track_kernel_exact, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             limit);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(atb_track_kernel_fast,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
    g_na_ptr[device] = static_cast<unsigned char*>(p);
    *out = g_na_ptr[device];
    return ATB_OK;
}

}  // namespace

/* Flags a table element compiled for another integrator of the GPU call:
   this entry point runs the default tracking kernels, which have only the
   Forest-Ruth steps.  The host reads the flag before it launches the
   tracking, so such a call fails with the particles untouched. */
__global__ void atb_noalloc_scan(const double* __restrict__ table,
                                 const uint32_t* __restrict__ elem_off, int nelem,
                                 int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nelem) {
        const uint64_t h = reinterpret_cast<const uint64_t*>(table)[elem_off[i]];
        if ((h >> ATB_H_FL_SHIFT) & ATB_F_INTEG) atomicOr(status, ATB_STATUS_INTEGRATOR);
    }
}

extern "C" int atb_track_noalloc(int32_t device, const double* table, int64_t nwords,
                                 const uint32_t* elem_off_host, const uint32_t* elem_off,
                                 int32_t nelem, double* r, int64_t np, int32_t nturns,
                                 int32_t turn0, int32_t losses, uint8_t* islost, uint32_t* lturn,
                                 uint32_t* lelem, double* lcoord, int32_t mode, void* stream) {
    if (device < 0 || device >= kMaxDevices) return na_fail(ATB_ERR_ARG, "invalid device id");
    if (nelem < 0 || nwords < 0 || np < 0 || nturns < 0) return na_fail(ATB_ERR_ARG, "negative size");
    if (mode != ATB_MODE_EXACT && mode != ATB_MODE_FAST) return na_fail(ATB_ERR_ARG, "bad mode");
    if (nelem > 0 && (!table || !elem_off || !elem_off_host))
        return na_fail(ATB_ERR_ARG, "lattice table pointers missing");
    if (np > 0 && !r) return na_fail(ATB_ERR_ARG, "r is NULL");
    if (losses && np > 0 && (!islost || !lturn || !lelem || !lcoord))
        return na_fail(ATB_ERR_ARG, "loss map buffers missing");
    if (nelem > 0 && (elem_off_host[0] != 0 || (int64_t)elem_off_host[nelem] != nwords))
        return na_fail(ATB_ERR_ARG, "element offsets do not span the table");
    /* the table is staged by 16-byte bulk copies and the particles and loss
       coordinates are moved in 16-byte vectors: the caller's buffers (which
       may come from its own sub-allocator) must allow that */
    if ((nwords & 1) != 0)
        return na_fail(ATB_ERR_ARG, "atb_track_noalloc: the table must hold an even number of "
                                    "words (whole 16-byte records)");
    if ((reinterpret_cast<uintptr_t>(table) | reinterpret_cast<uintptr_t>(r)) & 15u)
        return na_fail(ATB_ERR_ARG, "atb_track_noalloc: table and r must be 16-byte aligned");
    if (losses && ((reinterpret_cast<uintptr_t>(lcoord) & 15u) ||
                   ((reinterpret_cast<uintptr_t>(lturn) | reinterpret_cast<uintptr_t>(lelem)) & 3u)))
        return na_fail(ATB_ERR_ARG, "atb_track_noalloc: lcoord must be 16-byte and lturn/lelem "
                                    "4-byte aligned");
    if (nelem > 0 && (reinterpret_cast<uintptr_t>(elem_off) & 3u))
        return na_fail(ATB_ERR_ARG, "atb_track_noalloc: elem_off must be 4-byte aligned");
    for (int32_t i = 0; i < nelem; ++i)
        if ((elem_off_host[i] & 1u) || elem_off_host[i + 1] < elem_off_host[i])
            return na_fail(ATB_ERR_ARG, "atb_track_noalloc: element records must start on even "
                                        "words (16-byte boundaries), in increasing order");
    const int64_t ntiles64 = (np + NA_THREADS - 1) / NA_THREADS;
    if (ntiles64 > ATB_NOALLOC_MAX_TILES)
        return na_fail(ATB_ERR_ARG, "atb_track_noalloc: " + std::to_string(np) +
                                        " particles exceed the maximum of " +
                                        std::to_string((int64_t)ATB_NOALLOC_MAX_TILES * NA_THREADS));
    if (np == 0 || nturns == 0) return ATB_OK;

    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) cudaSetDevice(device);
    struct Restore {
        int d;
        ~Restore() { if (d >= 0) cudaSetDevice(d); }
    } restore{prev != device ? prev : -1};

    unsigned char* base = nullptr;
    int rc = na_setup(device, &base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;

    /* segment plan (host stack only) */
    AtbSeg segs[ATB_NOALLOC_MAX_SEGS];
    int nseg = 0;
    const bool resident = nelem > 0 && nwords <= NA_RESIDENT_MAX_WORDS;
    if (resident) {
        segs[0].first_elem = 0;
        segs[0].nelem = nelem;
        segs[0].word0 = 0;
        segs[0].nwords = (int32_t)nwords;
        segs[0].pad = 0;
        nseg = 1;
    } else {
        int i = 0;
        while (i < nelem) {
            int j = i;
            while (j < nelem && (int64_t)(elem_off_host[j + 1] - elem_off_host[i]) <= NA_SEG_CAP_WORDS) ++j;
            if (j == i) return na_fail(ATB_ERR_ARG, "element record longer than a segment");
            if (nseg >= ATB_NOALLOC_MAX_SEGS)
                return na_fail(ATB_ERR_ARG, "atb_track_noalloc: lattice needs more than " +
                                                std::to_string(ATB_NOALLOC_MAX_SEGS) + " segments");
            int nw = (int)(elem_off_host[j] - elem_off_host[i]);
            segs[nseg].first_elem = i;
            segs[nseg].nelem = j - i;
            segs[nseg].word0 = elem_off_host[i];
            segs[nseg].nwords = nw;
            segs[nseg].pad = 0;
            ++nseg;
            i = j;
        }
    }

    AtbJob J;
    std::memset(&J, 0, sizeof(J));
    J.table = table;
    J.segs = reinterpret_cast<const AtbSeg*>(base + NA_SEGS);
    J.elem_off = elem_off;
    J.nelem = nelem;
    J.resident = resident ? 1 : 0;
    J.start_elem = 0;
    J.end_elem = nelem;
    J.seg_first0 = 0;
    J.nseg_first = nseg;
    J.nseg_turn = nseg;
    if (resident) { J.nseg_first = 1; J.nseg_turn = 1; }
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

    /* the array keeps the previous call's contents: rewrite the lists and
       clear the counter and the status word */
    cudaError_t e = cudaMemcpyAsync(base + NA_JOB, &J, sizeof(J), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nseg)
        e = cudaMemcpyAsync(base + NA_SEGS, segs, nseg * sizeof(AtbSeg), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + NA_COUNTER, 0, 8, st);
    if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
    const int ntiles = (int)ntiles64;
    AtbTile* tiles = reinterpret_cast<AtbTile*>(base + NA_TILES);
    atb_noalloc_tiles<<<(ntiles + 255) / 256, 256, 0, st>>>(tiles, ntiles, np, NA_THREADS);
    int* status = reinterpret_cast<int*>(base + NA_STATUS);
    if (nelem > 0) {
        /* refuse a table for another integrator before anything is tracked */
        atb_noalloc_scan<<<(nelem + 255) / 256, 256, 0, st>>>(table, elem_off, nelem, status);
        int s0 = 0;
        e = cudaMemcpyAsync(&s0, status, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
        if (s0 & ATB_STATUS_INTEGRATOR)
            return na_fail(ATB_ERR_ARG, "atb_track_noalloc: the table uses another integrator "
                                        "than the default (4); use atb_track");
    }

    const int smem = resident ? segs[0].nwords * 8 : 2 * NA_SEG_CAP_WORDS * 8;
    const void* fn = mode == ATB_MODE_EXACT ? (const void*)atb_track_kernel_exact
                                            : (const void*)atb_track_kernel_fast;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NA_THREADS, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess || per_sm < 1) return na_fail(ATB_ERR_CUDA, "launch configuration failed");
    const int grid = std::min(ntiles, per_sm * sms);
    const AtbJob* dj = reinterpret_cast<const AtbJob*>(base + NA_JOB);
    int* counter = reinterpret_cast<int*>(base + NA_COUNTER);
    if (mode == ATB_MODE_EXACT)
        atb_track_kernel_exact<<<grid, NA_THREADS, smem, st>>>(dj, tiles, ntiles, counter,
                                                               nullptr, status,
                                                               NA_SEG_CAP_WORDS, nullptr);
    else
        atb_track_kernel_fast<<<grid, NA_THREADS, smem, st>>>(dj, tiles, ntiles, counter,
                                                              nullptr, status,
                                                              NA_SEG_CAP_WORDS, nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
    /* wait, then read the kernel's status word into a host variable */
    int s = 0;
    e = cudaMemcpyAsync(&s, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(ATB_ERR_CUDA, cudaGetErrorString(e));
    if (s & ATB_STATUS_WAIT_TIMEOUT)
        return na_fail(ATB_ERR_TIMEOUT, "a bounded shared-memory staging wait timed out");
    return ATB_OK;
}
