/* Tracking kernel, "fast" arithmetic: FMA contraction and reciprocal reuse. */
#define ATB_FAST 1
#include "track_kernel.cuh"
