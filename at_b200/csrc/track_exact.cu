/* Tracking kernel, "exact" arithmetic: the reference's expression order with
 * FMA contraction disabled (this file is compiled with -fmad=false). */
#define ATB_FAST 0
#include "track_kernel.cuh"
