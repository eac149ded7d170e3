/* Adjoint kernel unit: reverse-mode derivatives of multi-turn tracking, in
 * the "exact" arithmetic (compiled with -fmad=false like track_exact.cu, so
 * the tracked values equal those of the exact tracking kernel; the
 * derivative arithmetic uses explicit fma()). */
#define ATB_FAST 0
#define ATB_NO_TRACK_KERNEL
#include "adjoint_kernel.cuh"
