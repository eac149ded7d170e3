/* Tangent kernel unit (and the element-map kernel of the Ohmi envelope):
 * forward-mode derivatives of multi-turn tracking, in
 * the "exact" arithmetic (compiled with -fmad=false like track_exact.cu, so
 * the tracked values equal those of the exact tracking kernel). */
#define ATB_FAST 0
#define ATB_NO_TRACK_KERNEL
#include "atb_diffusion.cuh"
