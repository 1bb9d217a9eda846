/*
 * Measurement helpers of ausaxs_b200 (no counterpart in the reference, which has no GPU code).
 * They feed the roofline that bench.py reports for the pair kernel; the product path does not
 * call them.  Return codes as include/ausaxs_b200.h.
 */
#ifndef AUSAXS_B200_DIAG_H
#define AUSAXS_B200_DIAG_H
#include "ausaxs_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Shared-memory 32-bit atomicAdd throughput of one device: every SM full of 512-thread CTAs, each
 * adding 1 to words of a 4,096-word shared array.  conflict_free bit 0 set: the 32 lanes of a warp on
 * 32 distinct banks (the throughput bound); clear: bins uniformly random over the array.  Bit 1 set:
 * 64-bit atomicAdd on 2,048 words of the same 16 KB instead.  Returns atomics per second over the
 * whole device and the kernel's milliseconds (ms may be null).
 */
AUSAXS_API int ausaxs_gpu_smem_atomic_rate(int32_t device, int32_t conflict_free, double* atomics_per_s, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* AUSAXS_B200_DIAG_H */
