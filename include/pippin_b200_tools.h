/* pippin_b200 measurement helpers (no counterpart in the reference). */
#ifndef PIPPIN_B200_TOOLS_H
#define PIPPIN_B200_TOOLS_H

#ifdef __cplusplus
extern "C" {
#endif

/* FP64 FMA throughput of `device` in TFLOP/s (2 FLOPs per FMA), timed with
 * CUDA events over one launch of `iters` rounds of 8 x 16 dependent FMAs per
 * thread; the denominator of the FP64-pipe roofline. ms_out may be NULL.
 * Returns 0 on success. */
int pg_fp64_peak(int device, int iters, double* tflops, double* ms_out);

#ifdef __cplusplus
}
#endif

#endif
