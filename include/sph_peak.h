/*
 * sph_peak.h — FFMA / DFMA throughput probe (libsph_peak.so).
 *
 * The SPH pair loops run on the non-tensor FP32 (or FP64) pipe, whose peak
 * the tensor-core and copy figures of the pool do not give.  This library
 * measures it on the current device with long chains of independent fused
 * multiply-adds; bench.py divides the pair kernels' algorithmic FLOP rate by
 * it.  It has no counterpart in the reference, which has no GPU code.
 */
#ifndef SPH_PEAK_H
#define SPH_PEAK_H
#ifdef __cplusplus
extern "C" {
#endif
/* Returns achieved FLOP/s (2 per FMA) of `reps` timed launches; precision 0 =
 * FP32, 1 = FP64.  Returns a negative value on a CUDA error. */
double sph_peak_flops(int precision, int reps);
#ifdef __cplusplus
}
#endif
#endif
