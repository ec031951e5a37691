/*
 * fem_probe.h -- arithmetic-peak probes of the current GPU (libfemprobe.so).
 *
 * Calibration for the benchmark's roofline notes, kept out of the assembly
 * library (libfemb200.so, fem_b200.h).  No reference counterpart.
 */
#ifndef FEM_PROBE_H
#define FEM_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Measured arithmetic peak of the current device in TFLOP/s: kind 0 = FP64 FMA
 * pipe, 1 = FP32 FMA pipe, 2 = FP64 tensor-core MMA (m8n8k4), 3 = BF16
 * tensor-core MMA (m16n8k16, FP32 accumulate).  Allocates a scratch buffer and
 * synchronises the device.  Returns 0, -1 for bad arguments, or a cudaError_t. */
int fem_probe_peak(int kind, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* FEM_PROBE_H */
