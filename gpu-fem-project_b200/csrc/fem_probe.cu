// Arithmetic-peak probes (libfemprobe.so, include/fem_probe.h): calibration for
// the benchmark's roofline notes, built as a library of its own so that it is not
// part of the assembly library's interface.  Dependent-chain-free FMA streams on
// the FP64 and FP32 pipes, the FP64 tensor-core MMA (m8n8k4) of the FP64 stiffness
// stage and the BF16 MMA (m16n8k16, FP32 accumulate) of the BF16x6 stiffness
// stage.  Each thread runs 8 independent accumulator chains; the result is written
// so nothing is elided.
#include <cuda_runtime.h>

#include "fem_probe.h"

namespace fem {
namespace dev {

template <typename T>
__global__ void __launch_bounds__(256) fma_probe(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int j = 0; j < 8; j++) x[j] = T(threadIdx.x + j);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = fma(x[j], a, b);
  }
  T s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += x[j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) dmma_probe(double *out, int iters, double a, double b) {
  double c[8][2];
#pragma unroll
  for (int j = 0; j < 8; j++) c[j][0] = c[j][1] = double(threadIdx.x + j);
  const double av = a + threadIdx.x, bv = b - threadIdx.x;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[j][0]), "+d"(c[j][1])
                   : "d"(av), "d"(bv));
  }
  double s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += c[j][0] + c[j][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) bmma_probe(float *out, int iters, unsigned a, unsigned b) {
  float c[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) c[j][0] = c[j][1] = c[j][2] = c[j][3] = float(threadIdx.x + j);
  const unsigned av = a ^ threadIdx.x, bv = b ^ threadIdx.x;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++)
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%4,%4,%4}, {%5,%5}, {%0,%1,%2,%3};"
          : "+f"(c[j][0]), "+f"(c[j][1]), "+f"(c[j][2]), "+f"(c[j][3])
          : "r"(av), "r"(bv));
  }
  float s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace dev
}  // namespace fem

extern "C" {

// kind 0: FP64 FMA, 1: FP32 FMA, 2: FP64 MMA m8n8k4, 3: BF16 MMA m16n8k16 (FP32
// accumulate).  Returns TFLOP/s (2 flops per FMA).
int fem_probe_peak(int kind, double *tflops) {
  if (!tflops || kind < 0 || kind > 3) return -1;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = sms * 8, block = 256, iters = 4096;
  void *buf = nullptr;
  cudaError_t err = cudaMalloc(&buf, sizeof(double) * grid * block);
  if (err != cudaSuccess) return (int)err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    if (kind == 0)
      fem::dev::fma_probe<double><<<grid, block>>>((double *)buf, iters, 0.999999, 1e-7);
    else if (kind == 1)
      fem::dev::fma_probe<float><<<grid, block>>>((float *)buf, iters, 0.999999f, 1e-7f);
    else if (kind == 2)
      fem::dev::dmma_probe<<<grid, block>>>((double *)buf, iters, 1e-3, 1e-3);
    else
      fem::dev::bmma_probe<<<grid, block>>>((float *)buf, iters, 0x3c003c00u, 0x3c003c00u);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (err != cudaSuccess) return (int)err;
  const double threads = double(grid) * block;
  double flops;
  if (kind == 2)
    flops = threads / 32.0 * iters * 8 * (8 * 8 * 4) * 2.0;  // per warp: 8 MMAs of 256 FMAs
  else if (kind == 3)
    flops = threads / 32.0 * iters * 8 * (16 * 8 * 16) * 2.0;  // per warp: 8 MMAs of 2048 FMAs
  else
    flops = threads * iters * 8 * 2.0;
  *tflops = flops / (best * 1e-3) / 1e12;
  return 0;
}

}  // extern "C"
