// FP64 DFMA throughput microbenchmark: the denominator of the FP64-pipe
// roofline (measured peak figures for these GPUs cover HBM copy and BF16
// GEMM only).
// Every thread runs 8 independent FMA chains for `iters` rounds; the grid
// is 16 blocks of 256 threads per SM. FLOPs = 2 per FMA.
#include <cuda_runtime.h>

#include "../../include/pippin_b200_tools.h"

namespace {

__global__ void __launch_bounds__(256) dfma_kernel(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int pg_fp64_peak(int device, int iters, double* tflops, double* ms_out) {
  if (!tflops || iters < 1) return 1;
  if (cudaSetDevice(device) != cudaSuccess) return 3;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return 3;
  int blocks = p.multiProcessorCount * 16, threads = 256;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return 3;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dfma_kernel<<<blocks, threads>>>(out, iters / 4 + 1, 0.999999, 1e-7);  // warm-up and clocks up
  cudaEventRecord(e0);
  dfma_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return 3;
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  if (ms_out) *ms_out = ms;
  return 0;
}
