// peak.cu -- FP64 throughput probe used as the roofline denominator of the
// FP64 sweep (the pool's measured peaks cover HBM and BF16 only).
//
// Every warp of a full-occupancy grid runs long chains of independent FP64
// tensor-core products (mma.sync m8n8k4 f64) or FP64 FMAs on registers; the
// host times the launch with CUDA events and converts to TFLOP/s
// (2 flops per multiply-add).
#include <cuda_runtime.h>

#include "internal.h"

namespace msb {

constexpr int kPeakIters = 4096;

__global__ void __launch_bounds__(256) peak_dmma_kernel(double* out, double seed) {
  double acc[8][2];
  const double a = seed + threadIdx.x * 1e-9, b = seed - threadIdx.x * 1e-9;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c][0] = acc[c][1] = 0.0;
  for (int it = 0; it < kPeakIters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(acc[c][0]), "+d"(acc[c][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += acc[c][0] + acc[c][1];
  if (s == 12345.678) out[0] = s;  // keep the work alive
}

__global__ void __launch_bounds__(256) peak_dfma_kernel(double* out, double seed) {
  double acc[16];
  const double a = seed + threadIdx.x * 1e-9, b = seed - threadIdx.x * 1e-9;
#pragma unroll
  for (int c = 0; c < 16; ++c) acc[c] = c;
  for (int it = 0; it < kPeakIters; ++it) {
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c] = __fma_rn(a, acc[c], b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) s += acc[c];
  if (s == 12345.678) out[0] = s;
}

}  // namespace msb

// Measured FP64 peaks (TFLOP/s) of this GPU: tensor-core (mma.sync f64) and
// FMA pipe.  Each is the best of `reps` timed launches after one warm-up.
extern "C" int msb_measure_fp64_peak(double* tflops_dmma, double* tflops_dfma, int reps) {
  int dev = 0, nsm = 0, rc;
  if ((rc = msb::cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if ((rc = msb::cuda_check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count"))) return rc;
  double* out = nullptr;
  if ((rc = msb::cuda_check(cudaMalloc(&out, sizeof(double)), "cudaMalloc"))) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = nsm * 8, block = 256;
  const double warps = (double)grid * block / 32.0;
  float best[2] = {1e30f, 1e30f};
  for (int k = 0; k < 2; ++k) {
    for (int r = 0; r <= reps; ++r) {
      cudaEventRecord(e0);
      if (k == 0) msb::peak_dmma_kernel<<<grid, block>>>(out, 1.0);
      else msb::peak_dfma_kernel<<<grid, block>>>(out, 1.0);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0 && ms < best[k]) best[k] = ms;
    }
  }
  rc = msb::cuda_check(cudaGetLastError(), "peak kernels");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc) return rc;
  // dmma: 8 chains x 256 multiply-adds per warp per iteration
  const double fl_dmma = warps * msb::kPeakIters * 8 * 256 * 2.0;
  // dfma: 16 chains x 32 lanes per warp per iteration
  const double fl_dfma = warps * msb::kPeakIters * 16 * 32 * 2.0;
  if (tflops_dmma) *tflops_dmma = fl_dmma / (best[0] * 1e-3) / 1e12;
  if (tflops_dfma) *tflops_dfma = fl_dfma / (best[1] * 1e-3) / 1e12;
  return MSB_OK;
}
