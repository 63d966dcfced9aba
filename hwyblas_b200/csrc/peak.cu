// Issue-rate probe of the FP64 tensor pipe: a loop of independent DMMA
// (mma.sync.m16n8k8.f64) chains on every SM, timed with CUDA events. Its
// result is the FP64 roofline denominator that bench.py reports beside the
// GEMM's achieved FP64 TFLOP/s (no measured FP64 peak is provided otherwise).
#include <cuda_runtime.h>

#include "../../include/hwyblas_b200.h"
#include "internal.h"

namespace hb {
namespace {

__global__ void __launch_bounds__(256) DmmaPeakKernel(double* sink, int iters) {
  double acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  const double a0 = threadIdx.x * 1e-3, a1 = a0 + 1.0, a2 = a0 + 2.0,
               a3 = a0 + 3.0, b0 = 0.5, b1 = 0.25;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
          "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
          : "+d"(acc[i][0]), "+d"(acc[i][1]), "+d"(acc[i][2]), "+d"(acc[i][3])
          : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
    }
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) s += acc[i][j];
  if (s == 1234.5) sink[0] = s;  // keeps the loop alive
}

}  // namespace
}  // namespace hb

extern "C" {

// Measures the FP64 tensor-pipe throughput of the current device in
// TFLOP/s (best of three launches). No counterpart in the reference.
HWYBLAS_API double hwyblas_fp64_peak_tflops(void) {
  hb::Context& ctx = hb::Ctx();
  double* sink = static_cast<double*>(hb::Workspace(hb::kWsBatch, 64));
  const int blocks = ctx.num_sms * 2, threads = 256, iters = 8192;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  hb::DmmaPeakKernel<<<blocks, threads, 0, ctx.stream>>>(sink, 64);
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(e0, ctx.stream);
    hb::DmmaPeakKernel<<<blocks, threads, 0, ctx.stream>>>(sink, iters);
    cudaEventRecord(e1, ctx.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  hb::CountLaunch(4);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (hb::LaunchFailed("fp64 peak probe")) return 0.0;
  const double flops = 2.0 * 16 * 8 * 8 * 8.0 * iters * (threads / 32) * blocks;
  return flops / (best * 1e-3) / 1e12;
}

}  // extern "C"
