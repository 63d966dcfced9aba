// Issue-rate probes of the tensor pipes, timed with CUDA events: the FP64
// pipe (a loop of independent DMMA mma.sync.m16n8k8.f64 chains on every SM)
// and the INT8 pipe of the 5th-generation tensor cores (tcgen05.mma
// kind::i8 from shared memory into tensor memory, one CTA per SM). Their
// results are the roofline denominators that bench.py reports beside the
// GEMMs' achieved FP64 TFLOP/s and INT8 TOPS.
#include <cuda_runtime.h>

#include "../../include/hwyblas_b200.h"
#include "device.cuh"
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

// INT8 probe: one CTA per SM issues `iters` rounds of 4 MMAs (K = 32 bytes
// each, one 128-byte swizzled k block) of M = 128 and N = kN into alternating
// accumulators; the operands are zero tiles in shared memory (the rate does
// not depend on the values). The MMA completion is awaited through an
// mbarrier with a bounded wait before tensor memory is freed.
constexpr int kProbeSmem = 120 * 1024;  // > half the SM's shared memory: 1 CTA/SM

template <int kN>
__global__ void __launch_bounds__(64, 1) I8PeakKernel(int iters, int* timeout_flag) {
  extern __shared__ uint8_t probe_raw[];
  uint8_t* smem = probe_raw + ((1024 - (SmemAddr(probe_raw) & 1023)) & 1023);
  uint8_t* a_tile = smem;                 // 128 x 128 bytes
  uint8_t* b_tile = smem + 128 * 128;     // kN x 128 bytes
  uint64_t* done = reinterpret_cast<uint64_t*>(b_tile + kN * 128);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  for (int i = threadIdx.x; i < (128 + kN) * 128 / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  const int warp = threadIdx.x / 32;
  if (threadIdx.x == 0) {
    MbarInit(done, 1);
    FenceBarrierInit();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(SmemAddr(tmem_slot)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr int kAcc = 512 / kN;  // accumulators that fit tensor memory
  if (threadIdx.x == 0) {
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) |
                           (static_cast<uint32_t>(kN >> 3) << 17) |
                           (static_cast<uint32_t>(128 >> 4) << 24);
    const uint32_t sa = SmemAddr(a_tile), sb = SmemAddr(b_tile);
    for (int it = 0; it < iters; ++it) {
      const uint32_t d = tmem + (it % kAcc) * kN;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        MmaI8(d, SmemDesc(sa + kk * 32, 128), SmemDesc(sb + kk * 32, 128),
              idesc, (it >= kAcc || kk > 0) ? 1u : 0u);
    }
    MmaCommit(done);
  }
  __syncwarp();
  MbarWait(done, 0, timeout_flag);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 ::"r"(tmem), "r"(512));
  }
}

template <int kN>
double I8PeakTops() {
  Context& ctx = Ctx();
  auto* kernel = I8PeakKernel<kN>;
  static bool configured = false;
  if (!configured) {
    if (Failed(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kProbeSmem),
               "int8 peak probe smem"))
      return 0.0;
    configured = true;
  }
  const int iters = 20000;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  kernel<<<ctx.num_sms, 64, kProbeSmem, ctx.stream>>>(64, ctx.dev_status);
  float best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(e0, ctx.stream);
    kernel<<<ctx.num_sms, 64, kProbeSmem, ctx.stream>>>(iters, ctx.dev_status);
    cudaEventRecord(e1, ctx.stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  CountLaunch(4);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (LaunchFailed("int8 peak probe") || CheckDeviceStatus("int8 peak probe")) return 0.0;
  const double ops = 2.0 * 128 * kN * 32 * 4.0 * iters * ctx.num_sms;
  return ops / (best * 1e-3) / 1e12;
}

}  // namespace
}  // namespace hb

extern "C" {

// Measures the INT8 tensor-core throughput of the current device in TOPS:
// the better of N = 128 (the emulated GEMM's tile) and N = 256. No
// counterpart in the reference.
HWYBLAS_API double hwyblas_int8_peak_tops(void) {
  const double a = hb::I8PeakTops<128>();
  const double b = hb::I8PeakTops<256>();
  return a > b ? a : b;
}


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
