// Device-side helpers: mbarriers, TMA tile loads, bounded waits and the
// grid barrier of the cooperative kernels. Every wait here gives up after a
// bounded number of polls, sets the context's timeout flag and lets the
// kernel return, so that a broken invariant cannot hang the GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hb {

// Polls before a wait gives up (a poll is tens of ns: far above any real
// wait, far below a watchdog).
constexpr uint32_t kMaxPolls = 1u << 26;

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte asynchronous copy global -> shared (L2 only); bytes < 16 (0
// included) reads that many and zero-fills the rest.
__device__ __forceinline__ void CpAsync16(void* dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
               :
               : "r"(SmemAddr(dst)), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)),
               "r"(count));
}
__device__ __forceinline__ void FenceBarrierInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* bar,
                                                   uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          SmemAddr(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ void MbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar))
               : "memory");
}
__device__ __forceinline__ bool MbarTryWait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(SmemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of `bar`; false (and the timeout flag set) if it
// did not complete within kMaxPolls polls.
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity,
                                         int* timeout_flag) {
  for (uint32_t i = 0; i < kMaxPolls; ++i) {
    if (MbarTryWait(bar, parity)) return true;
  }
  if (timeout_flag) atomicExch(timeout_flag, 1);
  return false;
}

// 2-D TMA tile load into shared memory, completing on `bar`. c0 is the
// innermost coordinate.
__device__ __forceinline__ void TmaLoad2d(void* dst, const CUtensorMap* map,
                                          int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(SmemAddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1),
      "r"(SmemAddr(bar))
      : "memory");
}
__device__ __forceinline__ void PrefetchTmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

// tcgen05 (5th-generation tensor core) helpers.
//
// Shared-memory matrix descriptor of a K-major, swizzled operand tile whose
// rows are kb_bytes long (128, 64 or 32): leading byte offset 16 B (unused
// with swizzling), stride byte offset = 8 rows, descriptor version 1.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t addr, int kb_bytes) {
  const uint64_t layout = kb_bytes == 128 ? 2 : (kb_bytes == 64 ? 4 : 6);
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (1ull << 16) |
         (static_cast<uint64_t>((8 * kb_bytes) >> 4) << 32) | (1ull << 46) |
         (layout << 61);
}

__device__ __forceinline__ void MmaI8(uint32_t d_tmem, uint64_t a_desc,
                                      uint64_t b_desc, uint32_t idesc,
                                      uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void MmaCommit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
      ::"r"(SmemAddr(bar))
      : "memory");
}


// Grid barrier for cooperative launches: `counter` is zeroed before the
// launch; barrier number `gen` (1, 2, ...) completes when all `nblocks`
// blocks have arrived `gen` times. Bounded; false on timeout.
__device__ __forceinline__ bool GridBarrier(unsigned int* counter,
                                            unsigned int nblocks,
                                            unsigned int gen,
                                            int* timeout_flag) {
  __syncthreads();
  bool ok = true;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    const unsigned int target = nblocks * gen;
    uint32_t i = 0;
    while (true) {
      unsigned int v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                   : "=r"(v)
                   : "l"(counter)
                   : "memory");
      if (v >= target) break;
      if (++i >= kMaxPolls) {
        atomicExch(timeout_flag, 1);
        ok = false;
        break;
      }
    }
    __threadfence();
  }
  // Broadcast the outcome through shared memory.
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
  __syncthreads();
  return s_ok != 0;
}

}  // namespace hb
