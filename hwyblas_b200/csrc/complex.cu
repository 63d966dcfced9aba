// Complex GEMM (zgemm_, cgemm_), bit-identical to the reference's complex
// micro-kernel (src/gemm_kernel-inl.h:226-428) in its blocked driver
// (src/gemm-inl.h:152-232).
//
// Complex numbers are interleaved (re, im). For every element of C the
// reference accumulates four real FMA chains over each KC = 256 chunk of k:
//
//   rr = sum ar*br, ir = sum ai*br   (acc_re += a * re(b))
//   ri = sum ar*bi, ii = sum ai*bi   (acc_im += a * im(b))
//
// then forms ab = (rr - ii, ir + ri), r = alpha * ab as
// (ab.re*al.re - ab.im*al.im, ab.im*al.re + ab.re*al.im) with every product
// and sum rounded, and merges r into C: r (beta 0), r + C (beta 1, and every
// chunk after the first), or r + beta*C with beta*C formed the same way.
// op(A) and op(B) with 'C' are conjugated while loaded (the reference's
// packing), which negates imaginary parts exactly.
//
// The chains are independent per element, so a SIMT kernel computes them
// directly: 64 x 64 complex tiles per 256-thread CTA, 4 x 4 elements per
// thread, k in double-buffered shared-memory slices of 16.
#include <algorithm>
#include <cstdint>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

template <typename R>
__device__ __forceinline__ R Mul(R x, R y) {
  if constexpr (sizeof(R) == 8) return __dmul_rn(x, y);
  else return __fmul_rn(x, y);
}
template <typename R>
__device__ __forceinline__ R Add(R x, R y) {
  if constexpr (sizeof(R) == 8) return __dadd_rn(x, y);
  else return __fadd_rn(x, y);
}
template <typename R>
__device__ __forceinline__ R Sub(R x, R y) {
  if constexpr (sizeof(R) == 8) return __dsub_rn(x, y);
  else return __fsub_rn(x, y);
}
template <typename R>
__device__ __forceinline__ R Fma(R x, R y, R z) {
  if constexpr (sizeof(R) == 8) return fma(x, y, z);
  else return fmaf(x, y, z);
}

constexpr int kZM = 64, kZN = 64, kZK = 16, kZChunk = 256;

// A complex operand: element (i, p) has its real part at
// data[2 * (i * rs + p * cs)]; conj negates the imaginary part.
template <typename R>
struct ZView {
  const R* data;
  long long rs, cs;
  int conj;
};

template <typename R>
struct ZParams {
  int m, n, k;
  R alpha_re, alpha_im, beta_re, beta_im;
  ZView<R> a, b;
  R* c;
  long long ldc;  // complex elements
  const int* guard;
};

template <typename R>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// Asynchronous copy of one complex element (src_bytes 0: zero fill).
template <typename R>
__device__ __forceinline__ void CpAsyncElem(void* smem_dst, const R* src, bool valid) {
  const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  if constexpr (sizeof(R) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
  }
}

// One CTA: a 64 x 64 complex tile, 4 x 4 elements per thread (rows
// tx + 16 r, columns ty + 16 q). The k-slices of 16 stream through two
// shared-memory buffers with cp.async (complex elements stay interleaved, so
// one shared load gives both parts; conjugation is applied after the load),
// the next slice in flight while this one is multiplied. A chunk ends on a
// slice boundary (256 is a multiple of 16), where the thread merges its
// chunk into C in memory: the running value stays in C itself.
template <typename R>
__global__ void __launch_bounds__(256, 1) ZgemmKernel(ZParams<R> p) {
  if (p.guard != nullptr && *p.guard != 0) return;
  using V = typename Vec2<R>::type;
  extern __shared__ __align__(16) unsigned char zsmem[];
  V* sa = reinterpret_cast<V*>(zsmem);                 // [2][kZK][kZM]
  V* sb = sa + 2 * kZK * kZM;                          // [2][kZK][kZN]
  const int m0 = blockIdx.x * kZM, n0 = blockIdx.y * kZN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  R rr[4][4], ir[4][4], ri[4][4], ii[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) rr[r][q] = ir[r][q] = ri[r][q] = ii[r][q] = R(0);
  const bool beta_zero = (p.beta_re == R(0) && p.beta_im == R(0));
  const bool beta_one = (p.beta_re == R(1) && p.beta_im == R(0));
  // Consecutive threads copy consecutive addresses: along rows of op(A) when
  // A is not transposed, else along k; along k of op(B) when B is not
  // transposed, else along its columns.
  const bool a_rows = p.a.rs == 1, b_k = p.b.rs == 1;
  const auto issue = [&](int k0, int buf) {
    V* da = sa + buf * kZK * kZM;
    V* db = sb + buf * kZK * kZN;
    for (int idx = threadIdx.x; idx < kZK * kZM; idx += 256) {
      const int kk = a_rows ? idx / kZM : idx % kZK, mm = a_rows ? idx % kZM : idx / kZK;
      const int gi = m0 + mm, gk = k0 + kk;
      const bool ok = gi < p.m && gk < p.k;
      const R* src = ok ? p.a.data + 2 * (gi * p.a.rs + gk * p.a.cs) : p.a.data;
      CpAsyncElem<R>(da + kk * kZM + mm, src, ok);
    }
    for (int idx = threadIdx.x; idx < kZK * kZN; idx += 256) {
      const int kk = b_k ? idx % kZK : idx / kZN, nn = b_k ? idx / kZK : idx % kZN;
      const int gj = n0 + nn, gk = k0 + kk;
      const bool ok = gj < p.n && gk < p.k;
      const R* src = ok ? p.b.data + 2 * (gk * p.b.rs + gj * p.b.cs) : p.b.data;
      CpAsyncElem<R>(db + kk * kZN + nn, src, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const R sa_sign = p.a.conj ? R(-1) : R(1), sb_sign = p.b.conj ? R(-1) : R(1);
  issue(0, 0);
  int buf = 0;
  for (int k0 = 0; k0 < p.k; k0 += kZK, buf ^= 1) {
    if (k0 + kZK < p.k) {
      issue(k0 + kZK, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const V* ca = sa + buf * kZK * kZM;
    const V* cb = sb + buf * kZK * kZN;
    const int kend = min(kZK, p.k - k0);
#pragma unroll 2
    for (int kk = 0; kk < kend; ++kk) {
      R ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const V va = ca[kk * kZM + tx + 16 * r];
        const V vb = cb[kk * kZN + ty + 16 * r];
        ar[r] = va.x;
        ai[r] = Mul(va.y, sa_sign);
        br[r] = vb.x;
        bi[r] = Mul(vb.y, sb_sign);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          rr[r][q] = Fma(ar[r], br[q], rr[r][q]);
          ir[r][q] = Fma(ai[r], br[q], ir[r][q]);
          ri[r][q] = Fma(ar[r], bi[q], ri[r][q]);
          ii[r][q] = Fma(ai[r], bi[q], ii[r][q]);
        }
    }
    __syncthreads();
    if ((k0 + kZK) % kZChunk == 0 || k0 + kZK >= p.k) {
      const bool first = k0 < kZChunk;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = m0 + tx + 16 * r, j = n0 + ty + 16 * q;
          const R ab_re = Sub(rr[r][q], ii[r][q]);
          const R ab_im = Add(ir[r][q], ri[r][q]);
          rr[r][q] = ir[r][q] = ri[r][q] = ii[r][q] = R(0);
          if (i >= p.m || j >= p.n) continue;
          const R t_re = Sub(Mul(ab_re, p.alpha_re), Mul(ab_im, p.alpha_im));
          const R t_im = Add(Mul(ab_im, p.alpha_re), Mul(ab_re, p.alpha_im));
          R* ce = p.c + 2 * (i + j * p.ldc);
          if (first && beta_zero) {
            ce[0] = t_re;
            ce[1] = t_im;
          } else if (!first || beta_one) {
            ce[0] = Add(t_re, ce[0]);
            ce[1] = Add(t_im, ce[1]);
          } else {
            const R c0 = ce[0], c1 = ce[1];
            const R b_re = Sub(Mul(c0, p.beta_re), Mul(c1, p.beta_im));
            const R b_im = Add(Mul(c1, p.beta_re), Mul(c0, p.beta_im));
            ce[0] = Add(t_re, b_re);
            ce[1] = Add(t_im, b_im);
          }
        }
    }
  }
}

template <typename R>
constexpr int ZSmemBytes() {
  return 2 * (kZK * kZM + kZK * kZN) * 2 * static_cast<int>(sizeof(R));
}

// C := beta * C (beta 0: zeros, C not read), each element as the complex
// product (c.re*b.re - c.im*b.im, c.re*b.im + c.im*b.re) (gemm.cc:48-64).
template <typename R>
__global__ void ZScaleKernel(int m, int n, R beta_re, R beta_im, R* c, long long ldc,
                             const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  const long long total = static_cast<long long>(m) * n;
  const bool zero = (beta_re == R(0) && beta_im == R(0));
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    R* ce = c + 2 * (i + j * ldc);
    if (zero) {
      ce[0] = R(0);
      ce[1] = R(0);
    } else {
      const R c0 = ce[0], c1 = ce[1];
      ce[0] = Sub(Mul(c0, beta_re), Mul(c1, beta_im));
      ce[1] = Add(Mul(c0, beta_im), Mul(c1, beta_re));
    }
  }
}

}  // namespace

// GEMM (src/gemm.cc:67-123) for complex data after argument checks: a, b, c
// interleaved, leading dimensions in complex elements; alpha, beta as
// (re, im).
template <typename R>
void ZgemmFull(int ta, int tb, int m, int n, int k, const R* alpha, const R* a, int lda,
               const R* b, int ldb, const R* beta, R* c, int ldc) {
  if (m == 0 || n == 0) return;
  const bool alpha_zero = (alpha[0] == R(0) && alpha[1] == R(0));
  const bool beta_one = (beta[0] == R(1) && beta[1] == R(0));
  if ((k == 0 || alpha_zero) && beta_one) return;
  if (k == 0 || alpha_zero) {
    const long long total = static_cast<long long>(m) * n;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 8));
    ZScaleKernel<R><<<blocks, 256, 0, Ctx().stream>>>(m, n, beta[0], beta[1], c, ldc,
                                                        Ctx().guard);
    CountLaunch();
    LaunchFailed("complex scale");
    return;
  }
  // cp.async copies whole complex elements, which must be aligned to their
  // size; an operand that is not is copied to an aligned buffer first.
  const auto aligned = [](const R* x, int rows, int cols, int ld, int slot, int* ld_out) {
    *ld_out = ld;
    if (reinterpret_cast<uintptr_t>(x) % (2 * sizeof(R)) == 0) return x;
    R* dst = static_cast<R*>(Workspace(slot, 2 * sizeof(R) * static_cast<size_t>(rows) * cols));
    if (dst == nullptr) return static_cast<const R*>(nullptr);
    if (Failed(cudaMemcpy2DAsync(dst, 2 * sizeof(R) * rows, x, 2 * sizeof(R) * ld,
                                 2 * sizeof(R) * rows, cols, cudaMemcpyDeviceToDevice,
                                 Ctx().stream),
               "complex operand copy"))
      return static_cast<const R*>(nullptr);
    *ld_out = rows;
    return static_cast<const R*>(dst);
  };
  int lda2, ldb2;
  a = aligned(a, ta == 0 ? m : k, ta == 0 ? k : m, lda, kWsPackA, &lda2);
  b = aligned(b, tb == 0 ? k : n, tb == 0 ? n : k, ldb, kWsPackB, &ldb2);
  if (a == nullptr || b == nullptr) return;
  lda = lda2;
  ldb = ldb2;
  ZParams<R> p;
  p.m = m;
  p.n = n;
  p.k = k;
  p.alpha_re = alpha[0];
  p.alpha_im = alpha[1];
  p.beta_re = beta[0];
  p.beta_im = beta[1];
  // op: 0 N, 1 T, 2 C. Element (i, p) of op(A): A(i, p) or A(p, i).
  p.a = ta == 0 ? ZView<R>{a, 1, lda, 0} : ZView<R>{a, lda, 1, ta == 2 ? 1 : 0};
  p.b = tb == 0 ? ZView<R>{b, 1, ldb, 0} : ZView<R>{b, ldb, 1, tb == 2 ? 1 : 0};
  p.c = c;
  p.ldc = ldc;
  p.guard = Ctx().guard;
  const dim3 grid((m + kZM - 1) / kZM, (n + kZN - 1) / kZN);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(ZgemmKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         ZSmemBytes<R>());
    configured = true;
  }
  ZgemmKernel<R><<<grid, 256, ZSmemBytes<R>(), Ctx().stream>>>(p);
  CountLaunch();
  LaunchFailed("complex gemm");
}
template void ZgemmFull<double>(int, int, int, int, int, const double*, const double*, int,
                                const double*, int, const double*, double*, int);
template void ZgemmFull<float>(int, int, int, int, int, const float*, const float*, int,
                               const float*, int, const float*, float*, int);

}  // namespace hb
