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
#include <cfloat>
#include <cstdint>
#include <cstdio>

#include <cooperative_groups.h>

#include "device.cuh"
#include "internal.h"
#include "ref_order.cuh"

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
  // HERK: only the triangle `part` of C (1 lower, 2 upper; 0 all) is
  // updated. Elements in micro-tiles of the reference (tmr x tnr, on its
  // grid) that cross the diagonal merge as its MergeTile does, with the
  // diagonal's imaginary part dropped when real_diag is set.
  int part, real_diag, tmr, tnr;
  // Split over KC chunks: CTA z computes chunk z alone and stores its
  // alpha * ab to partial[(z n + j) m + i] (interleaved); ZSplitMergeKernel
  // then merges the chunks in order.
  R* partial;
};

// Merges one chunk's t = alpha * ab into element (i, j) of C as the
// reference does (first: the first KC chunk, which applies beta; later chunks
// add with beta 1): r, r + C or r + beta C in the micro-kernel's rounding,
// or the MergeTile rule for HERK tiles crossing the diagonal. Elements
// outside the triangle of a HERK are left alone.
template <typename R>
__device__ __forceinline__ void ZMergeElement(const ZParams<R>& p, int i, int j, bool first,
                                              R t_re, R t_im) {
  R* ce = p.c + 2 * (i + j * p.ldc);
  if (p.part != 0) {
    if (p.part == 1 ? i < j : i > j) return;
    const int i0 = i / p.tmr * p.tmr, j0 = j / p.tnr * p.tnr;
    const int il = min(i0 + p.tmr, p.m) - 1, jl = min(j0 + p.tnr, p.n) - 1;
    if (!(p.part == 1 ? i0 > jl : il < j0)) {
      // Crossing tile (src/gemm-inl.h:110-130): v = alpha ab, then v += beta
      // * c as the C++ runtime's complex product and sum (beta 1 after the
      // first chunk); on the diagonal with real_diag, v and c lose their
      // imaginary parts first.
      const R br = first ? p.beta_re : R(1), bi = first ? p.beta_im : R(0);
      const bool bz = br == R(0) && bi == R(0);
      R vr = t_re, vi = t_im;
      if (p.real_diag && i == j) {
        vi = R(0);
        if (!bz) {
          const R c0 = ce[0];
          vr = Add(vr, Sub(Mul(br, c0), Mul(bi, R(0))));
          vi = Add(vi, Add(Mul(br, R(0)), Mul(bi, c0)));
        }
      } else if (!bz) {
        const R c0 = ce[0], c1 = ce[1];
        vr = Add(vr, Sub(Mul(br, c0), Mul(bi, c1)));
        vi = Add(vi, Add(Mul(br, c1), Mul(bi, c0)));
      }
      ce[0] = vr;
      ce[1] = vi;
      return;
    }
  }
  const bool beta_zero = (p.beta_re == R(0) && p.beta_im == R(0));
  const bool beta_one = (p.beta_re == R(1) && p.beta_im == R(0));
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

// One m16n8k8 FP64 MMA: d += a b (a: rows g, g + 8 at k t, t + 4; b: k t,
// t + 4 at column g), the 8 products added in ascending k.
__device__ __forceinline__ void DmmaStep(double (&d)[4], const double (&a)[4],
                                         const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// The end of a KC chunk for a thread's N elements (ei[e], ej[e]): ab =
// (rr - ii, ir + ri), t = alpha * ab as the reference's complex product,
// then t to the chunk's partial buffer (split launches) or merged into C as
// ZMergeElement does. Plain tiles load all of their C elements before the
// first store, so the loads overlap; HERK tiles go element by element.
template <typename R, int N>
__device__ __forceinline__ void ZChunkTile(const ZParams<R>& p, const int (&ei)[N],
                                           const int (&ej)[N], bool first, const R (&rr)[N],
                                           const R (&ir)[N], const R (&ri)[N],
                                           const R (&ii)[N]) {
  R tr[N], ti[N];
#pragma unroll
  for (int e = 0; e < N; ++e) {
    const R ab_re = Sub(rr[e], ii[e]);
    const R ab_im = Add(ir[e], ri[e]);
    tr[e] = Sub(Mul(ab_re, p.alpha_re), Mul(ab_im, p.alpha_im));
    ti[e] = Add(Mul(ab_im, p.alpha_re), Mul(ab_re, p.alpha_im));
  }
  if (p.partial != nullptr) {
#pragma unroll
    for (int e = 0; e < N; ++e) {
      if (ei[e] >= p.m || ej[e] >= p.n) continue;
      R* pe = p.partial +
              2 * ((static_cast<long long>(blockIdx.z) * p.n + ej[e]) * p.m + ei[e]);
      pe[0] = tr[e];
      pe[1] = ti[e];
    }
    return;
  }
  if (p.part != 0) {
#pragma unroll
    for (int e = 0; e < N; ++e)
      if (ei[e] < p.m && ej[e] < p.n) ZMergeElement(p, ei[e], ej[e], first, tr[e], ti[e]);
    return;
  }
  const bool beta_zero = (p.beta_re == R(0) && p.beta_im == R(0));
  const bool beta_one = (p.beta_re == R(1) && p.beta_im == R(0));
  if (first && beta_zero) {
#pragma unroll
    for (int e = 0; e < N; ++e) {
      if (ei[e] >= p.m || ej[e] >= p.n) continue;
      R* ce = p.c + 2 * (ei[e] + ej[e] * p.ldc);
      ce[0] = tr[e];
      ce[1] = ti[e];
    }
    return;
  }
  R c0[N], c1[N];
#pragma unroll
  for (int e = 0; e < N; ++e) {
    c0[e] = c1[e] = R(0);
    if (ei[e] < p.m && ej[e] < p.n) {
      const R* ce = p.c + 2 * (ei[e] + ej[e] * p.ldc);
      c0[e] = ce[0];
      c1[e] = ce[1];
    }
  }
#pragma unroll
  for (int e = 0; e < N; ++e) {
    if (ei[e] >= p.m || ej[e] >= p.n) continue;
    R* ce = p.c + 2 * (ei[e] + ej[e] * p.ldc);
    if (!first || beta_one) {
      ce[0] = Add(tr[e], c0[e]);
      ce[1] = Add(ti[e], c1[e]);
    } else {
      const R b_re = Sub(Mul(c0[e], p.beta_re), Mul(c1[e], p.beta_im));
      const R b_im = Add(Mul(c1[e], p.beta_re), Mul(c0[e], p.beta_im));
      ce[0] = Add(tr[e], b_re);
      ce[1] = Add(ti[e], b_im);
    }
  }
}

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
// one shared load gives both parts; conjugation, chosen at compile time, is
// applied after the load), the next slice in flight while this one is
// multiplied; two CTAs an SM. A chunk ends on a slice boundary (256 is a
// multiple of 16), where the thread merges its chunk into C in memory: the
// running value stays in C itself. FP32 only: FP64 runs ZgemmDmmaKernel.
template <typename R, bool kConjA, bool kConjB>
__global__ void __launch_bounds__(256, 2) ZgemmKernel(ZParams<R> p) {
  if (p.guard != nullptr && *p.guard != 0) return;
  using V = typename Vec2<R>::type;
  extern __shared__ __align__(16) unsigned char zsmem[];
  V* sa = reinterpret_cast<V*>(zsmem);                 // [2][kZK][kZM]
  V* sb = sa + 2 * kZK * kZM;                          // [2][kZK][kZN]
  const int m0 = blockIdx.x * kZM, n0 = blockIdx.y * kZN;
  // A block wholly outside the triangle of C has nothing to do.
  if (p.part == 1 && min(m0 + kZM, p.m) - 1 < n0) return;
  if (p.part == 2 && m0 > min(n0 + kZN, p.n) - 1) return;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  R rr[4][4], ir[4][4], ri[4][4], ii[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) rr[r][q] = ir[r][q] = ri[r][q] = ii[r][q] = R(0);
  const bool split = p.partial != nullptr;
  const int kbeg = split ? blockIdx.z * kZChunk : 0;
  const int kend = split ? min(p.k, kbeg + kZChunk) : p.k;
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
  issue(kbeg, 0);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += kZK, buf ^= 1) {
    if (k0 + kZK < kend) {
      issue(k0 + kZK, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const V* ca = sa + buf * kZK * kZM;
    const V* cb = sb + buf * kZK * kZN;
    const int kslice = min(kZK, kend - k0);
#pragma unroll 2
    for (int kk = 0; kk < kslice; ++kk) {
      R ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const V va = ca[kk * kZM + tx + 16 * r];
        const V vb = cb[kk * kZN + ty + 16 * r];
        ar[r] = va.x;
        ai[r] = kConjA ? Mul(va.y, R(-1)) : va.y;
        br[r] = vb.x;
        bi[r] = kConjB ? Mul(vb.y, R(-1)) : vb.y;
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
    if ((k0 + kZK) % kZChunk == 0 || k0 + kZK >= kend) {
      const bool first = k0 < kZChunk;
      int ei[16], ej[16];
      R vrr[16], vir[16], vri[16], vii[16];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int e = 4 * r + q;
          ei[e] = m0 + tx + 16 * r, ej[e] = n0 + ty + 16 * q;
          vrr[e] = rr[r][q], vir[e] = ir[r][q], vri[e] = ri[r][q], vii[e] = ii[r][q];
          rr[r][q] = ir[r][q] = ri[r][q] = ii[r][q] = R(0);
        }
      ZChunkTile(p, ei, ej, first, vrr, vir, vri, vii);
    }
  }
}

// The FP64 complex GEMM on the FP64 tensor pipe. Each of the four real
// chains of an element (rr, ir, ri, ii) is a `mma.sync.m16n8k8.f64` chain
// over k, which accumulates its products in ascending k exactly as the
// reference's fma chain does; chains restart at every KC chunk, whose end
// goes through the same combine and merge (ZChunkTile). The CTA computes a
// 64 x 64 complex tile with 512 / kFa threads: warps of 16 kFa x 16
// elements (kFa x 2 fragments of 16 x 8, four chains each; kFa = 1 keeps
// 16 warps an SM under 128 registers, which measured faster than 8 warps of
// 32 x 16); k-slices of 16 stream through three shared buffers with
// cp.async (two slices in flight while one is multiplied), complex elements
// interleaved, rows padded to 66 elements so that the 16-byte fragment loads
// of a quarter warp (rows g, k rows t) fall in distinct banks. Zero-filled k
// beyond the end adds fma(0, 0, acc) = acc: a chain started at +0 never
// holds -0.
constexpr int kZdLd = 66, kZdStages = 3, kZdFa = 1;
constexpr int kZdSmemBytes = kZdStages * 2 * kZK * kZdLd * 16;

template <int kFa, bool kConjA, bool kConjB>
__global__ void __launch_bounds__(512 / kFa, 1) ZgemmDmmaKernel(ZParams<double> p) {
  constexpr int kThreads = 512 / kFa;
  if (p.guard != nullptr && *p.guard != 0) return;
  extern __shared__ __align__(16) unsigned char zsmem[];
  double2* sa = reinterpret_cast<double2*>(zsmem);  // [stages][kZK][kZdLd]
  double2* sb = sa + kZdStages * kZK * kZdLd;       // [stages][kZK][kZdLd]
  const int m0 = blockIdx.x * kZM, n0 = blockIdx.y * kZN;
  if (p.part == 1 && min(m0 + kZM, p.m) - 1 < n0) return;
  if (p.part == 2 && m0 > min(n0 + kZN, p.n) - 1) return;
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int g = lane / 4, t = lane % 4;
  constexpr int kWarpsM = 4 / kFa;  // warps along m; 4 along n
  const int wm = (warp % kWarpsM) * 16 * kFa, wn = (warp / kWarpsM) * 16;
  // acc[chain][mt][nt][r]: chains rr, ir, ri, ii; fragment rows g (+8),
  // columns 2t (+1).
  double acc[4][kFa][2][4];
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int a = 0; a < kFa; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[c][a][b][r] = 0.0;
  const bool split = p.partial != nullptr;
  const int kbeg = split ? blockIdx.z * kZChunk : 0;
  const int kend = split ? min(p.k, kbeg + kZChunk) : p.k;
  const bool a_rows = p.a.rs == 1, b_k = p.b.rs == 1;
  // Issues slice k0 into buffer buf (nothing past kend), always committing a
  // group so that the wait counts stay uniform.
  const auto issue = [&](int k0, int buf) {
    if (k0 < kend) {
      double2* da = sa + buf * kZK * kZdLd;
      double2* db = sb + buf * kZK * kZdLd;
      for (int idx = threadIdx.x; idx < kZK * kZM; idx += kThreads) {
        const int kk = a_rows ? idx / kZM : idx % kZK, mm = a_rows ? idx % kZM : idx / kZK;
        const int gi = m0 + mm, gk = k0 + kk;
        const bool ok = gi < p.m && gk < p.k;
        const double* src = ok ? p.a.data + 2 * (gi * p.a.rs + gk * p.a.cs) : p.a.data;
        CpAsyncElem<double>(da + kk * kZdLd + mm, src, ok);
      }
      for (int idx = threadIdx.x; idx < kZK * kZN; idx += kThreads) {
        const int kk = b_k ? idx % kZK : idx / kZN, nn = b_k ? idx / kZK : idx % kZN;
        const int gj = n0 + nn, gk = k0 + kk;
        const bool ok = gj < p.n && gk < p.k;
        const double* src = ok ? p.b.data + 2 * (gk * p.b.rs + gj * p.b.cs) : p.b.data;
        CpAsyncElem<double>(db + kk * kZdLd + nn, src, ok);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  issue(kbeg, 0);
  issue(kbeg + kZK, 1);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += kZK, buf = buf == kZdStages - 1 ? 0 : buf + 1) {
    // This slice's group is the oldest but one; after the barrier every
    // thread is done with the previous slice, whose buffer takes slice + 2.
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    issue(k0 + 2 * kZK, buf == 0 ? kZdStages - 1 : buf - 1);
    const double2* ca = sa + buf * kZK * kZdLd;
    const double2* cb = sb + buf * kZK * kZdLd;
    const int steps = (min(kZK, kend - k0) + 7) / 8;
#pragma unroll
    for (int ks = 0; ks < kZK / 8; ++ks) {
      if (ks >= steps) break;
      double ar[kFa][4], ai[kFa][4], br[2][2], bi[2][2];
#pragma unroll
      for (int a = 0; a < kFa; ++a) {
        const double2* pa = ca + (ks * 8 + t) * kZdLd + wm + a * 16 + g;
        const double2 v0 = pa[0], v1 = pa[8], v2 = pa[4 * kZdLd], v3 = pa[4 * kZdLd + 8];
        ar[a][0] = v0.x, ar[a][1] = v1.x, ar[a][2] = v2.x, ar[a][3] = v3.x;
        ai[a][0] = v0.y, ai[a][1] = v1.y, ai[a][2] = v2.y, ai[a][3] = v3.y;
        if constexpr (kConjA) {
#pragma unroll
          for (int r = 0; r < 4; ++r) ai[a][r] = Mul(ai[a][r], -1.0);
        }
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const double2* pb = cb + (ks * 8 + t) * kZdLd + wn + b * 8 + g;
        const double2 w0 = pb[0], w1 = pb[4 * kZdLd];
        br[b][0] = w0.x, br[b][1] = w1.x;
        bi[b][0] = w0.y, bi[b][1] = w1.y;
        if constexpr (kConjB) bi[b][0] = Mul(bi[b][0], -1.0), bi[b][1] = Mul(bi[b][1], -1.0);
      }
#pragma unroll
      for (int a = 0; a < kFa; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          DmmaStep(acc[0][a][b], ar[a], br[b]);
          DmmaStep(acc[1][a][b], ai[a], br[b]);
          DmmaStep(acc[2][a][b], ar[a], bi[b]);
          DmmaStep(acc[3][a][b], ai[a], bi[b]);
        }
    }
    if ((k0 + kZK) % kZChunk == 0 || k0 + kZK >= kend) {
      const bool first = k0 < kZChunk;
      int ei[8 * kFa], ej[8 * kFa];
      double vrr[8 * kFa], vir[8 * kFa], vri[8 * kFa], vii[8 * kFa];
#pragma unroll
      for (int a = 0; a < kFa; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int e = 8 * a + 4 * b + r;
            ei[e] = m0 + wm + a * 16 + g + (r >= 2 ? 8 : 0);
            ej[e] = n0 + wn + b * 8 + 2 * t + (r & 1);
            vrr[e] = acc[0][a][b][r], vir[e] = acc[1][a][b][r];
            vri[e] = acc[2][a][b][r], vii[e] = acc[3][a][b][r];
            acc[0][a][b][r] = acc[1][a][b][r] = acc[2][a][b][r] = acc[3][a][b][r] = 0.0;
          }
      ZChunkTile(p, ei, ej, first, vrr, vir, vri, vii);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// The in-order merge of a split complex GEMM: per element, chunk 0 with the
// first-chunk rule, then every later chunk (ZMergeElement).
template <typename R>
__global__ void ZSplitMergeKernel(ZParams<R> p, int nchunks) {
  if (p.guard != nullptr && *p.guard != 0) return;
  const long long total = static_cast<long long>(p.m) * p.n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % p.m), j = static_cast<int>(e / p.m);
    for (int c = 0; c < nchunks; ++c) {
      const R* pe = p.partial + 2 * ((static_cast<long long>(c) * p.n + j) * p.m + i);
      ZMergeElement(p, i, j, c == 0, pe[0], pe[1]);
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

// (a + i b) / (c + i d) as the C++ runtime's complex quotient: for double,
// Smith's method with its scalings for very large and very small magnitudes
// and its alternative when the ratio is subnormal; for float, the textbook
// quotient (a c + b d, b c - a d) / (c^2 + d^2) in double precision, rounded.
// (Checked against the host compiler's complex division on random quotients
// spanning 2^-60..2^60, zero parts included; non-finite inputs are not
// reproduced.)
template <typename R>
__device__ __forceinline__ void ZDiv(R ar, R ai, R cr, R ci, R* xr, R* xi) {
  if constexpr (sizeof(R) == 8) {
    double a = ar, b = ai, c = cr, d = ci;
    const double kBig = DBL_MAX / 2, kMin = DBL_MIN, kEps = DBL_EPSILON;
    const double kScale = 1.0 / kEps, kMax2 = kBig * kEps;
    double x, y;
    if (fabs(c) < fabs(d)) {
      if (fabs(d) >= kBig) {
        a = a / 2; b = b / 2; c = c / 2; d = d / 2;
      }
      if (fabs(d) < kEps) {
        a = a * kScale; b = b * kScale; c = c * kScale; d = d * kScale;
      } else if ((fabs(a) < kMin && fabs(b) < kMax2 && fabs(d) < kMax2) ||
                 (fabs(b) < kMin && fabs(a) < kMax2 && fabs(d) < kMax2)) {
        a = a * kScale; b = b * kScale; c = c * kScale; d = d * kScale;
      }
      const double ratio = c / d;
      const double denom = __dadd_rn(__dmul_rn(c, ratio), d);
      if (fabs(ratio) > kMin) {
        x = __dadd_rn(__dmul_rn(a, ratio), b) / denom;
        y = __dsub_rn(__dmul_rn(b, ratio), a) / denom;
      } else {
        x = __dadd_rn(__dmul_rn(c, a / d), b) / denom;
        y = __dsub_rn(__dmul_rn(c, b / d), a) / denom;
      }
    } else {
      if (fabs(c) >= kBig) {
        a = a / 2; b = b / 2; c = c / 2; d = d / 2;
      }
      if (fabs(c) < kEps) {
        a = a * kScale; b = b * kScale; c = c * kScale; d = d * kScale;
      } else if ((fabs(a) < kMin && fabs(b) < kMax2 && fabs(c) < kMax2) ||
                 (fabs(b) < kMin && fabs(a) < kMax2 && fabs(c) < kMax2)) {
        a = a * kScale; b = b * kScale; c = c * kScale; d = d * kScale;
      }
      const double ratio = d / c;
      const double denom = __dadd_rn(__dmul_rn(d, ratio), c);
      if (fabs(ratio) > kMin) {
        x = __dadd_rn(__dmul_rn(b, ratio), a) / denom;
        y = __dsub_rn(b, __dmul_rn(a, ratio)) / denom;
      } else {
        x = __dadd_rn(a, __dmul_rn(d, b / c)) / denom;
        y = __dsub_rn(b, __dmul_rn(d, a / c)) / denom;
      }
    }
    *xr = x;
    *xi = y;
  } else {
    const double a = ar, b = ai, c = cr, d = ci;
    const double den = __dadd_rn(__dmul_rn(c, c), __dmul_rn(d, d));
    const double re = __dadd_rn(__dmul_rn(a, c), __dmul_rn(b, d));
    const double im = __dsub_rn(__dmul_rn(b, c), __dmul_rn(a, d));
    *xr = static_cast<float>(re / den);
    *xi = static_cast<float>(im / den);
  }
}

// 1 / (c + i d): the quotient above with numerator (1, 0).
template <typename R>
__device__ __forceinline__ void ZRecip(R cr, R ci, R* xr, R* xi) {
  ZDiv<R>(R(1), R(0), cr, ci, xr, xi);
}

// Complex TRSM base: X T = B for independent rows of X (src/trsm-inl.h:
// 175-214), T r x r (r <= 32) read through a view. Column j (solve order) is
// b_j - sum of x_q t(q, j) over the solved q in increasing q, kept as four
// fma chains (xr tr, xi tr, xr ti, xi ti) combined as (rr - ii, ir + ri),
// then times inv_j = 1 / t(j, j). One thread owns one row; the row sits in
// registers indexed in solve order (static indices), T in shared memory.
// Element (row, j) of X is at x + 2 * (row * xs_row + j * xs_col).
template <typename R>
__global__ void __launch_bounds__(128)
    ZTrsmBaseKernel(ZView<R> tri, int lower, int unit, int r, int rows, R* x,
                    long long xs_row, long long xs_col, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  // st[s][u] = T(q(s), j(u)) in solve order (conjugated for 'C').
  __shared__ R st_re[32][33], st_im[32][33];
  __shared__ R inv_re[32], inv_im[32];
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int s = idx / 32, u = idx % 32;
    R vr = R(0), vi = R(0);
    if (s < r && u < r && (s < u || (s == u && !unit))) {
      const int q = lower ? r - 1 - s : s, j = lower ? r - 1 - u : u;
      const R* e = tri.data + 2 * (q * tri.rs + j * tri.cs);
      vr = e[0];
      vi = tri.conj ? -e[1] : e[1];
    }
    st_re[s][u] = vr;
    st_im[s][u] = vi;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int s = threadIdx.x;
    R a = R(1), b = R(0);
    if (s < r && !unit) ZRecip<R>(st_re[s][s], st_im[s][s], &a, &b);
    inv_re[s] = a;
    inv_im[s] = b;
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  R* xr = x + 2 * (row * xs_row);
  R yr[32], yi[32];
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) {
      const long long off = 2 * ((lower ? r - 1 - s : s) * xs_col);
      yr[s] = xr[off];
      yi[s] = xr[off + 1];
    }
  }
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s >= r) break;
    R s_rr = R(0), s_ir = R(0), s_ri = R(0), s_ii = R(0);
    // Solved columns in increasing original index: solve order 0..s-1 for
    // upper, s-1 down to 0 for lower.
    if (lower) {
#pragma unroll
      for (int w = 31; w >= 0; --w) {
        if (w >= s) continue;
        const R tr = st_re[w][s], ti = st_im[w][s];
        s_rr = Fma(yr[w], tr, s_rr);
        s_ir = Fma(yi[w], tr, s_ir);
        s_ri = Fma(yr[w], ti, s_ri);
        s_ii = Fma(yi[w], ti, s_ii);
      }
    } else {
#pragma unroll
      for (int w = 0; w < 32; ++w) {
        if (w >= s) break;
        const R tr = st_re[w][s], ti = st_im[w][s];
        s_rr = Fma(yr[w], tr, s_rr);
        s_ir = Fma(yi[w], tr, s_ir);
        s_ri = Fma(yr[w], ti, s_ri);
        s_ii = Fma(yi[w], ti, s_ii);
      }
    }
    R vr = Sub(yr[s], Sub(s_rr, s_ii));
    R vi = Sub(yi[s], Add(s_ir, s_ri));
    if (!unit) {
      const R a0 = Mul(vr, inv_re[s]), a1 = Mul(vi, inv_im[s]);
      const R a2 = Mul(vi, inv_re[s]), a3 = Mul(vr, inv_im[s]);
      vr = Sub(a0, a1);
      vi = Add(a2, a3);
    }
    yr[s] = vr;
    yi[s] = vi;
  }
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) {
      const long long off = 2 * ((lower ? r - 1 - s : s) * xs_col);
      xr[off] = yr[s];
      xr[off + 1] = yi[s];
    }
  }
}

// ---------------------------------------------------------------------------
// Complex LU leaf (src/lapack/factor_kernels.cc:107-139 for complex T).
//
// Per column j: the pivot is the first row of largest |re| + |im| (NaN
// magnitudes never win; a NaN at row j keeps row j: src/level1-inl.h:
// 343-411); the rows are interchanged across the leaf; the column below the
// diagonal is multiplied by 1/pivot as (x.re r.re - x.im r.im, x.im r.re +
// x.re r.im), or divided by the pivot when |pivot| (std::abs) is below the
// safe minimum; then every later column k gets y += (-a(j, k)) x in the
// reference's AXPY rounding (src/lapack/factor_kernels.cc:33-72):
//   columns of fewer reals than one vector: p = alpha x as a complex product
//   (ar xr - ai xi, ar xi + ai xr), then y + p;
//   otherwise re: fma(xi, -ai, fma(xr, ar, yr)), im: fma(xr, ai, fma(xi, ar, yi)).
//
// The m x w panel (w <= 16) is split by rows over P CTAs holding their rows
// in shared memory (a cooperative launch when P > 1); per column each CTA
// publishes its best candidate and one global exchange picks the pivot, as
// in the real leaf.
constexpr int kZLeafThreads = 512;
constexpr int kZLeafW = 16;
constexpr int kZLeafMaxRows = 512;  // rows per CTA
constexpr int kZLeafMaxP = 64;      // CTAs per panel (m <= 32768)
constexpr int kZSlot = 2 + 4 * kZLeafW;  // reals: |a|, row, candidate row, row j

template <typename R>
struct ZLeafArgs {
  int m, w, lanes;
  R* a;            // interleaved (re, im)
  long long lda;   // complex elements
  int* ipiv;
  int* info;
  int info_base;
  R* xchg;               // [2][P][kZSlot]
  unsigned int* tags;    // [2][P], zeroed before a cooperative launch
  int* timeout_flag;
};

template <typename R>
__device__ __forceinline__ R ZMag(R re, R im) {
  return Add(fabs(re), fabs(im));
}

template <typename R>
__device__ __forceinline__ bool ZBetter(R v, int i, R bv, int bi) {
  return v > bv || (v == bv && v >= R(0) && i < bi);
}

// std::abs(z) >= s for the safe minimum s. |z| is at least the larger part,
// so only two parts below s need the magnitude itself: they are scaled by an
// exact power of two (double) or widened (float) and the square root of the
// sum of squares is compared in double precision. (std::abs is hypot: an
// infinite part gives infinity, otherwise a NaN part gives NaN.)
template <typename R>
__device__ __forceinline__ bool ZAbsAtLeast(R re, R im, R s) {
  const R ar = fabs(re), ai = fabs(im);
  if (isinf(ar) || isinf(ai)) return true;
  if (isnan(ar) || isnan(ai)) return false;
  if ((ar > ai ? ar : ai) >= s) return true;
  const double k = sizeof(R) == 8 ? 0x1p600 : 1.0;
  const double sr = __dmul_rn(static_cast<double>(ar), k);
  const double si = __dmul_rn(static_cast<double>(ai), k);
  const double mag = sqrt(__dadd_rn(__dmul_rn(sr, sr), __dmul_rn(si, si)));
  return mag >= __dmul_rn(static_cast<double>(s), k);
}

// y += alpha x for one element of a column of len complex elements.
template <typename R>
__device__ __forceinline__ void ZAxpyRef(R& yr, R& yi, R ar, R ai, R xr, R xi, int len,
                                         int lanes) {
  if (2 * len < lanes) {
    const R pr = Sub(Mul(ar, xr), Mul(ai, xi));
    const R pi = Add(Mul(ar, xi), Mul(ai, xr));
    yr = Add(yr, pr);
    yi = Add(yi, pi);
  } else {
    const R tr = Fma(xr, ar, yr), ti = Fma(xi, ar, yi);
    yr = Fma(xi, -ai, tr);
    yi = Fma(xr, ai, ti);
  }
}

// kCluster: the P CTAs form one thread-block cluster and exchange their
// candidates through distributed shared memory (each publishes into its own
// shared slot, one cluster barrier, then every CTA reads the P slots)
// instead of global slots and polling.
template <typename R, bool kCluster>
__global__ void __launch_bounds__(kZLeafThreads) ZGetrfLeafKernel(ZLeafArgs<R> p) {
  constexpr int W = kZLeafW;
  __shared__ R s_slot[2 * kZSlot];  // kCluster: own slot per parity
  extern __shared__ __align__(16) unsigned char zleaf_smem[];
  R* sp = reinterpret_cast<R*>(zleaf_smem);  // [w][rows][2]
  __shared__ R s_piv[2 * W], s_rowj[2 * W];
  __shared__ R s_cand[kZLeafMaxP * kZSlot];
  __shared__ R s_wv[kZLeafThreads / 32];
  __shared__ int s_wi[kZLeafThreads / 32];
  __shared__ int s_p, s_abort;
  const int P = gridDim.x, cta = blockIdx.x;
  const int rows_per = (p.m + P - 1) / P;
  const int r0 = cta * rows_per, r1 = min(p.m, r0 + rows_per);
  const int RW = rows_per;
  const int w = p.w;
  const auto el = [&](int c, int lr) -> R* { return sp + 2 * (c * RW + lr); };

  if (threadIdx.x == 0) s_abort = 0;
  for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
    const R* src = p.a + 2 * (r0 + lr);
    R v[2 * W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
      if (c < w) {
        v[2 * c] = src[2 * c * p.lda];
        v[2 * c + 1] = src[2 * c * p.lda + 1];
      }
    }
#pragma unroll
    for (int c = 0; c < W; ++c) {
      if (c < w) {
        el(c, lr)[0] = v[2 * c];
        el(c, lr)[1] = v[2 * c + 1];
      }
    }
  }
  // kCluster: every CTA of the cluster is running before any remote access.
  if constexpr (kCluster) cooperative_groups::this_cluster().sync();
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // (a) local candidate over rows >= j.
    R bv = R(-1);
    int bi = 0x7fffffff;
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
      const int gi = r0 + lr;
      if (gi < j) continue;
      const R v = ZMag(el(j, lr)[0], el(j, lr)[1]);
      if (v > bv) { bv = v; bi = gi; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const R ov = __shfl_down_sync(0xffffffffu, bv, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ZBetter(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (threadIdx.x % 32 == 0) { s_wv[threadIdx.x / 32] = bv; s_wi[threadIdx.x / 32] = bi; }
    __syncthreads();
    if (threadIdx.x < 32) {
      bv = threadIdx.x < kZLeafThreads / 32 ? s_wv[threadIdx.x] : R(-1);
      bi = threadIdx.x < kZLeafThreads / 32 ? s_wi[threadIdx.x] : 0x7fffffff;
      for (int off = 16; off > 0; off >>= 1) {
        const R ov = __shfl_down_sync(0xffffffffu, bv, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ZBetter(ov, oi, bv, bi)) { bv = ov; bi = oi; }
      }
      __syncwarp();
      if (threadIdx.x == 0) {
        s_p = bi;
        s_wv[0] = bv;
      }
    }
    __syncthreads();
    // (b) exchange: slot = (|a|, row, candidate row, row j if owned).
    const int ci = s_p;
    R* slot = P == 1 ? s_cand
                     : (kCluster ? s_slot + par * kZSlot : p.xchg + (par * P + cta) * kZSlot);
    if (threadIdx.x == 0) {
      slot[0] = s_wv[0];
      slot[1] = static_cast<R>(ci == 0x7fffffff ? -1 : ci);
    }
    if (threadIdx.x < 2 * w) {
      const int c = threadIdx.x >> 1, part = threadIdx.x & 1;
      slot[2 + threadIdx.x] = (ci != 0x7fffffff) ? el(c, ci - r0)[part] : R(0);
      if (j >= r0 && j < r1) slot[2 + 2 * W + threadIdx.x] = el(c, j - r0)[part];
    }
    if (kCluster && P > 1) {
      // A parity's slot is rewritten two steps later, after the next
      // cluster barrier, which every CTA reaches only after reading it.
      cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
      cluster.sync();
      for (int idx = threadIdx.x; idx < P * kZSlot; idx += blockDim.x) {
        const int q = idx / kZSlot, e = idx - q * kZSlot;
        const R* peer = cluster.map_shared_rank(s_slot, q);
        s_cand[idx] = peer[par * kZSlot + e];
      }
    } else if (P > 1) {
      // Release the slot under the step's tag; poll the P tags (bounded) and
      // copy every slot. A parity is rewritten two steps later, after every
      // CTA has published the next step and so has read this one.
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p.tags + par * P + cta),
                     "r"(static_cast<unsigned>(j + 1))
                     : "memory");
      }
      if (threadIdx.x < P) {
        uint32_t polls = 0;
        while (true) {
          unsigned v;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                       : "=r"(v)
                       : "l"(p.tags + par * P + threadIdx.x)
                       : "memory");
          if (v >= static_cast<unsigned>(j + 1)) break;
          if (++polls >= kMaxPolls) {
            atomicExch(p.timeout_flag, 1);
            s_abort = 1;
            break;
          }
        }
      }
      __syncthreads();
      if (s_abort) return;
      for (int idx = threadIdx.x; idx < P * kZSlot; idx += blockDim.x)
        s_cand[idx] = *(volatile const R*)&p.xchg[par * P * kZSlot + idx];
    }
    __syncthreads();
    if (threadIdx.x < 2 * w)
      s_rowj[threadIdx.x] = s_cand[(j / rows_per) * kZSlot + 2 + 2 * W + threadIdx.x];
    __syncthreads();
    // (c) the pivot among the candidates; warp 0 fills the pivot row.
    if (threadIdx.x < 32) {
      R gv = R(-1);
      int gi = 0x7fffffff, wq = -1;
      for (int q = threadIdx.x; q < P; q += 32) {
        const R fi = s_cand[q * kZSlot + 1];
        if (fi < R(0)) continue;
        const R v = s_cand[q * kZSlot];
        const int i = static_cast<int>(fi);
        if (ZBetter(v, i, gv, gi)) { gv = v; gi = i; wq = q; }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const R ov = __shfl_down_sync(0xffffffffu, gv, off);
        const int oi = __shfl_down_sync(0xffffffffu, gi, off);
        const int oq = __shfl_down_sync(0xffffffffu, wq, off);
        if (ZBetter(ov, oi, gv, gi)) { gv = ov; gi = oi; wq = oq; }
      }
      gi = __shfl_sync(0xffffffffu, gi, 0);
      wq = __shfl_sync(0xffffffffu, wq, 0);
      if (isnan(ZMag(s_rowj[2 * j], s_rowj[2 * j + 1])) || gi == 0x7fffffff) gi = j;
      if (threadIdx.x == 0) s_p = gi;
      if (threadIdx.x < 2 * w)
        s_piv[threadIdx.x] = (gi == j) ? s_rowj[threadIdx.x]
                                       : s_cand[wq * kZSlot + 2 + threadIdx.x];
    }
    __syncthreads();
    const int piv = s_p;
    const R pr = s_piv[2 * j], pi = s_piv[2 * j + 1];
    const bool nonzero = pr != R(0) || pi != R(0);
    if (cta == 0 && threadIdx.x == 0) {
      p.ipiv[j] = piv + 1;
      if (!nonzero && *p.info == 0) *p.info = p.info_base + j + 1;
    }
    // (d) interchange rows j and piv across the leaf's columns.
    if (nonzero && piv != j && threadIdx.x < 2 * w) {
      const int c = threadIdx.x >> 1, part = threadIdx.x & 1;
      if (piv >= r0 && piv < r1) el(c, piv - r0)[part] = s_rowj[threadIdx.x];
      if (j >= r0 && j < r1) el(c, j - r0)[part] = s_piv[threadIdx.x];
    }
    __syncthreads();
    // (e) scale column j below the diagonal; (f) update columns j+1..w-1.
    const bool tiny = !ZAbsAtLeast(pr, pi, Sfmin<R>());
    R vr = R(0), vi = R(0);
    if (nonzero && !tiny) ZRecip<R>(pr, pi, &vr, &vi);
    const int len = p.m - j - 1;
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
      if (r0 + lr <= j) continue;
      R xr = el(j, lr)[0], xi = el(j, lr)[1];
      if (nonzero) {
        if (tiny) {
          ZDiv<R>(xr, xi, pr, pi, &xr, &xi);
        } else {
          const R nr = Sub(Mul(xr, vr), Mul(xi, vi));
          const R ni = Add(Mul(xi, vr), Mul(xr, vi));
          xr = nr;
          xi = ni;
        }
        el(j, lr)[0] = xr;
        el(j, lr)[1] = xi;
      }
      for (int k = j + 1; k < w; ++k) {
        R* y = el(k, lr);
        ZAxpyRef<R>(y[0], y[1], -s_piv[2 * k], -s_piv[2 * k + 1], xr, xi, len, p.lanes);
      }
    }
  }
  __syncthreads();
  // kCluster: no CTA exits while a peer may still read its slot.
  if constexpr (kCluster) cooperative_groups::this_cluster().sync();
  for (int c = 0; c < w; ++c) {
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
      R* dst = p.a + 2 * ((r0 + lr) + c * p.lda);
      dst[0] = el(c, lr)[0];
      dst[1] = el(c, lr)[1];
    }
  }
}

// Complex LU leaf, trailing columns (n > m, m <= 16): all interchanges, then
// the updates with the final multipliers (the same arithmetic as the
// reference's interleaved order, as in the real leaf). One thread per column.
template <typename R>
__global__ void ZGetrfLeafTrailingKernel(int m, int w, int n, R* a, long long lda,
                                         const int* ipiv, int lanes) {
  const int k = w + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  R* col = a + 2 * k * lda;
  for (int j = 0; j < w; ++j) {
    const int q = ipiv[j] - 1;
    if (q != j) {
      const R tr = col[2 * j], ti = col[2 * j + 1];
      col[2 * j] = col[2 * q];
      col[2 * j + 1] = col[2 * q + 1];
      col[2 * q] = tr;
      col[2 * q + 1] = ti;
    }
  }
  for (int j = 0; j < w; ++j) {
    const R ar = -col[2 * j], ai = -col[2 * j + 1];
    const int len = m - j - 1;
    for (int i = j + 1; i < m; ++i) {
      const R* x = a + 2 * (i + j * lda);
      ZAxpyRef<R>(col[2 * i], col[2 * i + 1], ar, ai, x[0], x[1], len, lanes);
    }
  }
}

// ---------------------------------------------------------------------------
// Complex Cholesky leaf (src/lapack/factor_kernels.cc:141-175 for complex T,
// n <= 32) in one CTA, the referenced triangle in shared memory. Per column
// j: the real part of the diagonal must be positive (else INFO = j + 1 and
// stop); it becomes (sqrt, 0) and rinv = 1 / sqrt scales the row (upper) or
// column (lower) part by part; then
//   upper: column k > j, rows j+1..k: y += (-U(j, k)) conj(U(j, i)), length k - j;
//   lower: column k > j, rows k..n-1: y += (-conj(L(k, j))) L(i, j), length n - k;
// in the reference's complex AXPY rounding.
template <typename R>
__global__ void __launch_bounds__(256)
    ZPotrfLeafKernel(int upper, int n, R* a, long long lda, int* info, int info_base,
                     int lanes, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ R sr[32][33], si[32][33];  // A(i, j)
  __shared__ R row_r[32], row_i[32];
  __shared__ R s_rinv;
  __shared__ int stop;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    const bool ref = upper ? (i <= j) : (i >= j);
    const R* e = a + 2 * (i + j * lda);
    sr[i][j] = ref ? e[0] : R(0);
    si[i][j] = ref ? e[1] : R(0);
  }
  if (threadIdx.x == 0) stop = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x == 0) {
      const R ajj = sr[j][j];
      if (ajj <= R(0) || isnan(ajj)) {
        stop = 1;
        if (*info == 0) *info = info_base + j + 1;
      } else {
        const R r = sqrt(ajj);
        sr[j][j] = r;
        si[j][j] = R(0);
        s_rinv = R(1) / r;
      }
    }
    __syncthreads();
    if (stop) break;
    const R rinv = s_rinv;
    if (upper) {
      for (int k = j + 1 + threadIdx.x; k < n; k += blockDim.x) {
        sr[j][k] = Mul(sr[j][k], rinv);
        si[j][k] = Mul(si[j][k], rinv);
        row_r[k] = sr[j][k];
        row_i[k] = -si[j][k];
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, k = idx / n;
        if (k <= j || i <= j || i > k) continue;
        ZAxpyRef<R>(sr[i][k], si[i][k], -sr[j][k], -si[j][k], row_r[i], row_i[i], k - j,
                    lanes);
      }
    } else {
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
        sr[i][j] = Mul(sr[i][j], rinv);
        si[i][j] = Mul(si[i][j], rinv);
      }
      __syncthreads();
      for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, k = idx / n;
        if (k <= j || i < k) continue;
        ZAxpyRef<R>(sr[i][k], si[i][k], -sr[k][j], si[k][j], sr[i][j], si[i][j], n - k,
                    lanes);
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    const bool ref = upper ? (i <= j) : (i >= j);
    if (ref) {
      R* e = a + 2 * (i + j * lda);
      e[0] = sr[i][j];
      e[1] = si[i][j];
    }
  }
}

// HERK's quick path with beta != 1 (src/gemm.cc:48-64 with real_diagonal):
// the triangle `part` of C times beta (zeros for beta 0) as the runtime's
// complex product, the diagonal first reduced to its real part.
template <typename R>
__global__ void ZScaleTriangleKernel(int n, int lower, R beta, R* c, long long ldc,
                                     const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  const long long total = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (lower ? i < j : i > j) continue;
    R* ce = c + 2 * (i + j * ldc);
    R c0 = ce[0], c1 = ce[1];
    if (i == j) c1 = R(0);
    if (beta == R(0)) {
      ce[0] = R(0);
      ce[1] = R(0);
    } else {
      ce[0] = Sub(Mul(c0, beta), Mul(c1, R(0)));
      ce[1] = Add(Mul(c0, R(0)), Mul(c1, beta));
    }
  }
}

}  // namespace

// The complex GEMM kernel on operand views (elements aligned to their size;
// m, n, k > 0): C := alpha op(A) op(B) + beta C with the reference's merges.
template <typename R>
void ZgemmViews(int m, int n, int k, const R* alpha, ZView<R> a, ZView<R> b, const R* beta,
                R* c, int ldc, int part = 0) {
  ZParams<R> p;
  p.m = m;
  p.n = n;
  p.k = k;
  p.alpha_re = alpha[0];
  p.alpha_im = alpha[1];
  p.beta_re = beta[0];
  p.beta_im = beta[1];
  p.a = a;
  p.b = b;
  p.c = c;
  p.ldc = ldc;
  p.guard = Ctx().guard;
  p.part = part;
  p.real_diag = part != 0 ? 1 : 0;
  // The reference's complex micro-tile: 2 vectors of lanes reals per column
  // (lanes / 2 complex rows each), 6 columns with 32 vector registers, 3
  // with 16 (src/gemm_kernel-inl.h:243-257).
  const int lanes = sizeof(R) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  p.tmr = lanes;
  p.tnr = RefLanesDouble() == 8 ? 6 : 3;
  const dim3 grid((m + kZM - 1) / kZM, (n + kZN - 1) / kZN);
  // FP64 runs the four chains on the tensor pipe, FP32 on the CUDA cores.
  void* fn;
  int smem, threads = 256;
  if constexpr (sizeof(R) == 8) {
    fn = a.conj ? (b.conj ? reinterpret_cast<void*>(ZgemmDmmaKernel<kZdFa, true, true>)
                          : reinterpret_cast<void*>(ZgemmDmmaKernel<kZdFa, true, false>))
                : (b.conj ? reinterpret_cast<void*>(ZgemmDmmaKernel<kZdFa, false, true>)
                          : reinterpret_cast<void*>(ZgemmDmmaKernel<kZdFa, false, false>));
    threads = 512 / kZdFa;
    smem = kZdSmemBytes;
  } else {
    fn = a.conj ? (b.conj ? reinterpret_cast<void*>(ZgemmKernel<R, true, true>)
                          : reinterpret_cast<void*>(ZgemmKernel<R, true, false>))
                : (b.conj ? reinterpret_cast<void*>(ZgemmKernel<R, false, true>)
                          : reinterpret_cast<void*>(ZgemmKernel<R, false, false>));
    smem = ZSmemBytes<R>();
  }
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  void* args[] = {&p};
  // Few tiles and several KC chunks: the chunks run in parallel (each one's
  // alpha * ab does not depend on C) and are merged in order afterwards,
  // which gives the same C as merging them one after another.
  const long long tiles = static_cast<long long>(grid.x) * grid.y;
  const int nchunks = (k + kZChunk - 1) / kZChunk;
  const size_t pbytes = 2 * sizeof(R) * static_cast<size_t>(nchunks) * m * n;
  p.partial = nullptr;
  if (nchunks >= 2 && tiles * 2 <= Ctx().num_sms && pbytes <= (size_t(1) << 30)) {
    p.partial = static_cast<R*>(Workspace(kWsSplitK, pbytes));
    if (p.partial == nullptr) return;
    cudaLaunchKernel(fn, dim3(grid.x, grid.y, nchunks), threads, args, smem, Ctx().stream);
    CountLaunch();
    if (LaunchFailed("complex gemm (split)")) return;
    const long long total = static_cast<long long>(m) * n;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 8));
    ZSplitMergeKernel<R><<<blocks, 256, 0, Ctx().stream>>>(p, nchunks);
    CountLaunch();
    LaunchFailed("complex gemm split merge");
    return;
  }
  cudaLaunchKernel(fn, grid, threads, args, smem, Ctx().stream);
  CountLaunch();
  LaunchFailed("complex gemm");
}

// Partial-buffer bytes of a complex GEMM that splits over its KC chunks (0
// when it does not split); the same rule as ZgemmViews.
template <typename R>
size_t ZSplitBytes(int m, int n, int k) {
  const long long tiles =
      static_cast<long long>((m + kZM - 1) / kZM) * ((n + kZN - 1) / kZN);
  const int nchunks = (k + kZChunk - 1) / kZChunk;
  const size_t pbytes = 2 * sizeof(R) * static_cast<size_t>(nchunks) * m * n;
  if (m <= 0 || n <= 0 || nchunks < 2 || tiles * 2 > Ctx().num_sms ||
      pbytes > (size_t(1) << 30))
    return 0;
  return pbytes;
}

// The largest split buffer any GEMM update of a TRSM recursion on an r x r
// triangle takes (both split orders, so either uplo).
template <typename R>
size_t ZTrsmSplitMax(int r, int other) {
  constexpr int kBase = 32;
  if (r <= kBase || other <= 0) return 0;
  const int r1 = std::max(kBase, (r / 2) / kBase * kBase), r2 = r - r1;
  return std::max({ZTrsmSplitMax<R>(r1, other), ZTrsmSplitMax<R>(r2, other),
                   ZSplitBytes<R>(r2, other, r1), ZSplitBytes<R>(r1, other, r2)});
}

// The same for the recursive LU of an m x n panel.
template <typename R>
size_t ZGetrfSplitMax(int m, int n) {
  if (m <= 0 || n <= 0 || std::min(m, n) <= 16) return 0;
  const int n1 = std::min(m, n) / 2, n2 = n - n1;
  return std::max({ZGetrfSplitMax<R>(m, n1), ZTrsmSplitMax<R>(n1, n2),
                   ZSplitBytes<R>(m - n1, n2, n1), ZGetrfSplitMax<R>(m - n1, n2)});
}

// Reserves the split buffer a whole driver call needs before its first
// launch: growing it between launches would synchronize and reallocate in
// the middle of the call.
template <typename R>
bool ZReserveSplit(size_t bytes) {
  return bytes == 0 || Workspace(kWsSplitK, bytes) != nullptr;
}

// The complex TRSM recursion (src/trsm.cc:87-135) on an op(A) view.
template <typename R>
static void ZTrsmRec(bool left, ZView<R> tri, bool lower, bool unit, int r, int other, R* b,
                     int ldb) {
  constexpr int kBase = 32;
  if (r <= 0 || other <= 0) return;
  if (r <= kBase) {
    ZView<R> t = tri;
    bool lo = lower;
    long long xs_row, xs_col;
    if (left) {  // T X = B  <=>  X^T T^T = B^T (src/trsm-inl.h:306-324)
      t.rs = tri.cs;
      t.cs = tri.rs;
      lo = !lower;
      xs_row = ldb;
      xs_col = 1;
    } else {
      xs_row = 1;
      xs_col = ldb;
    }
    ZTrsmBaseKernel<R><<<(other + 127) / 128, 128, 0, Ctx().stream>>>(
        t, lo ? 1 : 0, unit ? 1 : 0, r, other, b, xs_row, xs_col, Ctx().guard);
    CountLaunch();
    LaunchFailed("complex trsm base");
    return;
  }
  const int r1 = std::max(kBase, (r / 2) / kBase * kBase), r2 = r - r1;
  const auto sub = [&](int i0, int j0) {
    ZView<R> v = tri;
    v.data += 2 * (i0 * tri.rs + j0 * tri.cs);
    return v;
  };
  const ZView<R> t11 = tri, t22 = sub(r1, r1), toff = lower ? sub(r1, 0) : sub(0, r1);
  const R m1[2] = {R(-1), R(0)}, one[2] = {R(1), R(0)};
  const auto col = [&](R* p) { return ZView<R>{p, 1, ldb, 0}; };
  if (left) {
    R* b1 = b;
    R* b2 = b + 2 * r1;
    if (lower) {
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
      ZgemmViews<R>(r2, other, r1, m1, toff, col(b1), one, b2, ldb);
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
    } else {
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
      ZgemmViews<R>(r1, other, r2, m1, toff, col(b2), one, b1, ldb);
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
    }
  } else {
    R* b1 = b;
    R* b2 = b + 2 * static_cast<long long>(r1) * ldb;
    if (lower) {
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
      ZgemmViews<R>(other, r1, r2, m1, col(b2), toff, one, b1, ldb);
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
    } else {
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
      ZgemmViews<R>(other, r2, r1, m1, col(b1), toff, one, b2, ldb);
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
    }
  }
}

// Complex TRSM (src/trsm.cc:137-180) after argument checks: B := alpha B
// (alpha != 1), zero B for alpha 0, then the recursion on op(A) (op 0 N,
// 1 T, 2 C). A and B are used where they are when their elements are aligned
// to their size (cp.async in the GEMM updates), else through aligned copies.
template <typename R>
void ZtrsmFull(bool left, bool lower, int op, bool unit, int m, int n, const R* alpha,
               const R* a, int lda, R* b, int ldb) {
  if (m == 0 || n == 0) return;
  const bool alpha_one = alpha[0] == R(1) && alpha[1] == R(0);
  const bool alpha_zero = alpha[0] == R(0) && alpha[1] == R(0);
  if (!alpha_one) {
    const long long total = static_cast<long long>(m) * n;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 8));
    ZScaleKernel<R><<<blocks, 256, 0, Ctx().stream>>>(m, n, alpha[0], alpha[1], b, ldb,
                                                        Ctx().guard);
    CountLaunch();
    if (LaunchFailed("complex trsm scale")) return;
  }
  if (alpha_zero) return;
  const int ka = left ? m : n;
  const size_t esz = 2 * sizeof(R);
  if (reinterpret_cast<uintptr_t>(a) % esz != 0) {
    R* dst = static_cast<R*>(Workspace(kWsLevel3, esz * static_cast<size_t>(ka) * ka));
    if (dst == nullptr ||
        Failed(cudaMemcpy2DAsync(dst, esz * ka, a, esz * lda, esz * ka, ka,
                                 cudaMemcpyDeviceToDevice, Ctx().stream),
               "complex trsm copy"))
      return;
    a = dst;
    lda = ka;
  }
  R* bw = b;
  int ldbw = ldb;
  if (reinterpret_cast<uintptr_t>(b) % esz != 0) {
    bw = static_cast<R*>(Workspace(kWsLevel3Copy, esz * static_cast<size_t>(m) * n));
    if (bw == nullptr ||
        Failed(cudaMemcpy2DAsync(bw, esz * m, b, esz * ldb, esz * m, n,
                                 cudaMemcpyDeviceToDevice, Ctx().stream),
               "complex trsm copy"))
      return;
    ldbw = m;
  }
  const ZView<R> tri = op == 0 ? ZView<R>{a, 1, lda, 0} : ZView<R>{a, lda, 1, op == 2 ? 1 : 0};
  const bool op_lower = lower != (op != 0);
  if (!ZReserveSplit<R>(ZTrsmSplitMax<R>(ka, left ? n : m))) return;
  ZTrsmRec<R>(left, tri, op_lower, unit, ka, left ? n : m, bw, ldbw);
  if (bw != b) {
    Failed(cudaMemcpy2DAsync(b, esz * ldb, bw, esz * m, esz * m, n, cudaMemcpyDeviceToDevice,
                             Ctx().stream),
           "complex trsm copy back");
  }
}
template void ZtrsmFull<double>(bool, bool, int, bool, int, int, const double*, const double*,
                                int, double*, int);
template void ZtrsmFull<float>(bool, bool, int, bool, int, int, const float*, const float*,
                               int, float*, int);

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
  ZgemmViews<R>(m, n, k, alpha,
                ta == 0 ? ZView<R>{a, 1, lda, 0} : ZView<R>{a, lda, 1, ta == 2 ? 1 : 0},
                tb == 0 ? ZView<R>{b, 1, ldb, 0} : ZView<R>{b, ldb, 1, tb == 2 ? 1 : 0}, beta,
                c, ldc);
}
template void ZgemmFull<double>(int, int, int, int, int, const double*, const double*, int,
                                const double*, int, const double*, double*, int);
template void ZgemmFull<float>(int, int, int, int, int, const float*, const float*, int,
                               const float*, int, const float*, float*, int);

// ---------------------------------------------------------------------------
// Complex LU drivers: the reference's Getrf2 recursion and blocked Getrf
// (src/lapack/getrf.cc:112-280, nb = 64 from src/lapack/environment.cc:86-88)
// and Getrs (287-339), call for call, on the complex TRSM and GEMM above.

template <typename R>
void ZLaswp(int n, R* a, int lda, int k1, int k2, const int* ipiv, int incx) {
  Laswp<ZPair<R>>(n, reinterpret_cast<ZPair<R>*>(a), lda, k1, k2, ipiv, incx);
}
template void ZLaswp<double>(int, double*, int, int, int, const int*, int);
template void ZLaswp<float>(int, float*, int, int, int, const int*, int);

namespace {
template <typename R>
R* ZAt(R* a, int lda, int i, int j) {
  return a + 2 * (i + static_cast<long long>(j) * lda);
}

template <typename R>
void ZGetrfLeaf(int m, int n, R* a, int lda, int* ipiv, int* info, int info_base) {
  Context& ctx = Ctx();
  const int w = std::min(m, n);
  const int lanes = sizeof(R) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  const int P = (m + kZLeafMaxRows - 1) / kZLeafMaxRows;
  if (P > kZLeafMaxP) {
    fprintf(stderr, "hwyblas_b200: complex LU panel of %d rows exceeds the leaf's limit\n", m);
    Failed(cudaErrorInvalidValue, "complex getrf leaf size");
    return;
  }
  const int rows = (m + P - 1) / P;
  const size_t smem = 2 * sizeof(R) * static_cast<size_t>(w) * rows;
  static bool configured = false;
  static int max_cluster = 0;
  if (!configured) {
    const int smem_max = static_cast<int>(2 * sizeof(R) * kZLeafW * kZLeafMaxRows);
    cudaFuncSetAttribute(ZGetrfLeafKernel<R, false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ZGetrfLeafKernel<R, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(ZGetrfLeafKernel<R, true>,
                         cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kZLeafThreads);
    cfg.dynamicSmemBytes = smem_max;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 16;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int size = 0;
    if (cudaOccupancyMaxPotentialClusterSize(
            &size, reinterpret_cast<const void*>(ZGetrfLeafKernel<R, true>), &cfg) !=
        cudaSuccess) {
      cudaGetLastError();
      size = 0;
    }
    max_cluster = std::min(size, 16);
    configured = true;
  }
  ZLeafArgs<R> args;
  args.m = m;
  args.w = w;
  args.lanes = lanes;
  args.a = a;
  args.lda = lda;
  args.ipiv = ipiv;
  args.info = info;
  args.info_base = info_base;
  const size_t slot_bytes = sizeof(R) * 2 * kZLeafMaxP * kZSlot;
  args.xchg = static_cast<R*>(
      Workspace(kWsLeaf, slot_bytes + sizeof(unsigned int) * 2 * kZLeafMaxP));
  if (args.xchg == nullptr) return;
  args.tags = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(args.xchg) + slot_bytes);
  args.timeout_flag = ctx.dev_status;
  if (P > 1 && P <= max_cluster) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P);
    cfg.blockDim = dim3(kZLeafThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx.stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = P;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    Failed(cudaLaunchKernelEx(&cfg, ZGetrfLeafKernel<R, true>, args),
           "complex getrf leaf (cluster)");
  } else if (P > 1) {
    cudaMemsetAsync(args.tags, 0, sizeof(unsigned int) * 2 * P, ctx.stream);
    void* kargs[] = {&args};
    Failed(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(ZGetrfLeafKernel<R, false>), P,
                                       kZLeafThreads, kargs, smem, ctx.stream),
           "complex getrf leaf (cooperative)");
  } else {
    ZGetrfLeafKernel<R, false><<<1, kZLeafThreads, smem, ctx.stream>>>(args);
  }
  CountLaunch();
  LaunchFailed("complex getrf leaf");
  if (n > w) {
    ZGetrfLeafTrailingKernel<R><<<(n - w + 127) / 128, 128, 0, ctx.stream>>>(
        m, w, n, a, lda, ipiv, lanes);
    CountLaunch();
    LaunchFailed("complex getrf leaf trailing");
  }
}

template <typename R>
void ZGetrfRec(int m, int n, R* a, int lda, int* ipiv, int* info, int col0) {
  if (m == 0 || n == 0) return;
  if (std::min(m, n) <= 16) {
    ZGetrfLeaf<R>(m, n, a, lda, ipiv, info, col0);
    return;
  }
  const R one[2] = {R(1), R(0)}, m1[2] = {R(-1), R(0)};
  const int n1 = std::min(m, n) / 2, n2 = n - n1;
  ZGetrfRec<R>(m, n1, a, lda, ipiv, info, col0);
  ZLaswp<R>(n2, ZAt(a, lda, 0, n1), lda, 1, n1, ipiv, 1);
  ZtrsmFull<R>(true, true, 0, true, n1, n2, one, a, lda, ZAt(a, lda, 0, n1), lda);
  ZgemmFull<R>(0, 0, m - n1, n2, n1, m1, ZAt(a, lda, n1, 0), lda, ZAt(a, lda, 0, n1), lda,
               one, ZAt(a, lda, n1, n1), lda);
  ZGetrfRec<R>(m - n1, n2, ZAt(a, lda, n1, n1), lda, ipiv + n1, info, col0 + n1);
  AdjustPivots(ipiv, n1, std::min(m, n), n1);
  ZLaswp<R>(n1, a, lda, n1 + 1, std::min(m, n), ipiv, 1);
}
}  // namespace

template <typename R>
void ZGetrf(bool recursive, int m, int n, R* a, int lda, int* ipiv, int* info) {
  if (m == 0 || n == 0) return;
  const int nb = 64, mn = std::min(m, n);
  if (recursive || nb >= mn) {
    if (!ZReserveSplit<R>(ZGetrfSplitMax<R>(m, n))) return;
    ZGetrfRec<R>(m, n, a, lda, ipiv, info, 0);
    return;
  }
  size_t split_bytes = 0;
  for (int j = 0; j < mn; j += nb) {
    const int jb = std::min(mn - j, nb);
    split_bytes = std::max({split_bytes, ZGetrfSplitMax<R>(m - j, jb),
                            ZTrsmSplitMax<R>(jb, n - j - jb),
                            ZSplitBytes<R>(m - j - jb, n - j - jb, jb)});
  }
  if (!ZReserveSplit<R>(split_bytes)) return;
  const R one[2] = {R(1), R(0)}, m1[2] = {R(-1), R(0)};
  for (int j = 0; j < mn; j += nb) {
    const int jb = std::min(mn - j, nb);
    ZGetrfRec<R>(m - j, jb, ZAt(a, lda, j, j), lda, ipiv + j, info, j);
    AdjustPivots(ipiv, j, std::min(m, j + jb), j);
    ZLaswp<R>(j, a, lda, j + 1, j + jb, ipiv, 1);
    if (j + jb < n) {
      ZLaswp<R>(n - j - jb, ZAt(a, lda, 0, j + jb), lda, j + 1, j + jb, ipiv, 1);
      ZtrsmFull<R>(true, true, 0, true, jb, n - j - jb, one, ZAt(a, lda, j, j), lda,
                   ZAt(a, lda, j, j + jb), lda);
      if (j + jb < m) {
        ZgemmFull<R>(0, 0, m - j - jb, n - j - jb, jb, m1, ZAt(a, lda, j + jb, j), lda,
                     ZAt(a, lda, j, j + jb), lda, one, ZAt(a, lda, j + jb, j + jb), lda);
      }
    }
  }
}
template void ZGetrf<double>(bool, int, int, double*, int, int*, int*);
template void ZGetrf<float>(bool, int, int, float*, int, int*, int*);

template <typename R>
void ZGetrs(int op, int n, int nrhs, const R* a, int lda, const int* ipiv, R* b, int ldb) {
  if (n == 0 || nrhs == 0) return;
  const R one[2] = {R(1), R(0)};
  if (!ZReserveSplit<R>(ZTrsmSplitMax<R>(n, nrhs))) return;
  if (op == 0) {
    ZLaswp<R>(nrhs, b, ldb, 1, n, ipiv, 1);
    ZtrsmFull<R>(true, true, 0, true, n, nrhs, one, a, lda, b, ldb);
    ZtrsmFull<R>(true, false, 0, false, n, nrhs, one, a, lda, b, ldb);
  } else {
    ZtrsmFull<R>(true, false, op, false, n, nrhs, one, a, lda, b, ldb);
    ZtrsmFull<R>(true, true, op, true, n, nrhs, one, a, lda, b, ldb);
    ZLaswp<R>(nrhs, b, ldb, 1, n, ipiv, -1);
  }
}
template void ZGetrs<double>(int, int, int, const double*, int, const int*, double*, int);
template void ZGetrs<float>(int, int, int, const float*, int, const int*, float*, int);


// ---------------------------------------------------------------------------
// Complex HERK (src/level3.cc:85-140): C := alpha op(A) op(A)^H + beta C on
// the triangle of C, alpha and beta real, op 0 N (A n x k) / 2 C (A k x n).
// The elements are the complex GEMM's; tiles of the reference crossing the
// diagonal merge as its MergeTile with the diagonal kept real.
template <typename R>
void ZherkFull(bool lower, int op, int n, int k, R alpha, const R* a, int lda, R beta, R* c,
               int ldc) {
  if (n == 0 || ((alpha == R(0) || k == 0) && beta == R(1))) return;
  if (alpha == R(0) || k == 0) {
    const long long total = static_cast<long long>(n) * n;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 8));
    ZScaleTriangleKernel<R><<<blocks, 256, 0, Ctx().stream>>>(n, lower ? 1 : 0, beta, c, ldc,
                                                                Ctx().guard);
    CountLaunch();
    LaunchFailed("complex herk scale");
    return;
  }
  const R al[2] = {alpha, R(0)}, be[2] = {beta, R(0)};
  const ZView<R> plain{a, 1, lda, 0}, herm{a, lda, 1, 1};
  ZgemmViews<R>(n, n, k, al, op == 0 ? plain : herm, op == 0 ? herm : plain, be, c, ldc,
                lower ? 1 : 2);
}
template void ZherkFull<double>(bool, int, int, int, double, const double*, int, double,
                                double*, int);
template void ZherkFull<float>(bool, int, int, int, float, const float*, int, float, float*,
                               int);

// Complex Cholesky drivers: the reference's Potrf2 recursion (leaf n <= 32)
// and blocked Potrf (nb = 64, src/lapack/environment.cc:110-111), call for
// call (src/lapack/potrf.cc:48-199), and Potrs (src/lapack/posv.cc:31-76).
// The device INFO doubles as the guard that turns the call's later kernels
// into no-ops once a leaf finds a non-positive minor.
namespace {
template <typename R>
void ZPotrfLeaf(bool upper, int n, R* a, int lda, int* info, int info_base) {
  const int lanes = sizeof(R) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  ZPotrfLeafKernel<R><<<1, 256, 0, Ctx().stream>>>(upper ? 1 : 0, n, a, lda, info, info_base,
                                                    lanes, Ctx().guard);
  CountLaunch();
  LaunchFailed("complex potrf leaf");
}

template <typename R>
void ZPotrf2Rec(bool upper, int n, R* a, int lda, int* info, int col0) {
  if (n == 0) return;
  if (n <= 32) {
    ZPotrfLeaf<R>(upper, n, a, lda, info, col0);
    return;
  }
  const R one[2] = {R(1), R(0)};
  const int n1 = n / 2, n2 = n - n1;
  ZPotrf2Rec<R>(upper, n1, a, lda, info, col0);
  if (upper) {
    ZtrsmFull<R>(true, false, 2, false, n1, n2, one, a, lda, ZAt(a, lda, 0, n1), lda);
    ZherkFull<R>(false, 2, n2, n1, R(-1), ZAt(a, lda, 0, n1), lda, R(1), ZAt(a, lda, n1, n1),
                 lda);
  } else {
    ZtrsmFull<R>(false, true, 2, false, n2, n1, one, a, lda, ZAt(a, lda, n1, 0), lda);
    ZherkFull<R>(true, 0, n2, n1, R(-1), ZAt(a, lda, n1, 0), lda, R(1), ZAt(a, lda, n1, n1),
                 lda);
  }
  ZPotrf2Rec<R>(upper, n2, ZAt(a, lda, n1, n1), lda, info, col0 + n1);
}
}  // namespace

template <typename R>
void ZPotrf(bool recursive, bool upper, int n, R* a, int lda, int* info) {
  if (n == 0) return;
  Context& ctx = Ctx();
  const int* saved = ctx.guard;
  ctx.guard = info;
  const int nb = 64;
  if (recursive || nb >= n) {
    ZPotrf2Rec<R>(upper, n, a, lda, info, 0);
    ctx.guard = saved;
    return;
  }
  // The block updates have few tiles and long k, so the GEMMs split over
  // their KC chunks; their largest partial buffer is reserved up front
  // (growing it inside the loop would synchronize at every step).
  size_t split_bytes = 0;
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    const size_t chunks = static_cast<size_t>((j + kZChunk - 1) / kZChunk);
    split_bytes = std::max(split_bytes, 2 * sizeof(R) * chunks * std::max(n - j, jb) * jb);
  }
  if (split_bytes > 0 && Workspace(kWsSplitK, split_bytes) == nullptr) {
    ctx.guard = saved;
    return;
  }
  const R one[2] = {R(1), R(0)}, m1[2] = {R(-1), R(0)};
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    if (upper) {
      ZherkFull<R>(false, 2, jb, j, R(-1), ZAt(a, lda, 0, j), lda, R(1), ZAt(a, lda, j, j), lda);
      ZPotrf2Rec<R>(true, jb, ZAt(a, lda, j, j), lda, info, j);
      if (j + jb < n) {
        ZgemmFull<R>(2, 0, jb, n - j - jb, j, m1, ZAt(a, lda, 0, j), lda,
                     ZAt(a, lda, 0, j + jb), lda, one, ZAt(a, lda, j, j + jb), lda);
        ZtrsmFull<R>(true, false, 2, false, jb, n - j - jb, one, ZAt(a, lda, j, j), lda,
                     ZAt(a, lda, j, j + jb), lda);
      }
    } else {
      ZherkFull<R>(true, 0, jb, j, R(-1), ZAt(a, lda, j, 0), lda, R(1), ZAt(a, lda, j, j), lda);
      ZPotrf2Rec<R>(false, jb, ZAt(a, lda, j, j), lda, info, j);
      if (j + jb < n) {
        ZgemmFull<R>(0, 2, n - j - jb, jb, j, m1, ZAt(a, lda, j + jb, 0), lda,
                     ZAt(a, lda, j, 0), lda, one, ZAt(a, lda, j + jb, j), lda);
        ZtrsmFull<R>(false, true, 2, false, n - j - jb, jb, one, ZAt(a, lda, j, j), lda,
                     ZAt(a, lda, j + jb, j), lda);
      }
    }
  }
  ctx.guard = saved;
}
template void ZPotrf<double>(bool, bool, int, double*, int, int*);
template void ZPotrf<float>(bool, bool, int, float*, int, int*);

template <typename R>
void ZPotrs(bool upper, int n, int nrhs, const R* a, int lda, R* b, int ldb) {
  if (n == 0 || nrhs == 0) return;
  const R one[2] = {R(1), R(0)};
  if (upper) {
    ZtrsmFull<R>(true, false, 2, false, n, nrhs, one, a, lda, b, ldb);
    ZtrsmFull<R>(true, false, 0, false, n, nrhs, one, a, lda, b, ldb);
  } else {
    ZtrsmFull<R>(true, true, 0, false, n, nrhs, one, a, lda, b, ldb);
    ZtrsmFull<R>(true, true, 2, false, n, nrhs, one, a, lda, b, ldb);
  }
}
template void ZPotrs<double>(bool, int, int, const double*, int, double*, int);
template void ZPotrs<float>(bool, int, int, const float*, int, float*, int);


}  // namespace hb
