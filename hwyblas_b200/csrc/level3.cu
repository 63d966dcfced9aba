// Level-3 routines around the GEMM kernels: the FP32 GEMM (FFMA on the CUDA
// cores, the reference's FP32 order with KC = 384), the recursive TRSM with
// its base substitution kernel, SYRK, and the reference-semantics wrappers
// (argument-independent quick returns and alpha scaling).
#include <algorithm>
#include <cstdio>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

// ---------------------------------------------------------------------------
// FP32 GEMM: 64 x 64 tile per 256-thread CTA, 4 x 4 outputs per thread, each
// a sequential FFMA chain over k restarted every 384 (src/gemm_kernel-inl.h:72).
constexpr int kSB = 64, kSK = 16;

// `part` restricts C to one triangle (SYRK): elements outside it are neither
// computed nor written; inside, the chain is the one of the full GEMM.
__device__ __forceinline__ bool InPart(int part, int i, int j) {
  return part == kAll || (part == kLower ? i >= j : i <= j);
}

// Whether C(i, j) lies in a micro-tile of the reference's AVX-512 float
// kernel (MR 32, NR 12, MC 128, NC 4080) that crosses the diagonal: those
// tiles merge as alpha*acc + beta*C with two roundings (src/gemm-inl.h:93-130;
// src/gemm_kernel-inl.h:64-74).
__device__ __forceinline__ bool InCrossingTileF(int part, int m, int n, int i, int j) {
  constexpr int MR = 32, NR = 12, MC = 128, NC = 4080;
  const int ic = i / MC * MC, mcb = min(MC, m - ic);
  const int ir = (i - ic) / MR * MR, mr = min(MR, mcb - ir);
  const int jc = j / NC * NC, ncb = min(NC, n - jc);
  const int jr = (j - jc) / NR * NR, nr = min(NR, ncb - jr);
  const int i0 = ic + ir, j0 = jc + jr;
  if (part == kLower) return !(i0 > j0 + nr - 1);
  return !(i0 + mr - 1 < j0);
}

// k range [*kb, *ke) the reference multiplies for C(i, j) when an operand is
// triangular: NonZeroRange of the AVX-512 float micro-tile (MR 32, NR 12,
// MC 128, NC 4080) holding C(i, j) (src/gemm-inl.h:62-85). Row tiles start at
// multiples of 32 (MC is a multiple of MR), column tiles at multiples of 12
// within NC blocks.
__device__ __forceinline__ void TriRangeF(int tri, int m, int n, int k, int i, int j, int* kb,
                                          int* ke) {
  *kb = 0;
  *ke = k;
  if (tri == kTriALower || tri == kTriAUpper) {
    const int i0 = i & ~31, mr = min(32, m - i0);
    if (tri == kTriALower) *ke = min(k, i0 + mr);
    else *kb = i0;
  } else if (tri == kTriBLower || tri == kTriBUpper) {
    constexpr int NR = 12, NC = 4080;
    const int jc = j / NC * NC, jr = (j - jc) / NR * NR;
    const int nr = min(NR, min(NC, n - jc) - jr);
    if (tri == kTriBLower) *kb = jc + jr;
    else *ke = min(k, jc + jr + nr);
  }
}

// `tri` (TRMM): each element's chain runs over its micro-tile's k range only,
// and a chunk outside that range leaves the element unmerged, as the
// reference skips the micro-tile (src/gemm-inl.h:202-209).
__global__ void __launch_bounds__(256)
    SgemmKernel(int m, int n, int k, float alpha, View<float> a, View<float> b,
                float beta, float* c, long long ldc, int part, int tri,
                const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ float sa[kSK][kSB + 4];
  __shared__ float sb[kSK][kSB + 4];
  const int m0 = blockIdx.x * kSB, n0 = blockIdx.y * kSB;
  // A tile wholly outside the triangle has nothing to do.
  if ((part == kLower && m0 + kSB - 1 < n0) || (part == kUpper && m0 > n0 + kSB - 1)) return;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  float acc[4][4] = {}, cacc[4][4] = {};
  const int kchunk = 384;
  // Row- and column-dependent bounds of the elements' k ranges (tri).
  int rkb[4], rke[4], ckb[4], cke[4];
  const int tri_a = (tri == kTriALower || tri == kTriAUpper) ? tri : kTriNone;
  const int tri_b = (tri == kTriBLower || tri == kTriBUpper) ? tri : kTriNone;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    TriRangeF(tri_a, m, n, k, m0 + tx + 16 * r, 0, &rkb[r], &rke[r]);
    TriRangeF(tri_b, m, n, k, 0, n0 + ty + 16 * r, &ckb[r], &cke[r]);
  }
  for (int k0 = 0; k0 < k; k0 += kSK) {
    for (int idx = threadIdx.x; idx < kSK * kSB; idx += 256) {
      const int kk = idx / kSB, mm = idx % kSB;
      const int gi = m0 + mm, gk = k0 + kk;
      sa[kk][mm] = (gi < m && gk < k) ? a.data[gi * a.rs + gk * a.cs] : 0.f;
      const int gj = n0 + mm;
      sb[kk][mm] = (gj < n && gk < k) ? b.data[gk * b.rs + gj * b.cs] : 0.f;
    }
    __syncthreads();
    const int kend = min(kSK, k - k0);
    for (int kk = 0; kk < kend; ++kk) {
      float av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = sa[kk][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = sb[kk][ty + 16 * q];
      const int kg = k0 + kk;
      if (tri == kTriNone) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[r][q] = fmaf(av[r], bv[q], acc[r][q]);
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (kg >= max(rkb[r], ckb[q]) && kg < min(rke[r], cke[q]))
              acc[r][q] = fmaf(av[r], bv[q], acc[r][q]);
      }
      if ((kg + 1) % kchunk == 0 || kg + 1 == k) {
        const bool first = kg < kchunk;
        const int c_lo = kg / kchunk * kchunk, c_hi = kg + 1;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int i = m0 + tx + 16 * r, j = n0 + ty + 16 * q;
            const float rr = alpha * acc[r][q];
            if (!first && tri != kTriNone &&
                max(max(rkb[r], ckb[q]), c_lo) >= min(min(rke[r], cke[q]), c_hi)) {
              // Outside the element's k range: not merged.
            } else if (first) {
              if (i < m && j < n && InPart(part, i, j)) {
                if (beta == 0.f) {
                  cacc[r][q] = rr;
                } else {
                  const float cin = c[i + j * ldc];
                  if (beta == 1.f) {
                    cacc[r][q] = rr + cin;
                  } else if (part != kAll && InCrossingTileF(part, m, n, i, j)) {
                    const float bc = beta * cin;
                    cacc[r][q] = rr + bc;
                  } else {
                    cacc[r][q] = fmaf(cin, beta, rr);
                  }
                }
              }
            } else {
              cacc[r][q] = rr + cacc[r][q];
            }
            acc[r][q] = 0.f;
          }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = m0 + tx + 16 * r, j = n0 + ty + 16 * q;
      if (i < m && j < n && InPart(part, i, j)) c[i + j * ldc] = cacc[r][q];
    }
}

// ---------------------------------------------------------------------------
// TRSM base: solves X*T = B for independent rows of X (src/trsm-inl.h:107-174)
// with T (r x r, r <= 32) read from a strided view. Columns are solved in
// "solve order" s = 0..r-1 (column r-1-s for lower, s for upper), two per
// pass: b_j0 -= x_q t(q, j0) and b_j1 -= x_q t(q, j1) as fma(-x_q, t, b) for
// every solved q; x_j0 = b_j0 * (1/t(j0, j0)); b_j1 = fma(-x_j0, t(j0, j1), b_j1);
// x_j1 = b_j1 * (1/t(j1, j1)). One thread owns one row of X; the row is kept
// in registers indexed in solve order so all register indices are static.
// Element (row, col q) of X is x[row * xs_row + q * xs_col].
template <typename T>
__global__ void __launch_bounds__(128)
    TrsmBaseKernel(View<T> tri, int lower, int unit, int r, int rows, T* x,
                   long long xs_row, long long xs_col, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ T st[32][33];  // st[s][u] = T(col(s), col(u)) in solve order
  __shared__ T sinv[32];
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int s = idx / 32, u = idx % 32;
    T v = T(0);
    if (s < r && u < r) {
      const int q = lower ? r - 1 - s : s, j = lower ? r - 1 - u : u;
      // Only the triangle's solved-before part (s < u) and the diagonal are
      // referenced.
      if (s < u || (s == u && !unit)) v = tri.data[q * tri.rs + j * tri.cs];
    }
    st[s][u] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int s = threadIdx.x;
    sinv[s] = (s < r && !unit) ? T(1) / st[s][s] : T(1);
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  T* xr = x + row * xs_row;
  T y[32];
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) y[s] = xr[(lower ? r - 1 - s : s) * xs_col];
  }
#pragma unroll
  for (int step = 0; step + 1 < 32; step += 2) {
    if (step + 2 <= r) {
      T acc0 = y[step], acc1 = y[step + 1];
#pragma unroll
      for (int s = 0; s < step; ++s) {
        acc0 = fma(-y[s], st[s][step], acc0);
        acc1 = fma(-y[s], st[s][step + 1], acc1);
      }
      if (!unit) acc0 = acc0 * sinv[step];
      y[step] = acc0;
      acc1 = fma(-acc0, st[step][step + 1], acc1);
      if (!unit) acc1 = acc1 * sinv[step + 1];
      y[step + 1] = acc1;
    } else if (step < r) {  // odd r: the last column alone
      T acc = y[step];
#pragma unroll
      for (int s = 0; s < step; ++s) acc = fma(-y[s], st[s][step], acc);
      if (!unit) acc = acc * sinv[step];
      y[step] = acc;
    }
  }
  if (r == 32) {
    // step 30/31 handled above; nothing left.
  }
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) xr[(lower ? r - 1 - s : s) * xs_col] = y[s];
  }
}

template <typename T>
void LaunchGemm(int m, int n, int k, T alpha, View<T> a, View<T> b, T beta,
                T* c, int ldc);
template <>
void LaunchGemm<double>(int m, int n, int k, double alpha, View<double> a,
                        View<double> b, double beta, double* c, int ldc) {
  Dgemm(m, n, k, alpha, a, b, beta, c, ldc, kAll);
}
template <>
void LaunchGemm<float>(int m, int n, int k, float alpha, View<float> a,
                       View<float> b, float beta, float* c, int ldc) {
  Sgemm(m, n, k, alpha, a, b, beta, c, ldc, kAll);
}

// TrsmRecursive (src/trsm.cc:87-135): split at max(32, (r/2)/32*32).
template <typename T>
void TrsmRec(bool left, View<T> tri, bool lower, bool unit, int r, int other,
             T* b, int ldb) {
  if (r <= 32) {
    TrsmSolve<T>(left, tri, lower, unit, r, other, b, ldb);
    return;
  }
  const int r1 = std::max(32, (r / 2) / 32 * 32);
  const int r2 = r - r1;
  const View<T> t11 = tri;
  const View<T> t22 = tri.sub(r1, r1);
  const View<T> toff = lower ? tri.sub(r1, 0) : tri.sub(0, r1);
  const auto cm = [&](T* p) { return ColMajor<T>(p, ldb); };
  if (left) {
    T* b1 = b;
    T* b2 = b + r1;
    if (lower) {
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
      LaunchGemm<T>(r2, other, r1, T(-1), toff, cm(b1), T(1), b2, ldb);
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
    } else {
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
      LaunchGemm<T>(r1, other, r2, T(-1), toff, cm(b2), T(1), b1, ldb);
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
    }
  } else {
    T* b1 = b;
    T* b2 = b + static_cast<long long>(r1) * ldb;
    if (lower) {
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
      LaunchGemm<T>(other, r1, r2, T(-1), cm(b2), toff, T(1), b1, ldb);
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
    } else {
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
      LaunchGemm<T>(other, r2, r1, T(-1), cm(b1), toff, T(1), b2, ldb);
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
    }
  }
}

}  // namespace

void Sgemm(int m, int n, int k, float alpha, View<float> a, View<float> b,
           float beta, float* c, int ldc, Part part, Tri tri) {
  const dim3 grid((m + kSB - 1) / kSB, (n + kSB - 1) / kSB);
  SgemmKernel<<<grid, 256, 0, Ctx().stream>>>(m, n, k, alpha, a, b, beta, c, ldc,
                                              static_cast<int>(part),
                                              static_cast<int>(tri), Ctx().guard);
  CountLaunch();
  LaunchFailed("sgemm");
}

template <typename T>
void TrsmSolve(bool left, View<T> tri, bool lower, bool unit, int r, int other,
               T* b, int ldb) {
  if (r <= 0 || other <= 0) return;
  View<T> t = tri;
  bool lo = lower;
  long long xs_row, xs_col;
  if (left) {
    // T X = B  <=>  X^T T^T = B^T (src/trsm-inl.h:306-324): rows of X^T are
    // the columns of B.
    t.rs = tri.cs;
    t.cs = tri.rs;
    lo = !lower;
    xs_row = ldb;
    xs_col = 1;
  } else {
    xs_row = 1;
    xs_col = ldb;
  }
  const int threads = 128;
  TrsmBaseKernel<T><<<(other + threads - 1) / threads, threads, 0,
                      Ctx().stream>>>(t, lo ? 1 : 0, unit ? 1 : 0, r, other, b,
                                      xs_row, xs_col, Ctx().guard);
  CountLaunch();
  LaunchFailed("trsm base");
}
template void TrsmSolve<double>(bool, View<double>, bool, bool, int, int,
                                double*, int);
template void TrsmSolve<float>(bool, View<float>, bool, bool, int, int, float*,
                               int);

// Trsm (src/trsm.cc:137-180) after argument checks: B := alpha*B first
// (alpha != 1), zero B and return for alpha == 0, then the recursion on
// op(A) (strides swapped and triangle flipped when transposed).
template <typename T>
void TrsmFull(bool left, bool lower, bool trans, bool unit, int m, int n,
              T alpha, const T* a, int lda, T* b, int ldb) {
  if (m == 0 || n == 0) return;
  if (alpha != T(1)) ScaleMatrix<T>(m, n, alpha, b, ldb, kAll);
  if (alpha == T(0)) return;
  const View<T> tri = ColMajor<T>(a, lda, trans);
  const bool op_lower = trans ? !lower : lower;
  TrsmRec<T>(left, tri, op_lower, unit, left ? m : n, left ? n : m, b, ldb);
}
template void TrsmFull<double>(bool, bool, bool, bool, int, int, double,
                               const double*, int, double*, int);
template void TrsmFull<float>(bool, bool, bool, bool, int, int, float,
                              const float*, int, float*, int);

// Syrk (src/level3.cc:84-139; ssyrk_/dsyrk_ 410-421), real: C :=
// alpha*op(A)*op(A)^T + beta*C on one triangle, as a GEMM with a triangular C
// part (DMMA for double, the FP32 kernel for float).
template <typename T>
void SyrkFull(bool lower, bool trans, int n, int k, T alpha, const T* a, int lda, T beta,
              T* c, int ldc) {
  const Part part = lower ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return;
  }
  if constexpr (sizeof(T) == 8) {
    Dgemm(n, n, k, alpha, ColMajor<T>(a, lda, trans), ColMajor<T>(a, lda, !trans), beta, c,
          ldc, part);
  } else {
    Sgemm(n, n, k, alpha, ColMajor<T>(a, lda, trans), ColMajor<T>(a, lda, !trans), beta, c,
          ldc, part);
  }
}
template void SyrkFull<double>(bool, bool, int, int, double, const double*, int, double,
                               double*, int);
template void SyrkFull<float>(bool, bool, int, int, float, const float*, int, float, float*,
                              int);

namespace {

// A GEMM problem on the triangle `part` of C (DMMA for double, FP32 FFMA for
// float), with the reference's merge rules for tiles crossing the diagonal.
template <typename T>
void GemmPart(int m, int n, int k, T alpha, View<T> a, View<T> b, T beta, T* c, int ldc,
              Part part, Tri tri = kTriNone) {
  if constexpr (sizeof(T) == 8) {
    Dgemm(m, n, k, alpha, a, b, beta, c, ldc, part, tri);
  } else {
    Sgemm(m, n, k, alpha, a, b, beta, c, ldc, part, tri);
  }
}

// out (n x n, leading dimension ldo) := the symmetric matrix whose `lower`
// (or upper) triangle is stored in a; the other triangle of a is not read.
template <typename T>
__global__ void SymmetrizeFullKernel(int n, const T* a, long long lda, bool lower, T* out,
                                     long long ldo) {
  const long long total = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    const bool stored = lower ? i >= j : i <= j;
    out[i + j * ldo] = stored ? a[i + j * lda] : a[j + i * lda];
  }
}

// out (n x n) := the triangle `lower` of a with explicit zeros in the other
// one and ones on the diagonal when `unit` (the values the reference packs for
// a triangular operand, src/pack-inl.h:99-160); the rest of a is not read.
template <typename T>
__global__ void TriangleFullKernel(int n, const T* a, long long lda, bool lower, bool unit,
                                   T* out, long long ldo) {
  const long long total = static_cast<long long>(n) * n;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    T v = T(0);
    if (i == j) v = unit ? T(1) : a[i + j * lda];
    else if (lower ? i > j : i < j) v = a[i + j * lda];
    out[i + j * ldo] = v;
  }
}

int GridFor(long long total) {
  return static_cast<int>(std::min<long long>((total + 255) / 256, 8192));
}

}  // namespace

// SYMM: the reference packs the stored triangle mirrored (Structure::
// kSymmetric, src/pack-inl.h:99-160), i.e. the values of the full symmetric
// matrix; here that matrix is formed once and the plain GEMM runs on it, so
// every element's chain is the GEMM's (src/level3.cc:26-82).
template <typename T>
void SymmFull(bool left, bool lower, int m, int n, T alpha, const T* a, int lda, const T* b,
              int ldb, T beta, T* c, int ldc) {
  if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return;
  if (alpha == T(0)) {
    ScaleMatrix<T>(m, n, beta, c, ldc, kAll);
    return;
  }
  const int ka = left ? m : n;
  T* full = static_cast<T*>(Workspace(kWsLevel3, sizeof(T) * static_cast<size_t>(ka) * ka));
  if (full == nullptr) return;
  SymmetrizeFullKernel<T><<<GridFor(static_cast<long long>(ka) * ka), 256, 0, Ctx().stream>>>(
      ka, a, lda, lower, full, ka);
  CountLaunch();
  if (LaunchFailed("symm symmetrize")) return;
  const View<T> sym = ColMajor<T>(full, ka), gen = ColMajor<T>(b, ldb);
  GemmPart<T>(m, n, ka, alpha, left ? sym : gen, left ? gen : sym, beta, c, ldc, kAll);
}
template void SymmFull<double>(bool, bool, int, int, double, const double*, int,
                               const double*, int, double, double*, int);
template void SymmFull<float>(bool, bool, int, int, float, const float*, int, const float*,
                              int, float, float*, int);

// SYR2K: alpha op(A) op(B)^T + beta C, then + alpha op(B) op(A)^T (beta 1),
// each a GEMM problem on the uplo triangle (src/level3.cc:153-221).
template <typename T>
void Syr2kFull(bool lower, bool trans, int n, int k, T alpha, const T* a, int lda,
               const T* b, int ldb, T beta, T* c, int ldc) {
  const Part part = lower ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return;
  }
  GemmPart<T>(n, n, k, alpha, ColMajor<T>(a, lda, trans), ColMajor<T>(b, ldb, !trans), beta,
              c, ldc, part);
  GemmPart<T>(n, n, k, alpha, ColMajor<T>(b, ldb, trans), ColMajor<T>(a, lda, !trans), T(1),
              c, ldc, part);
}
template void Syr2kFull<double>(bool, bool, int, int, double, const double*, int,
                                const double*, int, double, double*, int);
template void Syr2kFull<float>(bool, bool, int, int, float, const float*, int, const float*,
                               int, float, float*, int);

// GEMMTR: op(A) (n x k) op(B) (k x n) on the uplo triangle of C
// (src/level3.cc:226-280).
template <typename T>
void GemmtrFull(bool lower, bool ta, bool tb, int n, int k, T alpha, const T* a, int lda,
                const T* b, int ldb, T beta, T* c, int ldc) {
  const Part part = lower ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return;
  }
  GemmPart<T>(n, n, k, alpha, ColMajor<T>(a, lda, ta), ColMajor<T>(b, ldb, tb), beta, c, ldc,
              part);
}
template void GemmtrFull<double>(bool, bool, bool, int, int, double, const double*, int,
                                 const double*, int, double, double*, int);
template void GemmtrFull<float>(bool, bool, bool, int, int, float, const float*, int,
                                const float*, int, float, float*, int);

// TRMM: B := alpha op(A) B (left) or alpha B op(A), computed from a copy of B
// with beta 0 (src/level3.cc:284-342). The triangle is stored out with its
// zeros and unit diagonal, and the GEMM multiplies only the k range of each
// reference micro-tile, so every element is the reference's chain.
template <typename T>
void TrmmFull(bool left, bool lower, bool trans, bool unit, int m, int n, T alpha,
              const T* a, int lda, T* b, int ldb) {
  if (m == 0 || n == 0) return;
  if (alpha == T(0)) {
    ScaleMatrix<T>(m, n, T(0), b, ldb, kAll);
    return;
  }
  const int ka = left ? m : n;
  T* tri = static_cast<T*>(Workspace(kWsLevel3, sizeof(T) * static_cast<size_t>(ka) * ka));
  if (tri == nullptr) return;
  TriangleFullKernel<T><<<GridFor(static_cast<long long>(ka) * ka), 256, 0, Ctx().stream>>>(
      ka, a, lda, lower, unit, tri, ka);
  CountLaunch();
  if (LaunchFailed("trmm triangle")) return;
  TrmmDense<T>(left, lower, trans, m, n, alpha, tri, ka, b, ldb);
}

// TRMM on a triangle already stored dense (zeros and unit diagonal written
// out), from a copy of B.
template <typename T>
void TrmmDense(bool left, bool lower, bool trans, int m, int n, T alpha, const T* tri, int ldt,
               T* b, int ldb) {
  if (m == 0 || n == 0) return;
  const int ka = left ? m : n;
  T* copy = static_cast<T*>(Workspace(kWsLevel3Copy, sizeof(T) * static_cast<size_t>(m) * n));
  if (copy == nullptr) return;
  if (Failed(cudaMemcpy2DAsync(copy, sizeof(T) * m, b, sizeof(T) * ldb, sizeof(T) * m, n,
                               cudaMemcpyDeviceToDevice, Ctx().stream),
             "trmm copy"))
    return;
  // op(A) is lower exactly when A is lower and not transposed, or upper and
  // transposed (src/api.h:133-140).
  const bool op_lower = (lower != trans);
  const View<T> t = ColMajor<T>(tri, ldt, trans), g = ColMajor<T>(copy, m);
  if (left) {
    GemmPart<T>(m, n, ka, alpha, t, g, T(0), b, ldb, kAll, op_lower ? kTriALower : kTriAUpper);
  } else {
    GemmPart<T>(m, n, ka, alpha, g, t, T(0), b, ldb, kAll, op_lower ? kTriBLower : kTriBUpper);
  }
}
template void TrmmDense<double>(bool, bool, bool, int, int, double, const double*, int,
                                double*, int);
template void TrmmDense<float>(bool, bool, bool, int, int, float, const float*, int, float*,
                               int);
template void TrmmFull<double>(bool, bool, bool, bool, int, int, double, const double*, int,
                               double*, int);
template void TrmmFull<float>(bool, bool, bool, bool, int, int, float, const float*, int,
                              float*, int);

// Gemm (src/gemm.cc:114-131) after argument checks.
template <typename T>
void GemmFull(bool ta, bool tb, int m, int n, int k, T alpha, const T* a,
              int lda, const T* b, int ldb, T beta, T* c, int ldc) {
  if (m == 0 || n == 0) return;
  if ((k == 0 || alpha == T(0)) && beta == T(1)) return;
  if (k == 0 || alpha == T(0)) {
    ScaleMatrix<T>(m, n, beta, c, ldc, kAll);
    return;
  }
  LaunchGemm<T>(m, n, k, alpha, ColMajor<T>(a, lda, ta), ColMajor<T>(b, ldb, tb),
                beta, c, ldc);
}
template void GemmFull<double>(bool, bool, int, int, int, double,
                               const double*, int, const double*, int, double,
                               double*, int);
template void GemmFull<float>(bool, bool, int, int, int, float, const float*,
                              int, const float*, int, float, float*, int);

}  // namespace hb
