// Mixed-precision linear solvers: dgesv / dposv whose factorization spends
// its flops on the INT8 tensor cores, with FP64 iterative refinement.
//
// The reference has no mixed-precision solver (README.md:81: ?sgesv/?sposv
// are not ported); the driver follows LAPACK's DSGESV / DSPOSV: factor in
// reduced precision, solve, then iterate r = b - A x (FP64), d = solve(r),
// x += d until every column satisfies DSGESV's backward criterion
// ||r||_inf <= ||x||_inf * ||A||_inf * eps * sqrt(n) and its correction has
// settled (see Refine), at most 30 times; if that fails (or the
// reduced-precision factorization breaks down), factor and solve in FP64 with
// the plain path (the reference's own dgetrf/dpotrf order). ITER and IPIV
// follow DSGESV: ITER >= 0 is the number of refinement steps, ITER < 0 means
// the FP64 path ran (-2 non-finite A, -3 factorization breakdown, -31 no
// convergence).
//
// The residual of the refinement is extra-precise (double-double accumulation
// of exactly split products, rounded once), so x converges to the solution of
// A x = b to about the last bit rather than to the FP64 residual's
// cond(A) eps.
//
// Factorization (right-looking, block nb):
//   LU        panel (pivot search, diagonal block, in-panel updates) in
//             FP64; the inverse of the panel's unit L11 in FP64; then
//             U12 = L11^-1 A12 and the trailing update A22 -= L21 U12 as
//             Ozaki GEMMs with few INT8 slices on tcgen05 (integer-exact
//             products, FP64 recombination).
//   Cholesky  diagonal block factored and inverted in FP64, L21 = A21 L11^-T
//             and A22 -= L21 L21^T (lower triangle) as Ozaki GEMMs.
// The factors stay in FP64 storage; their accuracy is that of the slices
// (about 8*S - 1 significant bits), which sets the refinement's contraction.
//
// Refinement solves: the diagonal 64 x 64 blocks of the factors are inverted
// once; each triangular solve is then one cooperative kernel per group of
// 16-column chains of right-hand sides in which each solved 64-row block is
// published through a flag and consumed by the CTAs owning later blocks
// (ChainTrsvKernel); above kChainSlots blocks per CTA, a kernel with a grid
// barrier per block (BlockTrsvKernel).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

constexpr int kTb = 64;         // diagonal block of the refinement solves
constexpr int kTrsvRhs = 64;    // right-hand sides per solve launch
constexpr int kTrsvThreads = 256;
constexpr int kResRows = 128;   // residual GEMV: rows per CTA
constexpr int kResK = 256;      // residual GEMV: k per CTA
constexpr int kResRhs = 16;     // residual GEMV: right-hand sides per launch
constexpr int kItMax = 30;      // LAPACK's ITERMAX (dsgesv.f)

template <typename T>
T* At(T* a, long long lda, long long i, long long j) {
  return a + i + j * lda;
}

// ||A||_inf partial row sums: CTA (bx, by) sums |a_ij| over columns
// [by*256, by*256 + 256) for its 256 rows.
__global__ void RowAbsPartialKernel(int n, const double* a, long long lda,
                                    double* part) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const int j0 = blockIdx.y * 256, j1 = min(n, j0 + 256);
  double s = 0.0;
  for (int j = j0; j < j1; ++j) s += fabs(a[i + j * lda]);
  part[static_cast<long long>(blockIdx.y) * n + i] = s;
}

// Max over rows of the row sums; NaN dominates (its bit pattern is above
// +Inf's as an unsigned integer).
__global__ void RowAbsFinishKernel(int n, int parts, const double* part,
                                   unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (i < n) {
    for (int c = 0; c < parts; ++c) s += part[static_cast<long long>(c) * n + i];
  }
  unsigned long long bits = __double_as_longlong(s);
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, bits, off);
    bits = o > bits ? o : bits;
  }
  if (threadIdx.x % 32 == 0) atomicMax(out, bits);
}

// Column-wise max |x_iq| for q < nrhs (bits of a non-negative double).
__global__ void ColAbsMaxKernel(int n, int nrhs, const double* x, long long ldx,
                                unsigned long long* out) {
  const int q = blockIdx.y;
  unsigned long long bits = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    const unsigned long long b = __double_as_longlong(fabs(x[i + q * ldx]));
    bits = b > bits ? b : bits;
  }
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xffffffffu, bits, off);
    bits = o > bits ? o : bits;
  }
  if (threadIdx.x % 32 == 0) atomicMax(out + q, bits);
}

// Residual with extra precision (few right-hand sides at a time): every
// product a(i, k) x(k, q) is split exactly into p = fl(a x) and
// e = fma(a, x, -p); the p are summed in double-double (TwoSum, Knuth) and the
// e in FP64, per chunk of kResK columns. part_hi / part_lo are [c][q][i].
// R right-hand sides per instantiation (1, 2, 4, 8 or 16; nrhs <= R), so
// that a few right-hand sides do not issue the arithmetic of sixteen.
template <int R>
__global__ void __launch_bounds__(kResRows)
    ResidualDdPartialKernel(int n, int nrhs, const double* a, long long lda,
                            const double* x, long long ldx, double* part_hi,
                            double* part_lo) {
  __shared__ double sx[R][kResK];
  const int k0 = blockIdx.y * kResK, kc = min(kResK, n - k0);
  for (int idx = threadIdx.x; idx < R * kResK; idx += kResRows) {
    const int q = idx / kResK, k = idx % kResK;
    sx[q][k] = (q < nrhs && k < kc) ? x[k0 + k + q * ldx] : 0.0;
  }
  __syncthreads();
  const int i = blockIdx.x * kResRows + threadIdx.x;
  if (i >= n) return;
  double hi[R], lo[R];
#pragma unroll
  for (int q = 0; q < R; ++q) hi[q] = lo[q] = 0.0;
  const double* ai = a + i + static_cast<long long>(k0) * lda;
  for (int k = 0; k < kc; ++k) {
    const double v = ai[static_cast<long long>(k) * lda];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      // Columns q >= nrhs multiply zeros: their sums stay zero and are not
      // stored.
      const double p = v * sx[q][k];
      const double pe = fma(v, sx[q][k], -p);
      const double s = hi[q] + p;
      const double bb = s - hi[q];
      const double e = (hi[q] - (s - bb)) + (p - bb);
      hi[q] = s;
      lo[q] += e + pe;
    }
  }
  const long long off = static_cast<long long>(blockIdx.y) * nrhs * n;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    if (q < nrhs) {
      part_hi[off + static_cast<long long>(q) * n + i] = hi[q];
      part_lo[off + static_cast<long long>(q) * n + i] = lo[q];
    }
  }
}

// r(i, q) = b(i, q) - sum of the chunks (in chunk order), in double-double,
// rounded once.
__global__ void ResidualDdFinishKernel(int n, int nrhs, int chunks,
                                       const double* part_hi, const double* part_lo,
                                       const double* b, long long ldb, double* r,
                                       long long ldr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  if (i >= n || q >= nrhs) return;
  double hi = b[i + q * ldb], lo = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const long long at = (static_cast<long long>(c) * nrhs + q) * n + i;
    const double p = -part_hi[at];
    const double s = hi + p;
    const double bb = s - hi;
    const double e = (hi - (s - bb)) + (p - bb);
    hi = s;
    lo += e - part_lo[at];
  }
  r[i + q * ldr] = hi + lo;
}

__global__ void AxpyMatrixKernel(int n, int nrhs, const double* d, long long ldd,
                                 double* x, long long ldx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  if (i < n && q < nrhs) x[i + q * ldx] += d[i + q * ldd];
}

// dst(i, q) = src(perm[i], q).
__global__ void GatherRowsKernel(int n, int nrhs, const int* perm, const double* src,
                                 long long lds, double* dst, long long ldd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  if (i < n && q < nrhs) dst[i + q * ldd] = src[perm[i] + q * lds];
}

// The row permutation of LAPACK pivots: applying the interchanges i <->
// ipiv[i] - 1 in order to the identity gives perm, and P b = b[perm]. The
// interchanges are sequential: one thread replays them, on perm and ipiv
// staged in shared memory when n <= kPermSmem, else in place in global
// memory.
constexpr int kPermSmem = 24576;
__global__ void PermFromPivotsKernel(int n, const int* ipiv, int* perm) {
  extern __shared__ int sm[];
  const bool staged = n <= kPermSmem;
  int* sp = staged ? sm : perm;
  int* sv = staged ? sm + n : nullptr;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sp[i] = i;
    if (staged) sv[i] = ipiv[i] - 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) {
      int p = staged ? sv[i] : ipiv[i] - 1;
      if (p < 0 || p >= n) p = i;  // never out of bounds
      const int t = sp[i];
      sp[i] = sp[p];
      sp[p] = t;
    }
  }
  __syncthreads();
  if (staged)
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = sp[i];
}

// Full symmetric matrix from one triangle: dst(i, j) = src(i, j) on the
// referenced side and src(j, i) on the other. 32 x 32 tiles through shared
// memory so that both the direct and the mirrored reads are coalesced.
__global__ void SymmetrizeKernel(int n, int upper, const double* src,
                                 long long lds, double* dst, long long ldd) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  // Mirrored source tile (j0.., i0..) read along its rows.
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int si = j0 + threadIdx.x, sj = i0 + r;
    if (si < n && sj < n) tile[r][threadIdx.x] = src[si + static_cast<long long>(sj) * lds];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + r;
    if (i >= n || j >= n) continue;
    const bool referenced = upper ? (i <= j) : (i >= j);
    dst[i + static_cast<long long>(j) * ldd] =
        referenced ? src[i + static_cast<long long>(j) * lds] : tile[threadIdx.x][r];
  }
}

// Inverses of the diagonal kTb x kTb blocks of a triangular factor stored in
// w: inv[b] (column-major kTb x kTb, zero outside the triangle). Thread c
// computes column c by substitution against e_c.
__global__ void __launch_bounds__(kTb)
    InvertDiagBlocksKernel(int n, const double* w, long long ldw, int lower,
                           int unit, double* inv) {
  extern __shared__ double inv_smem[];  // t, then y: [kTb][kTb + 1] each
  double(*t)[kTb + 1] = reinterpret_cast<double(*)[kTb + 1]>(inv_smem);
  double(*y)[kTb + 1] = reinterpret_cast<double(*)[kTb + 1]>(inv_smem + kTb * (kTb + 1));
  const int b = blockIdx.x, r0 = b * kTb, bs = min(kTb, n - r0);
  const int c = threadIdx.x;
  for (int r = 0; r < kTb; ++r)
    t[r][c] = (r < bs && c < bs) ? w[(r0 + r) + static_cast<long long>(r0 + c) * ldw] : 0.0;
  __syncthreads();
  if (c < bs) {
    if (lower) {
      for (int r = 0; r < c; ++r) y[r][c] = 0.0;
      y[c][c] = unit ? 1.0 : 1.0 / t[c][c];
      for (int r = c + 1; r < bs; ++r) {
        double s = 0.0;
        for (int q = c; q < r; ++q) s = fma(t[r][q], y[q][c], s);
        y[r][c] = unit ? -s : -s / t[r][r];
      }
    } else {
      for (int r = c + 1; r < bs; ++r) y[r][c] = 0.0;
      y[c][c] = unit ? 1.0 : 1.0 / t[c][c];
      for (int r = c - 1; r >= 0; --r) {
        double s = 0.0;
        for (int q = r + 1; q <= c; ++q) s = fma(t[r][q], y[q][c], s);
        y[r][c] = unit ? -s : -s / t[r][r];
      }
    }
  }
  __syncthreads();
  double* out = inv + static_cast<long long>(b) * kTb * kTb;
  for (int r = 0; r < kTb; ++r)
    out[r + c * kTb] = (r < bs && c < bs) ? y[r][c] : 0.0;
}

// Triangular solve T x = x in place for nrhs <= kTrsvRhs columns of x, with
// T the lower (forward) or upper (backward) triangle of w and inv the
// inverses of its diagonal blocks. Cooperative: all CTAs are resident; each
// step solves one block row redundantly in every CTA (x_b = inv_b * x_b from
// shared memory; CTA 0 stores it) and then updates the CTA's share of the
// remaining rows, one row per thread with the block row's 64 factor entries
// in registers; a grid barrier ends the step. x is read and written through
// L2 only (.cg), since rows change owner between steps.
constexpr int kLd = kTb + 1;  // padded column stride of the shared blocks
constexpr int kTrsvSmem = (kTb * kLd + 2 * kLd * kTrsvRhs) * 8;
template <bool kLower>
__global__ void __launch_bounds__(kTrsvThreads)
    BlockTrsvKernel(int n, int nrhs, const double* w, long long ldw,
                    const double* inv, double* x, long long ldx,
                    unsigned int* barrier, int* timeout_flag) {
  extern __shared__ double trsv_smem[];
  double* si = trsv_smem;              // inv block: si[r + c * kLd]
  double* sb = si + kTb * kLd;         // sb[q * kLd + r]
  double* sx = sb + kLd * kTrsvRhs;    // sx[q * kLd + r]
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane >> 2, t = lane & 3;
  const int nbl = (nrhs + 7) / 8;
  const int nblk = (n + kTb - 1) / kTb;
  unsigned int gen = 0;
  for (int step = 0; step < nblk; ++step) {
    const int blk = kLower ? step : nblk - 1 - step;
    const int r0 = blk * kTb, bs = min(kTb, n - r0);
    const double* ib = inv + static_cast<long long>(blk) * kTb * kTb;
    for (int idx = threadIdx.x; idx < kTb * kTb; idx += kTrsvThreads)
      si[(idx % kTb) + (idx / kTb) * kLd] = ib[idx];
    for (int idx = threadIdx.x; idx < kTb * nbl * 8; idx += kTrsvThreads) {
      const int r = idx % kTb, q = idx / kTb;
      sb[q * kLd + r] = (r < bs && q < nrhs) ? __ldcg(x + r0 + r + q * ldx) : 0.0;
    }
    __syncthreads();
    if (nrhs >= 8) {
      // x_b = inv_b * b_b on the FP64 tensor pipe: warp w computes 16-row
      // block w % 4 for the 8-column blocks w / 4, w / 4 + 2, ...
      const int mb = warp % 4;
      for (int nb = warp / 4; nb < nbl; nb += kTrsvThreads / 128) {
        double d[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int kk = 0; kk < kTb / 8; ++kk) {
          const int c0 = kk * 8 + t;
          const double a0 = si[(mb * 16 + g) + c0 * kLd];
          const double a1 = si[(mb * 16 + g + 8) + c0 * kLd];
          const double a2 = si[(mb * 16 + g) + (c0 + 4) * kLd];
          const double a3 = si[(mb * 16 + g + 8) + (c0 + 4) * kLd];
          const double b0 = sb[(nb * 8 + g) * kLd + c0];
          const double b1 = sb[(nb * 8 + g) * kLd + c0 + 4];
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
              "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
              : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
              : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
        }
        const int q0 = nb * 8 + 2 * t, row0 = mb * 16 + g;
        sx[q0 * kLd + row0] = d[0];
        sx[(q0 + 1) * kLd + row0] = d[1];
        sx[q0 * kLd + row0 + 8] = d[2];
        sx[(q0 + 1) * kLd + row0 + 8] = d[3];
      }
    } else {
      for (int idx = threadIdx.x; idx < kTb * nrhs; idx += kTrsvThreads) {
        const int r = idx % kTb, q = idx / kTb;
        const double* bq = sb + q * kLd;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
        for (int c = 0; c < kTb; c += 2) {
          s0 = fma(si[r + c * kLd], bq[c], s0);
          s1 = fma(si[r + (c + 1) * kLd], bq[c + 1], s1);
        }
        sx[q * kLd + r] = s0 + s1;
      }
    }
    __syncthreads();
    if (blockIdx.x == 0) {
      for (int idx = threadIdx.x; idx < kTb * nrhs; idx += kTrsvThreads) {
        const int r = idx % kTb, q = idx / kTb;
        if (r < bs) __stcg(x + r0 + r + q * ldx, sx[q * kLd + r]);
      }
    }
    const int lo = kLower ? r0 + bs : 0, hi = kLower ? n : r0;
    if (nrhs >= 8) {
      // Many right-hand sides: the update is a (rows x 64) x (64 x nrhs)
      // product; each warp takes 16-row blocks on the FP64 tensor pipe
      // (m16n8k8: A from the factor, B from the solved block in shared
      // memory).
      const int nwarps = kTrsvThreads / 32;
      for (int rb = lo + 16 * (blockIdx.x * nwarps + warp); rb < hi;
           rb += 16 * gridDim.x * nwarps) {
        const int i0 = rb + g, i1 = rb + g + 8;
        const double* w0 = w + i0 + static_cast<long long>(r0) * ldw;
        const double* w1 = w + i1 + static_cast<long long>(r0) * ldw;
        double af[kTb / 8][4];
#pragma unroll
        for (int kk = 0; kk < kTb / 8; ++kk) {
          const int c0 = kk * 8 + t, c1 = c0 + 4;
          af[kk][0] = (i0 < hi && c0 < bs) ? w0[static_cast<long long>(c0) * ldw] : 0.0;
          af[kk][1] = (i1 < hi && c0 < bs) ? w1[static_cast<long long>(c0) * ldw] : 0.0;
          af[kk][2] = (i0 < hi && c1 < bs) ? w0[static_cast<long long>(c1) * ldw] : 0.0;
          af[kk][3] = (i1 < hi && c1 < bs) ? w1[static_cast<long long>(c1) * ldw] : 0.0;
        }
        // All products first, then all loads of x, then all stores: the
        // read-modify-writes must not wait on one another.
        double d[kTrsvRhs / 8][4];
#pragma unroll
        for (int nb = 0; nb < kTrsvRhs / 8; ++nb) d[nb][0] = d[nb][1] = d[nb][2] = d[nb][3] = 0.0;
        // k outer, column blocks inner: consecutive MMAs are independent.
#pragma unroll
        for (int kk = 0; kk < kTb / 8; ++kk) {
#pragma unroll
          for (int nb = 0; nb < kTrsvRhs / 8; ++nb) {
            if (nb >= nbl) continue;
            const int qb = nb * 8 + g;  // this lane's B column
            const double b0 = sx[qb * kLd + kk * 8 + t];
            const double b1 = sx[qb * kLd + kk * 8 + t + 4];
            asm volatile(
                "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                : "+d"(d[nb][0]), "+d"(d[nb][1]), "+d"(d[nb][2]), "+d"(d[nb][3])
                : "d"(af[kk][0]), "d"(af[kk][1]), "d"(af[kk][2]), "d"(af[kk][3]),
                  "d"(b0), "d"(b1));
          }
        }
        double xv[kTrsvRhs / 8][4];
#pragma unroll
        for (int nb = 0; nb < kTrsvRhs / 8; ++nb) {
          const int q0 = nb * 8 + 2 * t, q1 = q0 + 1;
          xv[nb][0] = (i0 < hi && q0 < nrhs) ? __ldcg(x + i0 + q0 * ldx) : 0.0;
          xv[nb][1] = (i0 < hi && q1 < nrhs) ? __ldcg(x + i0 + q1 * ldx) : 0.0;
          xv[nb][2] = (i1 < hi && q0 < nrhs) ? __ldcg(x + i1 + q0 * ldx) : 0.0;
          xv[nb][3] = (i1 < hi && q1 < nrhs) ? __ldcg(x + i1 + q1 * ldx) : 0.0;
        }
#pragma unroll
        for (int nb = 0; nb < kTrsvRhs / 8; ++nb) {
          const int q0 = nb * 8 + 2 * t, q1 = q0 + 1;
          if (i0 < hi && q0 < nrhs) __stcg(x + i0 + q0 * ldx, xv[nb][0] - d[nb][0]);
          if (i0 < hi && q1 < nrhs) __stcg(x + i0 + q1 * ldx, xv[nb][1] - d[nb][1]);
          if (i1 < hi && q0 < nrhs) __stcg(x + i1 + q0 * ldx, xv[nb][2] - d[nb][2]);
          if (i1 < hi && q1 < nrhs) __stcg(x + i1 + q1 * ldx, xv[nb][3] - d[nb][3]);
        }
      }
      if (!GridBarrier(barrier, gridDim.x, ++gen, timeout_flag)) return;
      continue;
    }
    for (int i = lo + blockIdx.x * kTrsvThreads + threadIdx.x; i < hi;
         i += gridDim.x * kTrsvThreads) {
      const double* wi = w + i + static_cast<long long>(r0) * ldw;
      double l[kTb];
#pragma unroll
      for (int c = 0; c < kTb; ++c)
        l[c] = c < bs ? wi[static_cast<long long>(c) * ldw] : 0.0;
      for (int q = 0; q < nrhs; ++q) {
        const double* xq = sx + q * kLd;
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int c = 0; c < kTb; c += 2) {
          a0 = fma(l[c], xq[c], a0);
          a1 = fma(l[c + 1], xq[c + 1], a1);
        }
        double* xi = x + i + q * ldx;
        __stcg(xi, __ldcg(xi) - (a0 + a1));
      }
    }
    if (!GridBarrier(barrier, gridDim.x, ++gen, timeout_flag)) return;
  }
}

// Triangular solve without grid barriers: x := T^{-1} x in 16-column chains
// of right-hand sides, one group of CTAs per chain. Block position p (solve
// order: block p for the lower triangle, nblk-1-p for the upper) is owned by
// one CTA of the chain, in zigzag order (round r = p / P, CTA p % P for even
// r and P-1 - p % P for odd r, which evens out the row blocks' unequal
// work). A CTA keeps the partial right-hand sides of its blocks in shared
// memory and sweeps the positions in order: once x_p is published (a flag
// per position), it subtracts T_ip x_p from each of its blocks i after p.
// The owner of p+1 does that block first and finishes it at once,
// x_{p+1} = inv_{p+1} * acc, and publishes it before its other blocks: the
// critical path is one 64 x 64 product, one inverse product and one flag
// per block. Factor tiles and inverse blocks stream through a 4-stage
// cp.async ring in the order the sweeps consume them, independent of x (the
// depth matters: 3 stages left the critical tiles waiting on HBM).
constexpr int kCw = 16;           // right-hand sides per chain
constexpr int kChainLd = kTb + 4; // padded stride: conflict-free fragments
constexpr int kChainSlots = 8;    // row blocks per CTA at most
constexpr int kChainStages = 4;
constexpr int kChainThreads = 256;
constexpr int kChainTile = kTb * kChainLd;  // doubles per staged tile
constexpr int kChainVec = kCw * kChainLd;   // doubles per 64 x 16 block
constexpr int kChainSmem =
    (kChainStages * kChainTile + (kChainSlots + 2) * kChainVec) * 8;

struct ChainOwn {
  int c, P, owned, nblk;
  __device__ int Pos(int s) const { return s * P + ((s & 1) ? P - 1 - c : c); }
  __device__ bool Owns(int p) const {
    const int r = p / P, j = p % P;
    return ((r & 1) ? P - 1 - j : j) == c;
  }
};

// Walks the items of a CTA in consumption order: sweep -1 holds the inverse
// of position 0 (its owner only); sweep p >= 0 holds, for each own slot s
// with Pos(s) > p in order, the tile (s, p) and, when Pos(s) == p + 1, the
// inverse of slot s right after it.
struct ChainCursor {
  int p = -1, s = 0, sf = 0, phase = 0;
  // kind: 0 tile, 1 inverse; false at the end.
  __device__ bool Next(const ChainOwn& o, int& kind, int& slot, int& sweep) {
    while (true) {
      if (p < 0) {
        if (phase == 0 && o.owned > 0 && o.Pos(0) == 0) {
          phase = 1;
          kind = 1, slot = 0, sweep = -1;
          return true;
        }
        p = 0, phase = 0;
        while (sf < o.owned && o.Pos(sf) <= p) ++sf;
        s = sf;
        continue;
      }
      if (p > o.nblk - 2) return false;
      if (s >= o.owned) {
        ++p, phase = 0;
        while (sf < o.owned && o.Pos(sf) <= p) ++sf;
        s = sf;
        continue;
      }
      sweep = p, slot = s;
      if (phase == 0) {
        kind = 0;
        if (o.Pos(s) == p + 1) phase = 1; else ++s;
      } else {
        kind = 1, phase = 0, ++s;
      }
      return true;
    }
  }
};

// One m16n8k8 FP64 product chain over k = 0..63: d += A(16 x 64) B(64 x 8),
// A column-major with stride kChainLd starting at row `row`, B stored by
// column (b[col * kChainLd + k]).
__device__ __forceinline__ void ChainMma(const double* a, int row, const double* b,
                                         int g, int t, double d[4]) {
#pragma unroll
  for (int kk = 0; kk < kTb / 8; ++kk) {
    const int c0 = kk * 8 + t;
    const double a0 = a[c0 * kChainLd + row + g];
    const double a1 = a[c0 * kChainLd + row + g + 8];
    const double a2 = a[(c0 + 4) * kChainLd + row + g];
    const double a3 = a[(c0 + 4) * kChainLd + row + g + 8];
    const double b0 = b[g * kChainLd + c0];
    const double b1 = b[g * kChainLd + c0 + 4];
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
  }
}

template <bool kLower>
__global__ void __launch_bounds__(kChainThreads, 1)
    ChainTrsvKernel(int n, int nrhs, const double* w, long long ldw, const double* inv,
                    double* x, long long ldx, int P, unsigned int* flags,
                    unsigned int epoch, int* timeout_flag) {
  extern __shared__ __align__(16) double chain_smem[];
  double* stage = chain_smem;                        // kChainStages tiles
  double* acc = stage + kChainStages * kChainTile;   // kChainSlots blocks
  double* xs = acc + kChainSlots * kChainVec;        // 2 blocks
  __shared__ int s_ok;
  const int nblk = (n + kTb - 1) / kTb;
  const int chain = blockIdx.x / P;
  const int q0 = chain * kCw;
  if (q0 >= nrhs) return;
  const int ncols = min(kCw, nrhs - q0);
  const int nbl = (ncols + 7) / 8;
  ChainOwn own;
  own.c = blockIdx.x % P, own.P = P, own.nblk = nblk;
  own.owned = 0;
  while (own.owned < kChainSlots && own.Pos(own.owned) < nblk) ++own.owned;
  if (own.owned == 0) return;
  unsigned int* cflags = flags + static_cast<long long>(chain) * nblk;
  double* xc = x + static_cast<long long>(q0) * ldx;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, t = lane & 3;
  const int rg = warp & 3, nb = warp >> 2;  // 16-row group, 8-column block
  auto blk = [&](int p) { return kLower ? p : nblk - 1 - p; };

  // Partial right-hand sides of the own blocks: b restricted to their rows.
  for (int s = 0; s < own.owned; ++s) {
    const int r0 = blk(own.Pos(s)) * kTb, bs = min(kTb, n - r0);
    for (int idx = tid; idx < kTb * kCw; idx += kChainThreads) {
      const int r = idx % kTb, q = idx / kTb;
      acc[s * kChainVec + q * kChainLd + r] =
          (r < bs && q < ncols) ? xc[r0 + r + static_cast<long long>(q) * ldx] : 0.0;
    }
  }

  // Stages one item: tile (rows of slot s, columns of position p) or the
  // inverse block of slot s, zero-filled outside the matrix.
  auto issue = [&](int kind, int slot, int sweep, double* dst) {
    const double* src;
    long long ld;
    int rows, cols;
    if (kind == 0) {
      const int ri = blk(own.Pos(slot)) * kTb, ci = blk(sweep) * kTb;
      src = w + ri + static_cast<long long>(ci) * ldw;
      ld = ldw, rows = min(kTb, n - ri), cols = min(kTb, n - ci);
    } else {
      src = inv + static_cast<long long>(blk(own.Pos(slot))) * kTb * kTb;
      ld = kTb, rows = kTb, cols = kTb;
    }
#pragma unroll
    for (int j = 0; j < kTb * kTb / 2 / kChainThreads; ++j) {
      const int idx = tid + j * kChainThreads;
      const int col = idx / (kTb / 2), row = (idx % (kTb / 2)) * 2;
      const int bytes = col < cols ? max(0, min(2, rows - row)) * 8 : 0;
      CpAsync16(dst + col * kChainLd + row, bytes > 0 ? src + row + col * ld : w, bytes);
    }
  };

  ChainCursor fetch, use;
  int fk, fs, fp;
#pragma unroll
  for (int i = 0; i < kChainStages - 1; ++i) {
    if (fetch.Next(own, fk, fs, fp)) issue(fk, fs, fp, stage + i * kChainTile);
    CpAsyncCommit();
  }
  int item = 0, cur_sweep = -2;
  int kind, slot, sweep;
  while (use.Next(own, kind, slot, sweep)) {
    if (sweep != cur_sweep) {
      cur_sweep = sweep;
      if (sweep >= 0 && !own.Owns(sweep)) {
        // Wait for x at this position, then bring it into shared memory.
        if (tid == 0) {
          uint32_t polls = 0;
          int good = 1;
          while (true) {
            unsigned int v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                         : "=r"(v)
                         : "l"(cflags + sweep)
                         : "memory");
            if (v == epoch) break;
            if ((++polls & 255u) == 0 &&
                (*reinterpret_cast<volatile int*>(timeout_flag) != 0 || polls >= kMaxPolls)) {
              atomicExch(timeout_flag, 1);
              good = 0;
              break;
            }
          }
          s_ok = good;
        }
        __syncthreads();
        if (!s_ok) break;  // timed out: the host reports it
        const int r0 = blk(sweep) * kTb, bs = min(kTb, n - r0);
        double* xd = xs + (sweep & 1) * kChainVec;
        for (int idx = tid; idx < kTb * kCw; idx += kChainThreads) {
          const int r = idx % kTb, q = idx / kTb;
          xd[q * kChainLd + r] =
              (r < bs && q < ncols) ? __ldcg(xc + r0 + r + static_cast<long long>(q) * ldx)
                                    : 0.0;
        }
      }
    }
    CpAsyncWait<kChainStages - 2>();
    __syncthreads();
    // Refill the stage consumed one item ago.
    if (fetch.Next(own, fk, fs, fp))
      issue(fk, fs, fp, stage + ((item + kChainStages - 1) % kChainStages) * kChainTile);
    CpAsyncCommit();
    const double* tile = stage + (item % kChainStages) * kChainTile;
    double* as = acc + slot * kChainVec;
    if (kind == 0) {
      // acc_s -= T(rows of s, columns of sweep) * x_sweep
      if (nb < nbl) {
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        ChainMma(tile, rg * 16, xs + (sweep & 1) * kChainVec + nb * 8 * kChainLd, g, t, d);
        const int row = rg * 16 + g, q = nb * 8 + 2 * t;
        as[q * kChainLd + row] -= d[0];
        as[(q + 1) * kChainLd + row] -= d[1];
        as[q * kChainLd + row + 8] -= d[2];
        as[(q + 1) * kChainLd + row + 8] -= d[3];
      }
    } else {
      // x at position sweep + 1 (this slot): inv * acc_s, kept and published.
      const int pos = sweep + 1;
      const int r0 = blk(pos) * kTb, bs = min(kTb, n - r0);
      double* xd = xs + (pos & 1) * kChainVec;
      if (nb < nbl) {
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        ChainMma(tile, rg * 16, as + nb * 8 * kChainLd, g, t, d);
        const int row = rg * 16 + g, q = nb * 8 + 2 * t;
        const double v[4] = {d[0], d[1], d[2], d[3]};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int rr = row + (e >> 1) * 8, qq = q + (e & 1);
          xd[qq * kChainLd + rr] = v[e];
          if (rr < bs && qq < ncols) xc[r0 + rr + static_cast<long long>(qq) * ldx] = v[e];
        }
      }
      // The barrier orders every thread's stores of x before thread 0's
      // release at GPU scope, which makes them visible to the acquirer.
      __syncthreads();
      if (tid == 0)
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(cflags + pos), "r"(epoch)
                     : "memory");
    }
    ++item;
  }
  CpAsyncWait<0>();
}

// Buffers of one mixed solve (device pointers into the thread's workspace).
struct MixedBuffers {
  double* w = nullptr;      // n x n factor, leading dimension ldw
  long long ldw = 0;
  double* afull = nullptr;  // dposv: the full symmetric A (leading dimension ldw)
  double* inv_lo = nullptr; // inverses of the diagonal blocks of L and U
  double* inv_up = nullptr;
  double* r = nullptr;      // n x nrhs residual
  double* d = nullptr;      // n x nrhs correction
  long long ldr = 0;        // of r and d
  double* part = nullptr;   // residual and norm partial sums
  int* perm = nullptr;      // LU row permutation
  unsigned long long* norms = nullptr;  // [0] ||A||, then ||x||, ||r|| columns
  unsigned int* barrier = nullptr;  // [0]: grid barrier; [32]: Cholesky arrivals
  unsigned int* flags = nullptr;  // per-position ready flags of the chained solve
  size_t flag_stride = 0;         // flags of a second, concurrent chained solve
};

long long Round(long long v, long long m) { return (v + m - 1) / m * m; }

bool AllocBuffers(int n, int nrhs, bool sym, MixedBuffers* bf) {
  bf->ldw = Round(std::max(n, 1), 32);
  const size_t wbytes = sizeof(double) * static_cast<size_t>(bf->ldw) * n;
  bf->w = static_cast<double*>(Workspace(kWsMixed, wbytes));
  if (bf->w == nullptr) return false;
  if (sym) {
    bf->afull = static_cast<double*>(Workspace(kWsMixed2, wbytes));
    if (bf->afull == nullptr) return false;
  }
  const size_t nblk = (n + kTb - 1) / kTb;
  bf->ldr = bf->ldw;
  const size_t chunks = (n + kResK - 1) / kResK;
  const size_t rowparts = (n + 255) / 256;
  const size_t inv_elems = nblk * kTb * kTb;
  const size_t r_elems = static_cast<size_t>(bf->ldr) * nrhs;
  const size_t part_elems =
      std::max(2 * chunks * std::min(nrhs, kResRhs) * n, rowparts * n);
  const size_t norm_elems = 1 + 3 * static_cast<size_t>(nrhs);
  // Chained solves launch at most num_sms / ceil(nblk / kChainSlots) chains
  // of nblk flags, which is at most max(nblk, kChainSlots * num_sms); the
  // factorization runs two at once (one a stream).
  bf->flag_stride = Round(
      std::max<size_t>(nblk, static_cast<size_t>(kChainSlots) * Ctx().num_sms) + 64, 64);
  const size_t flag_elems = 2 * bf->flag_stride;
  const size_t total = sizeof(double) * (2 * inv_elems + 2 * r_elems + part_elems) +
                       sizeof(int) * Round(n, 64) +
                       sizeof(unsigned long long) * (norm_elems + 8) +
                       sizeof(unsigned int) * flag_elems + 4096;
  uint8_t* base = static_cast<uint8_t*>(Workspace(kWsMixed3, total));
  if (base == nullptr) return false;
  double* d = reinterpret_cast<double*>(base);
  bf->inv_lo = d;
  bf->inv_up = d + inv_elems;
  bf->r = d + 2 * inv_elems;
  bf->d = bf->r + r_elems;
  bf->part = bf->d + r_elems;
  bf->perm = reinterpret_cast<int*>(bf->part + part_elems);
  bf->norms = reinterpret_cast<unsigned long long*>(bf->perm + Round(n, 64));
  bf->barrier = reinterpret_cast<unsigned int*>(bf->norms + norm_elems + 8);
  bf->flags = bf->barrier + 64;
  return true;
}

double BitsToDouble(unsigned long long b) {
  double v;
  std::memcpy(&v, &b, sizeof v);
  return v;
}

void Copy2D(int m, int n, const double* src, long long lds, double* dst,
            long long ldd) {
  if (m <= 0 || n <= 0) return;
  Failed(cudaMemcpy2DAsync(dst, sizeof(double) * ldd, src, sizeof(double) * lds,
                           sizeof(double) * m, n, cudaMemcpyDeviceToDevice,
                           Ctx().stream),
         "mixed copy");
}

// ||A||_inf of an n x n matrix (host value; waits for the stream).
double InfNorm(int n, const double* a, long long lda, MixedBuffers& bf) {
  cudaStream_t st = Ctx().stream;
  const int rowparts = (n + 255) / 256;
  cudaMemsetAsync(bf.norms, 0, sizeof(unsigned long long), st);
  RowAbsPartialKernel<<<dim3(rowparts, rowparts), 256, 0, st>>>(n, a, lda, bf.part);
  RowAbsFinishKernel<<<rowparts, 256, 0, st>>>(n, rowparts, bf.part, bf.norms);
  CountLaunch(2);
  LaunchFailed("mixed norm");
  unsigned long long bits = 0;
  cudaMemcpyAsync(&bits, bf.norms, sizeof bits, cudaMemcpyDeviceToHost, st);
  if (Failed(cudaStreamSynchronize(st), "mixed norm")) return NAN;
  return BitsToDouble(bits);
}

// r := b - A x in FP64 through the DMMA GEMM (the refinement's first phase
// for 16 or more right-hand sides).
void Residual(int n, int nrhs, const double* a, long long lda, const double* b,
              long long ldb, const double* x, long long ldx, MixedBuffers& bf) {
  Copy2D(n, nrhs, b, ldb, bf.r, bf.ldr);
  Dgemm(n, nrhs, n, -1.0, ColMajor(a, lda), ColMajor(x, ldx), 1.0, bf.r,
        static_cast<int>(bf.ldr), kAll);
}

}  // namespace

// r := b - A x with extra precision: each entry is the exact value up to a
// relative error of about n eps^2 |A| |x| / |r|, then rounded once. Groups of
// kResRhs right-hand sides; `part` holds 2 chunks kResRhs n doubles.
void ResidualDd(int n, int nrhs, const double* a, long long lda, const double* b,
                long long ldb, const double* x, long long ldx, double* r, long long ldr,
                double* part) {
  cudaStream_t st = Ctx().stream;
  const int chunks = (n + kResK - 1) / kResK;
  for (int q0 = 0; q0 < nrhs; q0 += kResRhs) {
    const int g = std::min(kResRhs, nrhs - q0);
    double* ph = part;
    double* pl = part + static_cast<size_t>(chunks) * g * n;
    const dim3 grid((n + kResRows - 1) / kResRows, chunks);
    const double* xq = x + q0 * ldx;
    if (g == 1) {
      ResidualDdPartialKernel<1><<<grid, kResRows, 0, st>>>(n, g, a, lda, xq, ldx, ph, pl);
    } else if (g == 2) {
      ResidualDdPartialKernel<2><<<grid, kResRows, 0, st>>>(n, g, a, lda, xq, ldx, ph, pl);
    } else if (g <= 4) {
      ResidualDdPartialKernel<4><<<grid, kResRows, 0, st>>>(n, g, a, lda, xq, ldx, ph, pl);
    } else if (g <= 8) {
      ResidualDdPartialKernel<8><<<grid, kResRows, 0, st>>>(n, g, a, lda, xq, ldx, ph, pl);
    } else {
      ResidualDdPartialKernel<16><<<grid, kResRows, 0, st>>>(n, g, a, lda, xq, ldx, ph, pl);
    }
    ResidualDdFinishKernel<<<dim3((n + 255) / 256, g), 256, 0, st>>>(
        n, g, chunks, ph, pl, b + q0 * ldb, ldb, r + q0 * ldr, ldr);
    CountLaunch(2);
    if (LaunchFailed("extra-precise residual")) return;
  }
}

size_t ResidualDdPartBytes(int n, int nrhs) {
  const size_t chunks = (n + kResK - 1) / kResK;
  return sizeof(double) * 2 * chunks * std::min(nrhs, kResRhs) * static_cast<size_t>(n);
}

namespace {

// Column max-norms of `count` n x nrhs matrices into host arrays (waits for
// the stream); norms[c][q] = max_i |m_c(i, q)|.
bool ColumnNorms(int n, int nrhs, int count, const double* const* mats,
                 const long long* lds, MixedBuffers& bf,
                 std::vector<std::vector<double>>* norms) {
  cudaStream_t st = Ctx().stream;
  unsigned long long* dn = bf.norms + 1;
  cudaMemsetAsync(dn, 0, sizeof(unsigned long long) * count * nrhs, st);
  const int blocks = std::min(64, (n + 255) / 256);
  for (int c = 0; c < count; ++c) {
    ColAbsMaxKernel<<<dim3(blocks, nrhs), 256, 0, st>>>(n, nrhs, mats[c], lds[c],
                                                        dn + c * nrhs);
  }
  CountLaunch(count);
  LaunchFailed("mixed column norms");
  std::vector<unsigned long long> bits(static_cast<size_t>(count) * nrhs);
  cudaMemcpyAsync(bits.data(), dn, sizeof(unsigned long long) * bits.size(),
                  cudaMemcpyDeviceToHost, st);
  if (Failed(cudaStreamSynchronize(st), "mixed column norms")) return false;
  norms->assign(count, std::vector<double>(nrhs));
  for (int c = 0; c < count; ++c)
    for (int q = 0; q < nrhs; ++q) (*norms)[c][q] = BitsToDouble(bits[c * nrhs + q]);
  return true;
}

void InvertDiagBlocks(int n, const double* w, long long ldw, bool lower, bool unit,
                      double* inv) {
  const int nblk = (n + kTb - 1) / kTb;
  const int smem = 2 * kTb * (kTb + 1) * static_cast<int>(sizeof(double));
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(InvertDiagBlocksKernel,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  InvertDiagBlocksKernel<<<nblk, kTb, smem, Ctx().stream>>>(n, w, ldw, lower ? 1 : 0,
                                                            unit ? 1 : 0, inv);
  CountLaunch();
  LaunchFailed("mixed diagonal inverses");
}

void PermFromPivots(int n, const int* ipiv, int* perm) {
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(PermFromPivotsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         2 * kPermSmem * static_cast<int>(sizeof(int)));
    configured = true;
  }
  const size_t smem = n <= kPermSmem ? 2 * sizeof(int) * n : 0;
  PermFromPivotsKernel<<<1, 1024, smem, Ctx().stream>>>(n, ipiv, perm);
  CountLaunch();
  LaunchFailed("mixed permutation");
}

// Chained solve (ChainTrsvKernel) of x := T^{-1} x; false when the row
// blocks do not fit the CTAs' slots (n above kChainSlots * 64 * resident
// CTAs), in which case nothing was launched.
bool ChainTrsv(bool lower, int n, int nrhs, const double* w, long long ldw,
               const double* inv, double* x, long long ldx, unsigned int* flags) {
  Context& ctx = Ctx();
  static int capacity = -1;
  if (capacity < 0) {
    cudaFuncSetAttribute(ChainTrsvKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kChainSmem);
    cudaFuncSetAttribute(ChainTrsvKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kChainSmem);
    int lo = 0, up = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lo, ChainTrsvKernel<true>, kChainThreads,
                                                  kChainSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up, ChainTrsvKernel<false>, kChainThreads,
                                                  kChainSmem);
    capacity = ctx.num_sms * std::min(lo, up);
    cudaGetLastError();
  }
  const int nblk = (n + kTb - 1) / kTb;
  const int pmin = (nblk + kChainSlots - 1) / kChainSlots;
  if (capacity <= 0 || pmin > capacity) return false;
  const int chains = (nrhs + kCw - 1) / kCw;
  const int per_launch = std::max(1, std::min(chains, capacity / pmin));
  int nn = n;
  long long lw = ldw, lx = ldx;
  int* tflag = ctx.dev_status;
  unsigned int epoch = 1;
  const void* fn = lower ? reinterpret_cast<const void*>(ChainTrsvKernel<true>)
                         : reinterpret_cast<const void*>(ChainTrsvKernel<false>);
  for (int c0 = 0; c0 < chains; c0 += per_launch) {
    const int nc = std::min(per_launch, chains - c0);
    int P = std::min(nblk, capacity / nc);
    int nr = std::min(nrhs - c0 * kCw, nc * kCw);
    double* xq = x + static_cast<long long>(c0) * kCw * ldx;
    cudaMemsetAsync(flags, 0, sizeof(unsigned int) * nblk * nc, ctx.stream);
    void* args[] = {&nn, &nr, const_cast<double**>(&w), &lw, const_cast<double**>(&inv),
                    &xq, &lx, &P, &flags, &epoch, &tflag};
    Failed(cudaLaunchCooperativeKernel(fn, nc * P, kChainThreads, args, kChainSmem,
                                       ctx.stream),
           "mixed triangular solve");
    CountLaunch();
  }
  return true;
}

// x := T^{-1} x for the lower or upper triangle of w.
void BlockTrsv(bool lower, int n, int nrhs, const double* w, long long ldw,
               const double* inv, double* x, long long ldx, unsigned int* barrier,
               unsigned int* flags) {
  if (ChainTrsv(lower, n, nrhs, w, ldw, inv, x, ldx, flags)) return;
  Context& ctx = Ctx();
  static int grid = 0;
  if (grid == 0) {
    cudaFuncSetAttribute(BlockTrsvKernel<true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTrsvSmem);
    cudaFuncSetAttribute(BlockTrsvKernel<false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kTrsvSmem);
    int lo = 0, up = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lo, BlockTrsvKernel<true>,
                                                  kTrsvThreads, kTrsvSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&up, BlockTrsvKernel<false>,
                                                  kTrsvThreads, kTrsvSmem);
    grid = ctx.num_sms * std::max(1, std::min({lo, up, 2}));
  }
  int nn = n;
  long long lw = ldw, lx = ldx;
  int* flag = ctx.dev_status;
  const void* fn = lower ? reinterpret_cast<const void*>(BlockTrsvKernel<true>)
                         : reinterpret_cast<const void*>(BlockTrsvKernel<false>);
  for (int q0 = 0; q0 < nrhs; q0 += kTrsvRhs) {
    int nr = std::min(kTrsvRhs, nrhs - q0);
    double* xq = x + static_cast<long long>(q0) * ldx;
    cudaMemsetAsync(barrier, 0, sizeof(unsigned int), ctx.stream);
    void* args[] = {&nn, &nr, const_cast<double**>(&w), &lw,
                    const_cast<double**>(&inv), &xq, &lx, &barrier, &flag};
    Failed(cudaLaunchCooperativeKernel(fn, grid, kTrsvThreads, args, kTrsvSmem,
                                       ctx.stream),
           "mixed triangular solve");
    CountLaunch();
  }
}

// dst := A^{-1} src with the mixed factors (LU: P, unit L, U; Cholesky: L,
// and L^T mirrored into the upper triangle of w).
void MixedSolve(bool lu, int n, int nrhs, MixedBuffers& bf, const double* src,
                long long lds, double* dst, long long ldd) {
  if (lu) {
    GatherRowsKernel<<<dim3((n + 255) / 256, nrhs), 256, 0, Ctx().stream>>>(
        n, nrhs, bf.perm, src, lds, dst, ldd);
    CountLaunch();
    LaunchFailed("mixed gather");
  } else {
    Copy2D(n, nrhs, src, lds, dst, ldd);
  }
  BlockTrsv(true, n, nrhs, bf.w, bf.ldw, bf.inv_lo, dst, ldd, bf.barrier, bf.flags);
  BlockTrsv(false, n, nrhs, bf.w, bf.ldw, bf.inv_up, dst, ldd, bf.barrier, bf.flags);
}

// Panel width: wide enough that the trailing updates amortize their
// slicing and epilogue (measured at n = 16384: 1024 beats 512 by ~5 %).
int MixedBlock(int n) { return n >= 8192 ? 1024 : (n >= 4096 ? 512 : 256); }


// A high-priority stream of the calling thread for the look-ahead panel
// work, and two events to order it against the context's stream.
__global__ void SetIdentityKernel(int n, double* x, long long ldx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < n) x[i + j * ldx] = (i == j) ? 1.0 : 0.0;
}

struct Lookahead {
  cudaStream_t stream = nullptr;
  cudaEvent_t to_look = nullptr, to_main = nullptr;
  bool ok = false;
};
Lookahead& GetLookahead() {
  static thread_local Lookahead la;
  if (!la.ok) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    la.ok = cudaStreamCreateWithPriority(&la.stream, cudaStreamNonBlocking, greatest) ==
                cudaSuccess &&
            cudaEventCreateWithFlags(&la.to_look, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&la.to_main, cudaEventDisableTiming) == cudaSuccess;
    if (!la.ok) cudaGetLastError();
  }
  return la;
}

// Runs f with the context's stream switched to s.
template <typename F>
void OnStream(cudaStream_t s, F f) {
  Context& ctx = Ctx();
  const cudaStream_t saved = ctx.stream;
  ctx.stream = s;
  f();
  ctx.stream = saved;
}

// Right-looking LU of w with FP64 panels and Ozaki trailing updates, with a
// look-ahead of one panel: on a high-priority stream, the pivots of panel j
// are applied to the columns of panel j+1, which are updated and factored,
// while the context's stream applies them to all other columns and updates
// the rest of the trailing matrix. The two touch disjoint columns; each
// waits for the other where one reads what the other writes (panel j+1's
// columns need the previous trailing update finished, the rest needs the
// adjusted pivots).
void MixedGetrf(int n, double* w, long long ldw, int* ipiv, int* info, int slices,
                MixedBuffers& bf) {
  Context& ctx = Ctx();
  const int nb = MixedBlock(n);
  const int lw = static_cast<int>(ldw);
  const cudaStream_t main = ctx.stream;
  Lookahead& la = GetLookahead();
  const cudaStream_t look = la.ok ? la.stream : main;
  auto signal = [&](cudaEvent_t ev, cudaStream_t from, cudaStream_t to) {
    if (from == to) return;
    cudaEventRecord(ev, from);
    cudaStreamWaitEvent(to, ev, 0);
  };
  // Inverses of the 64 x 64 diagonal blocks of panel j's unit L11, in one
  // of two buffers by panel parity (look writes panel j+1's while main may
  // still read panel j's).
  const auto l11_inv = [&](int j) { return ((j / nb) & 1) ? bf.inv_up : bf.inv_lo; };
  // The inverse of panel j's unit lower diagonal block L11 (nb x nb, in one
  // of two buffers by panel parity), formed in FP64 by the chained solve of
  // L11 X = I with the inverted 64 x 64 diagonal blocks.
  double* xinv = static_cast<double*>(
      Workspace(kWsMixedInv, sizeof(double) * 2 * static_cast<size_t>(nb) * nb));
  if (xinv == nullptr) return;
  const auto l11_full_inv = [&](int j) { return xinv + ((j / nb) & 1) * static_cast<size_t>(nb) * nb; };
  const auto invert = [&](int j, int jb) {
    if (j + jb >= n) return;
    InvertDiagBlocks(jb, At(w, ldw, j, j), ldw, true, true, l11_inv(j));
    double* x = l11_full_inv(j);
    SetIdentityKernel<<<dim3((jb + 255) / 256, jb), 256, 0, Ctx().stream>>>(jb, x, nb);
    CountLaunch();
    if (!ChainTrsv(true, jb, jb, At(w, ldw, j, j), ldw, l11_inv(j), x, nb,
                   bf.flags + bf.flag_stride))
      TrsmFull<double>(true, true, false, true, jb, jb, 1.0, At(w, ldw, j, j), lw, x, nb);
  };
  const auto update = [&](int j, int jb, int c0, int nc, int ws_set) {
    // Columns [c0, c0 + nc) of the trailing matrix, both products on the
    // INT8 tensor cores: U12 = L11^{-1} A12 (in place: the slicing reads A12
    // before the product writes it), then A22 -= L21 U12.
    const int rest = n - j - jb;
    DgemmEmulated(jb, nc, jb, 1.0, ColMajor<double>(l11_full_inv(j), nb),
                  ColMajor<double>(At(w, ldw, j, c0), ldw), 0.0, At(w, ldw, j, c0), lw,
                  slices, false, ws_set);
    DgemmEmulated(rest, nc, jb, -1.0, ColMajor<double>(At(w, ldw, j + jb, j), ldw),
                  ColMajor<double>(At(w, ldw, j, c0), ldw), 1.0, At(w, ldw, j + jb, c0), lw,
                  slices, false, ws_set);
  };
  signal(la.to_look, main, look);
  OnStream(look, [&] {
    const int jb0 = std::min(nb, n);
    MixedPanel(n, jb0, w, lw, ipiv, info, 0);
    invert(0, jb0);
  });
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    const int rest = n - j - jb;
    const int next = std::min(nb, rest);
    // Panel j is factored (on look). Once main's previous trailing update is
    // done, look applies the panel's interchanges to the next panel's
    // columns, updates and factors them; main applies them to the columns
    // left of the panel and to the rest of the trailing matrix, then updates
    // the rest. The two streams touch disjoint columns.
    signal(la.to_look, main, look);
    OnStream(look, [&] {
      if (j > 0) AdjustPivots(ipiv, j, j + jb, j);
    });
    signal(la.to_main, look, main);
    if (rest > 0) {
      OnStream(look, [&] {
        Laswp<double>(next, At(w, ldw, 0, j + jb), lw, j + 1, j + jb, ipiv, 1);
        update(j, jb, j + jb, next, 1);
        MixedPanel(rest, next, At(w, ldw, j + jb, j + jb), lw, ipiv + j + jb, info, j + jb);
        invert(j + jb, next);
      });
    }
    OnStream(main, [&] {
      if (j > 0) Laswp<double>(j, w, lw, j + 1, j + jb, ipiv, 1);
      if (rest > next) {
        Laswp<double>(rest - next, At(w, ldw, 0, j + jb + next), lw, j + 1, j + jb, ipiv, 1);
        update(j, jb, j + jb + next, rest - next, 0);
      }
    });
  }
  signal(la.to_main, look, main);
}

// Right-looking lower Cholesky of w (full symmetric storage; the lower
// triangle is read and factored, the upper one receives L^T at the end) with
// a look-ahead of one block column, like the LU:
//
//   look (high priority): update the next block column with the current L21,
//     factor its diagonal block in FP64 (the recursive POTRF2), invert that
//     block in FP64 (the chained triangular solve of L11 X = I), then form
//     the block column below it as L21 = A21 L11^-T, an Ozaki GEMM (in
//     place: the slicing reads A21 before the product writes it);
//   main: the rest of the trailing update, A22 -= L21 L21^T, an Ozaki GEMM
//     that skips the tiles above the diagonal (only the lower triangle is
//     wanted).
//
// The streams touch disjoint block columns; events order them as the data
// flow requires (main's update waits for the L21 it reads; look's next
// block column waits for main's previous update). FP64 runs only in the
// diagonal blocks; every flop outside them is on the INT8 tensor cores.
void MixedPotrf(int n, double* w, long long ldw, int* info, int slices, MixedBuffers& bf) {
  Context& ctx = Ctx();
  const int nb = MixedBlock(n);
  const int lw = static_cast<int>(ldw);
  const cudaStream_t main = ctx.stream;
  Lookahead& la = GetLookahead();
  const cudaStream_t look = la.ok ? la.stream : main;
  auto signal = [&](cudaEvent_t ev, cudaStream_t from, cudaStream_t to) {
    if (from == to) return;
    cudaEventRecord(ev, from);
    cudaStreamWaitEvent(to, ev, 0);
  };
  double* xinv = static_cast<double*>(
      Workspace(kWsMixedInv, sizeof(double) * static_cast<size_t>(nb) * nb));
  if (xinv == nullptr) return;
  // Diagonal block at j (jb columns): FP64 factor and inverse, then the
  // block column below it, rows [j + jb, n).
  const auto panel = [&](int j, int jb) {
    CholBlock(jb, At(w, ldw, j, j), lw, info, j, bf.barrier + 32);
    const int below = n - j - jb;
    if (below <= 0) return;
    InvertDiagBlocks(jb, At(w, ldw, j, j), ldw, true, false, bf.inv_lo);
    SetIdentityKernel<<<dim3((jb + 255) / 256, jb), 256, 0, ctx.stream>>>(jb, xinv, nb);
    CountLaunch();
    if (!ChainTrsv(true, jb, jb, At(w, ldw, j, j), ldw, bf.inv_lo, xinv, nb,
                   bf.flags + bf.flag_stride))
      TrsmFull<double>(true, true, false, false, jb, jb, 1.0, At(w, ldw, j, j), lw, xinv, nb);
    DgemmEmulated(below, jb, jb, 1.0, ColMajor<double>(At(w, ldw, j + jb, j), ldw),
                  ColMajor<double>(xinv, nb, true), 0.0, At(w, ldw, j + jb, j), lw, slices,
                  false, 1);
  };
  signal(la.to_look, main, look);
  OnStream(look, [&] { panel(0, std::min(nb, n)); });
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    const int rest = n - j - jb;
    if (rest <= 0) break;
    const int next = std::min(nb, rest);
    signal(la.to_main, look, main);  // L21 of block j
    signal(la.to_look, main, look);  // main's previous update
    OnStream(look, [&] {
      // The next block column: rows [j + jb, n), columns [j + jb, + next).
      DgemmEmulated(rest, next, jb, -1.0, ColMajor<double>(At(w, ldw, j + jb, j), ldw),
                    ColMajor<double>(At(w, ldw, j + jb, j), ldw, true), 1.0,
                    At(w, ldw, j + jb, j + jb), lw, slices, false, 1);
      panel(j + jb, next);
    });
    if (rest > next) {
      const int r2 = rest - next;
      const double* l21 = At(w, ldw, j + jb + next, j);
      DgemmEmulated(r2, r2, jb, -1.0, ColMajor<double>(l21, ldw),
                    ColMajor<double>(l21, ldw, true), 1.0,
                    At(w, ldw, j + jb + next, j + jb + next), lw, slices, false, 0, true);
    }
  }
  signal(la.to_main, look, main);
  const dim3 grid((n + 31) / 32, (n + 31) / 32);
  // Upper triangle := transpose of the lower one (in place is safe: each
  // tile reads only the lower triangle and writes only the upper one).
  SymmetrizeKernel<<<grid, dim3(32, 8), 0, Ctx().stream>>>(n, 0, w, ldw, w, ldw);
  CountLaunch();
  LaunchFailed("mixed mirror");
}

// The refinement loop shared by both solvers. Each step computes r = b - A x
// in FP64, d = A^{-1} r with the reduced-precision factors, and x += d. It
// stops once every column meets LAPACK's DSGESV backward criterion
// ||r||_inf <= ||x||_inf ||A||_inf eps sqrt(n) (dsgesv.f) and its correction
// has settled: ||d||_inf <= 2^-52 ||x||_inf, or no longer halving (the
// forward-error stopping rule of iterative refinement). Returns the number of
// corrections applied, or -31 if 30 did not get there.
int Refine(bool lu, int n, int nrhs, const double* a, long long lda, const double* b,
           long long ldb, double* x, long long ldx, double anrm, MixedBuffers& bf) {
  cudaStream_t st = Ctx().stream;
  const double eps = 0.5 * 2.220446049250313e-16;  // DLAMCH('Epsilon')
  const double cte = anrm * eps * std::sqrt(static_cast<double>(n));
  MixedSolve(lu, n, nrhs, bf, b, ldb, x, ldx);  // x = A^{-1} b, reduced precision
  std::vector<std::vector<double>> nm;
  std::vector<double> dprev(nrhs, INFINITY);
  std::vector<char> settled_col(nrhs, 0);
  const double* mats[3] = {x, bf.r, bf.d};
  const long long lds[3] = {ldx, bf.ldr, bf.ldr};
  // The residual is extra-precise (ResidualDd), so the corrections converge
  // to the solution of A x = b itself rather than stalling at the FP64
  // residual's noise (cond(A) eps). For few right-hand sides it costs what
  // the FP64 GEMV costs (both read A once); for many, the FP64 DMMA residual
  // runs until every column meets the backward criterion and the
  // extra-precise one then finishes.
  bool extra = nrhs < kResRhs;
  for (int it = 0; it < kItMax; ++it) {
    if (extra) {
      ResidualDd(n, nrhs, a, lda, b, ldb, x, ldx, bf.r, bf.ldr, bf.part);
    } else {
      Residual(n, nrhs, a, lda, b, ldb, x, ldx, bf);
    }
    MixedSolve(lu, n, nrhs, bf, bf.r, bf.ldr, bf.d, bf.ldr);
    if (!ColumnNorms(n, nrhs, 3, mats, lds, bf, &nm)) return -kItMax - 1;
    AxpyMatrixKernel<<<dim3((n + 255) / 256, nrhs), 256, 0, st>>>(n, nrhs, bf.d, bf.ldr,
                                                                  x, ldx);
    CountLaunch();
    // A column is done once it meets the backward criterion and its
    // correction has settled: it moved x by at most an ulp, it no longer
    // halves (the corrections have reached the residual's noise), or, at the
    // observed rate of contraction dn / dprev, the next one would move x by
    // less than half an ulp. Later corrections only move it within the last
    // bit.
    bool done = true, backward_all = true;
    for (int q = 0; q < nrhs; ++q) {
      const double xn = nm[0][q], rn = nm[1][q], dn = nm[2][q];
      const bool backward = rn <= xn * cte;  // false on NaN
      const bool settled = dn <= 0x1p-52 * xn || dn > 0.5 * dprev[q] ||
                           (std::isfinite(dprev[q]) && (dn / dprev[q]) * dn <= 0x1p-53 * xn);
      if (backward && settled) settled_col[q] = 1;
      if (!settled_col[q]) done = false;
      if (!backward) backward_all = false;
      dprev[q] = dn;
    }
    if (extra && done) return it + 1;
    if (!extra && backward_all) {
      extra = true;
      std::fill(settled_col.begin(), settled_col.end(), 0);
      std::fill(dprev.begin(), dprev.end(), INFINITY);
    }
  }
  return -kItMax - 1;
}

}  // namespace

int DgesvMixed(int n, int nrhs, double* a, int lda, int* ipiv, const double* b,
               int ldb, double* x, int ldx, int slices, int* iter) {
  Context& ctx = Ctx();
  cudaStream_t st = ctx.stream;
  MixedBuffers bf;
  *iter = 0;
  if (!AllocBuffers(n, nrhs, false, &bf)) return -1;
  int* dinfo = ctx.dev_status + 1;
  const double anrm = InfNorm(n, a, lda, bf);
  int fallback = 0;
  if (!std::isfinite(anrm)) {
    fallback = -2;
  } else {
    cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    Copy2D(n, n, a, lda, bf.w, bf.ldw);
    MixedGetrf(n, bf.w, bf.ldw, ipiv, dinfo, slices, bf);
    int finfo = 0;
    cudaMemcpyAsync(&finfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (Failed(cudaStreamSynchronize(st), "mixed getrf")) return -1;
    if (finfo != 0) {
      fallback = -3;
    } else {
      InvertDiagBlocks(n, bf.w, bf.ldw, true, true, bf.inv_lo);
      InvertDiagBlocks(n, bf.w, bf.ldw, false, false, bf.inv_up);
      PermFromPivots(n, ipiv, bf.perm);
      const int it = Refine(true, n, nrhs, a, lda, b, ldb, x, ldx, anrm, bf);
      if (it >= 0) {
        *iter = it;
        return 0;
      }
      fallback = it;
    }
  }
  // FP64: the plain LU and solve on A itself.
  *iter = fallback;
  cudaMemsetAsync(dinfo, 0, sizeof(int), st);
  Getrf<double>(n, n, a, lda, ipiv, dinfo);
  int finfo = 0;
  cudaMemcpyAsync(&finfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (Failed(cudaStreamSynchronize(st), "mixed fallback getrf")) return -1;
  if (finfo == 0) {
    Copy2D(n, nrhs, b, ldb, x, ldx);
    Getrs<double>(false, n, nrhs, a, lda, ipiv, x, ldx);
  }
  return finfo;
}

int DposvMixed(bool upper, int n, int nrhs, double* a, int lda, const double* b,
               int ldb, double* x, int ldx, int slices, int* iter) {
  Context& ctx = Ctx();
  cudaStream_t st = ctx.stream;
  MixedBuffers bf;
  *iter = 0;
  if (!AllocBuffers(n, nrhs, true, &bf)) return -1;
  int* dinfo = ctx.dev_status + 1;
  const dim3 grid((n + 31) / 32, (n + 31) / 32);
  SymmetrizeKernel<<<grid, dim3(32, 8), 0, st>>>(n, upper ? 1 : 0, a, lda, bf.afull,
                                                 bf.ldw);
  CountLaunch();
  LaunchFailed("mixed symmetrize");
  const double anrm = InfNorm(n, bf.afull, bf.ldw, bf);
  int fallback = 0;
  if (!std::isfinite(anrm)) {
    fallback = -2;
  } else {
    cudaMemsetAsync(dinfo, 0, sizeof(int), st);
    Copy2D(n, n, bf.afull, bf.ldw, bf.w, bf.ldw);
    MixedPotrf(n, bf.w, bf.ldw, dinfo, slices, bf);
    int finfo = 0;
    cudaMemcpyAsync(&finfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (Failed(cudaStreamSynchronize(st), "mixed potrf")) return -1;
    if (finfo != 0) {
      fallback = -3;
    } else {
      InvertDiagBlocks(n, bf.w, bf.ldw, true, false, bf.inv_lo);
      InvertDiagBlocks(n, bf.w, bf.ldw, false, false, bf.inv_up);
      const int it = Refine(false, n, nrhs, bf.afull, bf.ldw, b, ldb, x, ldx, anrm, bf);
      if (it >= 0) {
        *iter = it;
        return 0;
      }
      fallback = it;
    }
  }
  *iter = fallback;
  cudaMemsetAsync(dinfo, 0, sizeof(int), st);
  Potrf(upper, n, a, lda, dinfo);
  int finfo = 0;
  cudaMemcpyAsync(&finfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (Failed(cudaStreamSynchronize(st), "mixed fallback potrf")) return -1;
  if (finfo == 0) {
    Copy2D(n, nrhs, b, ldb, x, ldx);
    Potrs(upper, n, nrhs, a, lda, x, ldx);
  }
  return finfo;
}

}  // namespace hb
