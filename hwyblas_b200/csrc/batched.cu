// Batched LU, LU solve and GEMM for many small problems of uneven sizes
// (n up to a few hundred): one persistent launch per routine in which each
// CTA takes whole problems from a work queue (largest first) and runs the
// reference's algorithm on it, call for call:
//   GETRF  src/lapack/getrf.cc:216-280 (nb = 64) and 112-207 (recursion to
//          the 16-column leaf of src/lapack/factor_kernels.cc:79-183)
//   GETRS  src/lapack/getrf.cc:287-339
//   TRSM   src/trsm.cc:87-135 (split max(32, (r/2)/32*32)), base solves of
//          src/trsm-inl.h:107-174 (reciprocal diagonal, column pairs)
//   GEMM   src/gemm_kernel-inl.h:161-224 (a sequential FMA chain per element,
//          restarted every KC = 256 (double) / 384 (float), merged in order)
// so every problem's result is bit-identical to the single-problem routines.
// The reference has no batched API; the entry points follow the argument
// conventions of its single-problem routines with arrays of sizes, leading
// dimensions and device pointers.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>
#include <vector>

#include "../../include/hwyblas_b200.h"
#include "device.cuh"
#include "internal.h"
#include "ref_order.cuh"

namespace hb {

int RefLanesDouble();

namespace {

template <typename T>
struct Kc;
template <>
struct Kc<double> {
  static constexpr int value = 256;
};
template <>
struct Kc<float> {
  static constexpr int value = 384;
};

// A strided matrix operand on the device: element (i, j) at p[i*rs + j*cs].
template <typename T>
struct Mat {
  T* p;
  long long rs, cs;
  __device__ T& operator()(long long i, long long j) const { return p[i * rs + j * cs]; }
  __device__ Mat sub(long long i, long long j) const { return {p + i * rs + j * cs, rs, cs}; }
};

template <typename T>
__device__ __forceinline__ Mat<T> Col(T* p, long long ld) {
  return {p, 1, ld};
}

// C := alpha*A*B + beta*C (m x n, inner k) with the reference's per-element
// order; the CTA's threads share the elements.
template <typename T>
__device__ void CtaGemm(int m, int n, int k, T alpha, Mat<T> a, Mat<T> b, T beta,
                        Mat<T> c) {
  constexpr int KC = Kc<T>::value;
  const int total = m * n;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int i = idx % m, j = idx / m;
    T cv = T(0);
    for (int pc = 0; pc < k; pc += KC) {
      const int pe = min(k, pc + KC);
      T acc = T(0);
      for (int q = pc; q < pe; ++q) acc = fma(a(i, q), b(q, j), acc);
      const T r = alpha * acc;
      if (pc != 0 || beta == T(1)) {
        if (pc == 0) cv = c(i, j);
        cv = r + cv;
      } else if (beta == T(0)) {
        cv = r;
      } else {
        cv = fma(c(i, j), beta, r);
      }
    }
    if (k > 0) c(i, j) = cv;
  }
  __syncthreads();
}

// The same product on the FP64 tensor pipe: the CTA's WM x WN warps walk C in
// tiles of (16 WM) x (8 NB WN); each warp computes a 16 x 8 NB block with NB
// mma.sync.m16n8k8.f64 per k8 step. The MMA accumulates its 8 products in
// ascending k as a chain of correctly rounded FMAs starting from the
// accumulator, so chaining the MMAs over k and restarting every KC = 256
// gives every element the reference's chain; zero padding past k adds +0.
// Each 256-deep chunk is merged into C exactly as CtaGemm merges it. Operand k-blocks of 32 are staged in shared memory with
// rows padded to a stride of 8 (mod 32) words, which makes every fragment
// load conflict free; the next block is fetched into registers while the
// current one is multiplied.
constexpr int kDmmaKb = 32;

__device__ __forceinline__ void BatchDmma(double (&d)[4], double a0, double a1, double a2,
                                          double a3, double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

template <int WM, int WN, int NB>
struct DmmaTile {
  static constexpr int kTM = 16 * WM, kTN = 8 * NB * WN;
  static constexpr int kThreads = 32 * WM * WN;
  static constexpr int kSA = kTM + 4, kSB = kTN + 4;  // row strides (doubles)
  static constexpr int kLoadA = kDmmaKb * kTM / kThreads;  // elements per thread
  static constexpr int kLoadB = kDmmaKb * kTN / kThreads;
};

template <int WM, int WN, int NB>
__device__ void CtaGemmDmma(int m, int n, int k, double alpha, Mat<double> a, Mat<double> b,
                            double beta, Mat<double> c, double* sA, double* sB) {
  using Cfg = DmmaTile<WM, WN, NB>;
  constexpr int TM = Cfg::kTM, TN = Cfg::kTN, SA = Cfg::kSA, SB = Cfg::kSB;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int wm = warp % WM, wn = warp / WM;
  const int g = lane >> 2, t = lane & 3;
  // Operand loads: along the contiguous index of each operand.
  const bool a_rows = a.rs == 1;  // A(i, q) contiguous in i
  const bool b_rows = b.rs == 1;  // B(q, j) contiguous in q
  for (int m0 = 0; m0 < m; m0 += TM) {
    for (int n0 = 0; n0 < n; n0 += TN) {
      double acc[NB][4];
      double ra[Cfg::kLoadA], rb[Cfg::kLoadB];
      const auto fetch = [&](int kb0) {
#pragma unroll
        for (int l = 0; l < Cfg::kLoadA; ++l) {
          const int idx = threadIdx.x + l * Cfg::kThreads;
          const int i = a_rows ? idx % TM : idx / kDmmaKb;
          const int q = a_rows ? idx / TM : idx % kDmmaKb;
          ra[l] = (m0 + i < m && kb0 + q < k) ? a(m0 + i, kb0 + q) : 0.0;
        }
#pragma unroll
        for (int l = 0; l < Cfg::kLoadB; ++l) {
          const int idx = threadIdx.x + l * Cfg::kThreads;
          const int q = b_rows ? idx % kDmmaKb : idx / TN;
          const int j = b_rows ? idx / kDmmaKb : idx % TN;
          rb[l] = (n0 + j < n && kb0 + q < k) ? b(kb0 + q, n0 + j) : 0.0;
        }
      };
      const auto stash = [&]() {
#pragma unroll
        for (int l = 0; l < Cfg::kLoadA; ++l) {
          const int idx = threadIdx.x + l * Cfg::kThreads;
          const int i = a_rows ? idx % TM : idx / kDmmaKb;
          const int q = a_rows ? idx / TM : idx % kDmmaKb;
          sA[q * SA + i] = ra[l];
        }
#pragma unroll
        for (int l = 0; l < Cfg::kLoadB; ++l) {
          const int idx = threadIdx.x + l * Cfg::kThreads;
          const int q = b_rows ? idx % kDmmaKb : idx / TN;
          const int j = b_rows ? idx / kDmmaKb : idx % TN;
          sB[q * SB + j] = rb[l];
        }
      };
      fetch(0);
      for (int pc = 0; pc < k; pc += 256) {
        const int pe = min(k, pc + 256);
#pragma unroll
        for (int nb = 0; nb < NB; ++nb)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[nb][e] = 0.0;
        for (int kb0 = pc; kb0 < pe; kb0 += kDmmaKb) {
          __syncthreads();  // the previous block's fragments are read
          stash();
          __syncthreads();
          if (kb0 + kDmmaKb < k) fetch(kb0 + kDmmaKb);
          const int steps = (min(pe, kb0 + kDmmaKb) - kb0 + 7) / 8;
          for (int ks = 0; ks < steps; ++ks) {
            const double* pa = sA + (ks * 8 + t) * SA + wm * 16 + g;
            const double a0 = pa[0], a1 = pa[8], a2 = pa[4 * SA], a3 = pa[4 * SA + 8];
#pragma unroll
            for (int nb = 0; nb < NB; ++nb) {
              const double* pb = sB + (ks * 8 + t) * SB + wn * 8 * NB + nb * 8 + g;
              BatchDmma(acc[nb], a0, a1, a2, a3, pb[0], pb[4 * SB]);
            }
          }
        }
        // Merge the chunk into C (CtaGemm's rules; each element is read and
        // written by its own thread only).
#pragma unroll
        for (int nb = 0; nb < NB; ++nb) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = m0 + wm * 16 + g + (e >> 1) * 8;
            const int j = n0 + wn * 8 * NB + nb * 8 + 2 * t + (e & 1);
            if (i >= m || j >= n) continue;
            const double r = alpha * acc[nb][e];
            if (pc != 0 || beta == 1.0) {
              c(i, j) = r + c(i, j);
            } else if (beta == 0.0) {
              c(i, j) = r;
            } else {
              c(i, j) = fma(c(i, j), beta, r);
            }
          }
        }
      }
    }
  }
  __syncthreads();
}

// The same per-element chains with register tiles: the CTA's Threads threads
// form a 16 x (Threads / 16) grid, each computing a 4 x 4 block of C; k-blocks
// of 16 of A and B are staged in shared memory (the next one fetched into
// registers while the current one is used) and each element's FMA chain runs
// over q in ascending order, restarted every KC, exactly as in CtaGemm.
template <typename T, int Threads>
struct RegTile {
  static constexpr int kTM = 64, kTN = 4 * (Threads / 16), kKb = 16;
  static constexpr int kSA = kTM + 4, kSB = kTN + 4;  // row strides (elements)
  static constexpr int kLoadA = kKb * kTM / Threads, kLoadB = kKb * kTN / Threads;
};

template <typename T>
__device__ __forceinline__ void Load4(const T* p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 x = *reinterpret_cast<const float4*>(p);
    v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
  } else {
    const double2 x = *reinterpret_cast<const double2*>(p);
    const double2 y = *reinterpret_cast<const double2*>(p + 2);
    v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
  }
}

template <typename T, int Threads>
__device__ void CtaGemmReg(int m, int n, int k, T alpha, Mat<T> a, Mat<T> b, T beta,
                           Mat<T> c, T* sA, T* sB) {
  using Cfg = RegTile<T, Threads>;
  constexpr int KC = Kc<T>::value, TM = Cfg::kTM, TN = Cfg::kTN, KB = Cfg::kKb;
  constexpr int SA = Cfg::kSA, SB = Cfg::kSB;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const bool a_rows = a.rs == 1;  // A(i, q) contiguous in i
  const bool b_rows = b.rs == 1;  // B(q, j) contiguous in q
  for (int m0 = 0; m0 < m; m0 += TM) {
    for (int n0 = 0; n0 < n; n0 += TN) {
      T acc[4][4];
      T ra[Cfg::kLoadA], rb[Cfg::kLoadB];
      const auto fetch = [&](int kb0) {
#pragma unroll
        for (int l = 0; l < Cfg::kLoadA; ++l) {
          const int idx = threadIdx.x + l * Threads;
          const int i = a_rows ? idx % TM : idx / KB;
          const int q = a_rows ? idx / TM : idx % KB;
          ra[l] = (m0 + i < m && kb0 + q < k) ? a(m0 + i, kb0 + q) : T(0);
        }
#pragma unroll
        for (int l = 0; l < Cfg::kLoadB; ++l) {
          const int idx = threadIdx.x + l * Threads;
          const int q = b_rows ? idx % KB : idx / TN;
          const int j = b_rows ? idx / KB : idx % TN;
          rb[l] = (n0 + j < n && kb0 + q < k) ? b(kb0 + q, n0 + j) : T(0);
        }
      };
      const auto stash = [&]() {
#pragma unroll
        for (int l = 0; l < Cfg::kLoadA; ++l) {
          const int idx = threadIdx.x + l * Threads;
          const int i = a_rows ? idx % TM : idx / KB;
          const int q = a_rows ? idx / TM : idx % KB;
          sA[q * SA + i] = ra[l];
        }
#pragma unroll
        for (int l = 0; l < Cfg::kLoadB; ++l) {
          const int idx = threadIdx.x + l * Threads;
          const int q = b_rows ? idx % KB : idx / TN;
          const int j = b_rows ? idx / KB : idx % TN;
          sB[q * SB + j] = rb[l];
        }
      };
      fetch(0);
      for (int pc = 0; pc < k; pc += KC) {
        const int pe = min(k, pc + KC);
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[r][s] = T(0);
        for (int kb0 = pc; kb0 < pe; kb0 += KB) {
          __syncthreads();  // the previous block is read
          stash();
          __syncthreads();
          if (kb0 + KB < k) fetch(kb0 + KB);
          const int steps = min(pe, kb0 + KB) - kb0;
          for (int q = 0; q < steps; ++q) {
            T av[4], bv[4];
            Load4(sA + q * SA + 4 * tx, av);
            Load4(sB + q * SB + 4 * ty, bv);
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
              for (int s = 0; s < 4; ++s) acc[r][s] = fma(av[r], bv[s], acc[r][s]);
          }
        }
        // Merge the chunk into C (CtaGemm's rules; each element is read and
        // written by its own thread only).
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            const int i = m0 + 4 * tx + r, j = n0 + 4 * ty + s;
            if (i >= m || j >= n) continue;
            const T v = alpha * acc[r][s];
            if (pc != 0 || beta == T(1)) {
              c(i, j) = v + c(i, j);
            } else if (beta == T(0)) {
              c(i, j) = v;
            } else {
              c(i, j) = fma(c(i, j), beta, v);
            }
          }
        }
      }
    }
  }
  __syncthreads();
}

// The GEMM a batched factorization or solve calls for its updates: the
// per-element chains (any type, any CTA size) or, in FP64, the tensor-pipe
// tiles for blocks of at least 16 x 16 (the CTA has the tile's warps). Both
// give every element the same bits.
template <typename T>
struct ElemGemm {
  __device__ void operator()(int m, int n, int k, T alpha, Mat<T> a, Mat<T> b, T beta,
                             Mat<T> c) const {
    CtaGemm<T>(m, n, k, alpha, a, b, beta, c);
  }
};

template <typename T, int Threads>
struct RegGemm {
  T* sA;
  T* sB;
  __device__ void operator()(int m, int n, int k, T alpha, Mat<T> a, Mat<T> b, T beta,
                             Mat<T> c) const {
    if (m < 16 || n < 16)
      CtaGemm<T>(m, n, k, alpha, a, b, beta, c);
    else
      CtaGemmReg<T, Threads>(m, n, k, alpha, a, b, beta, c, sA, sB);
  }
};

template <int WM, int WN, int NB>
struct TileGemm {
  double* sA;
  double* sB;
  __device__ void operator()(int m, int n, int k, double alpha, Mat<double> a,
                             Mat<double> b, double beta, Mat<double> c) const {
    if (m < 16 || n < 16)
      CtaGemm<double>(m, n, k, alpha, a, b, beta, c);
    else
      CtaGemmDmma<WM, WN, NB>(m, n, k, alpha, a, b, beta, c, sA, sB);
  }
};

// Row interchanges k1..k2 (1-based, increasing) of ncols columns.
template <typename T>
__device__ void CtaLaswp(int ncols, Mat<T> a, int k1, int k2, const int* ipiv) {
  for (int col = threadIdx.x; col < ncols; col += blockDim.x) {
    for (int i = k1; i <= k2; ++i) {
      const int ip = ipiv[i - 1];
      if (ip != i) {
        const T t = a(i - 1, col);
        a(i - 1, col) = a(ip - 1, col);
        a(ip - 1, col) = t;
      }
    }
  }
  __syncthreads();
}

// Backward interchanges (incx = -1): k2 down to k1.
template <typename T>
__device__ void CtaLaswpBack(int ncols, Mat<T> a, int k1, int k2, const int* ipiv) {
  for (int col = threadIdx.x; col < ncols; col += blockDim.x) {
    for (int i = k2; i >= k1; --i) {
      const int ip = ipiv[i - 1];
      if (ip != i) {
        const T t = a(i - 1, col);
        a(i - 1, col) = a(ip - 1, col);
        a(ip - 1, col) = t;
      }
    }
  }
  __syncthreads();
}

// Base solve of the TRSM recursion (r <= 32): x op(T) = b for each of the
// `other` rows of x, in solve order with the reciprocal diagonal and column
// pairs; t is already the right-side triangle (lower: solved from the last
// column). st and sinv are shared scratch.
template <typename T>
__device__ void CtaTrsmBase(Mat<T> t, bool lower, bool unit, int r, int other, T* x,
                            long long xs_row, long long xs_col, T (*st)[33], T* sinv) {
  for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
    const int s = idx / 32, u = idx % 32;
    T v = T(0);
    if (s < r && u < r) {
      const int q = lower ? r - 1 - s : s, j = lower ? r - 1 - u : u;
      if (s < u || (s == u && !unit)) v = t(q, j);
    }
    st[s][u] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int s = threadIdx.x;
    sinv[s] = (s < r && !unit) ? T(1) / st[s][s] : T(1);
  }
  __syncthreads();
  for (int row = threadIdx.x; row < other; row += blockDim.x) {
    T* xr = x + row * xs_row;
    T y[32];
#pragma unroll
    for (int s = 0; s < 32; ++s)
      if (s < r) y[s] = xr[(lower ? r - 1 - s : s) * xs_col];
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
      } else if (step < r) {
        T acc = y[step];
#pragma unroll
        for (int s = 0; s < step; ++s) acc = fma(-y[s], st[s][step], acc);
        if (!unit) acc = acc * sinv[step];
        y[step] = acc;
      }
    }
#pragma unroll
    for (int s = 0; s < 32; ++s)
      if (s < r) xr[(lower ? r - 1 - s : s) * xs_col] = y[s];
  }
  __syncthreads();
}

// Left-side triangular solve op(T) X = B (op(T) is `tri`, r x r; X is r x
// other, column-major ld ldb) by the reference's recursion, emulated with an
// explicit stack: top half, GEMM update, bottom half (lower; upper mirrored).
template <typename T, typename G>
__device__ void CtaTrsmLeft(Mat<T> tri, bool lower, bool unit, int r, int other, T* b,
                            long long ldb, T (*st)[33], T* sinv, const G& gemm) {
  if (r <= 0 || other <= 0) return;
  int s_off[8], s_r[8], s_ph[8];
  int sp = 0;
  s_off[0] = 0;
  s_r[0] = r;
  s_ph[0] = 0;
  while (sp >= 0) {
    const int off = s_off[sp], rr = s_r[sp];
    if (rr <= 32) {
      // TrsmSolve for the left side: X^T op(T)^T = B^T, rows of X^T are the
      // columns of B.
      Mat<T> t = tri.sub(off, off);
      const Mat<T> tt = {t.p, t.cs, t.rs};
      CtaTrsmBase(tt, !lower, unit, rr, other, b + off, ldb, 1, st, sinv);
      --sp;
      continue;
    }
    const int r1 = max(32, (rr / 2) / 32 * 32), r2 = rr - r1;
    const int ph = s_ph[sp]++;
    if (ph == 2) {
      --sp;
      continue;
    }
    if (lower) {
      if (ph == 0) {
        ++sp;
        s_off[sp] = off;
        s_r[sp] = r1;
        s_ph[sp] = 0;
      } else {
        gemm(r2, other, r1, T(-1), tri.sub(off + r1, off), Col(b + off, ldb), T(1),
             Col(b + off + r1, ldb));
        ++sp;
        s_off[sp] = off + r1;
        s_r[sp] = r2;
        s_ph[sp] = 0;
      }
    } else {
      if (ph == 0) {
        ++sp;
        s_off[sp] = off + r1;
        s_r[sp] = r2;
        s_ph[sp] = 0;
      } else {
        gemm(r1, other, r2, T(-1), tri.sub(off, off + r1), Col(b + off + r1, ldb), T(1),
             Col(b + off, ldb));
        ++sp;
        s_off[sp] = off;
        s_r[sp] = r1;
        s_ph[sp] = 0;
      }
    }
  }
}

// Right-side triangular solve X op(T) = B (X is other x r, column-major ld
// ldb), the reference's recursion for the right side: lower solves the
// trailing block first, upper the leading one.
template <typename T, typename G>
__device__ void CtaTrsmRight(Mat<T> tri, bool lower, bool unit, int r, int other, T* b,
                             long long ldb, T (*st)[33], T* sinv, const G& gemm) {
  if (r <= 0 || other <= 0) return;
  int s_off[8], s_r[8], s_ph[8];
  int sp = 0;
  s_off[0] = 0;
  s_r[0] = r;
  s_ph[0] = 0;
  while (sp >= 0) {
    const int off = s_off[sp], rr = s_r[sp];
    if (rr <= 32) {
      CtaTrsmBase(tri.sub(off, off), lower, unit, rr, other, b + off * ldb, 1, ldb, st,
                  sinv);
      --sp;
      continue;
    }
    const int r1 = max(32, (rr / 2) / 32 * 32), r2 = rr - r1;
    const int ph = s_ph[sp]++;
    if (ph == 2) {
      --sp;
      continue;
    }
    const bool first_trailing = lower;
    if (ph == 0) {
      ++sp;
      s_off[sp] = first_trailing ? off + r1 : off;
      s_r[sp] = first_trailing ? r2 : r1;
      s_ph[sp] = 0;
    } else {
      if (lower) {
        gemm(other, r1, r2, T(-1), Col(b + (off + r1) * ldb, ldb), tri.sub(off + r1, off),
             T(1), Col(b + off * ldb, ldb));
      } else {
        gemm(other, r2, r1, T(-1), Col(b + off * ldb, ldb), tri.sub(off, off + r1), T(1),
             Col(b + (off + r1) * ldb, ldb));
      }
      ++sp;
      s_off[sp] = first_trailing ? off : off + r1;
      s_r[sp] = first_trailing ? r1 : r2;
      s_ph[sp] = 0;
    }
  }
}

// Shared scratch of the per-CTA LU.
template <typename T>
struct LuShared {
  T st[32][33];
  T sinv[32];
  T wv[32];
  int wi[32];
  int piv;
};

// LU leaf (min(m, n) <= 16) on an m x n block: partial pivoting with the
// reference's pivot choice, reciprocal scaling (or division below sfmin) and
// AXPY rounding; trailing columns (n > m) take all interchanges, then the
// updates with the final L.
template <typename T>
__device__ void CtaLeaf(int m, int n, Mat<T> a, int* ipiv, int* info, int col0, int lanes,
                        LuShared<T>& sh) {
  const int w = min(m, n);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int nwarps = blockDim.x / 32;
  for (int j = 0; j < w; ++j) {
    T bv = T(-1);
    int bi = 0x7fffffff;
    for (int i = j + threadIdx.x; i < m; i += blockDim.x) {
      const T v = fabs(a(i, j));
      if (v > bv) { bv = v; bi = i; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const T ov = __shfl_down_sync(0xffffffffu, bv, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (Better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { sh.wv[warp] = bv; sh.wi[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
      bv = lane < nwarps ? sh.wv[lane] : T(-1);
      bi = lane < nwarps ? sh.wi[lane] : 0x7fffffff;
      for (int off = 16; off > 0; off >>= 1) {
        const T ov = __shfl_down_sync(0xffffffffu, bv, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (Better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
      }
      if (lane == 0) {
        if (isnan(fabs(a(j, j))) || bi == 0x7fffffff) bi = j;
        sh.piv = bi;
        ipiv[j] = bi + 1;
        if (a(bi, j) == T(0) && *info == 0) *info = col0 + j + 1;
      }
    }
    __syncthreads();
    const int piv = sh.piv;
    const T pivot = a(piv, j);
    if (pivot != T(0) && piv != j) {
      for (int c = threadIdx.x; c < w; c += blockDim.x) {
        const T t = a(j, c);
        a(j, c) = a(piv, c);
        a(piv, c) = t;
      }
    }
    __syncthreads();
    const bool scale = pivot != T(0);
    const bool tiny = !(fabs(pivot) >= Sfmin<T>());
    const T rinv = T(1) / pivot;
    const int len = m - j - 1;
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
      T x = a(i, j);
      if (scale) {
        x = tiny ? x / pivot : x * rinv;
        a(i, j) = x;
      }
      for (int k = j + 1; k < w; ++k) a(i, k) = Axpy(a(i, k), -a(j, k), x, len, lanes);
    }
    __syncthreads();
  }
  for (int k = w + threadIdx.x; k < n; k += blockDim.x) {
    for (int j = 0; j < w; ++j) {
      const int p = ipiv[j] - 1;
      if (p != j) {
        const T t = a(j, k);
        a(j, k) = a(p, k);
        a(p, k) = t;
      }
    }
    for (int j = 0; j < w; ++j) {
      const T alpha = -a(j, k);
      const int len = m - j - 1;
      for (int i = j + 1; i < m; ++i) a(i, k) = Axpy(a(i, k), alpha, a(i, j), len, lanes);
    }
  }
  __syncthreads();
}

// The reference's recursive LU (Getrf2) of an m x n block at a, with the
// block's pivots in ipiv (block-relative, 1-based) and col0 its first global
// column (for INFO). Recursion emulated with an explicit stack; frames sit
// on the block's diagonal at offset off.
template <typename T, typename G>
__device__ void CtaGetrfRec(int m, int n, Mat<T> a, int* ipiv, int* info, int col0,
                            int lanes, LuShared<T>& sh, const G& gemm) {
  int s_m[12], s_n[12], s_off[12], s_ph[12];
  int sp = 0;
  s_m[0] = m;
  s_n[0] = n;
  s_off[0] = 0;
  s_ph[0] = 0;
  while (sp >= 0) {
    const int fm = s_m[sp], fn = s_n[sp], off = s_off[sp];
    const Mat<T> fa = a.sub(off, off);
    int* fp = ipiv + off;
    if (fm == 0 || fn == 0) {
      --sp;
      continue;
    }
    const int mn = min(fm, fn);
    if (mn <= 16) {
      CtaLeaf(fm, fn, fa, fp, info, col0 + off, lanes, sh);
      --sp;
      continue;
    }
    const int n1 = mn / 2, n2 = fn - n1;
    const int ph = s_ph[sp]++;
    if (ph == 0) {
      ++sp;
      s_m[sp] = fm;
      s_n[sp] = n1;
      s_off[sp] = off;
      s_ph[sp] = 0;
    } else if (ph == 1) {
      CtaLaswp(n2, fa.sub(0, n1), 1, n1, fp);
      CtaTrsmLeft(fa, true, true, n1, n2, &fa(0, n1), fa.cs, sh.st, sh.sinv, gemm);
      gemm(fm - n1, n2, n1, T(-1), fa.sub(n1, 0), fa.sub(0, n1), T(1), fa.sub(n1, n1));
      ++sp;
      s_m[sp] = fm - n1;
      s_n[sp] = n2;
      s_off[sp] = off + n1;
      s_ph[sp] = 0;
    } else {
      for (int i = n1 + threadIdx.x; i < mn; i += blockDim.x) fp[i] += n1;
      __syncthreads();
      CtaLaswp(n1, fa, n1 + 1, mn, fp);
      --sp;
    }
  }
}

// The reference's blocked LU (Getrf, nb = 64) of an n x n matrix.
template <typename T, typename G>
__device__ void CtaGetrf(int n, Mat<T> a, int* ipiv, int* info, int lanes,
                         LuShared<T>& sh, const G& gemm) {
  constexpr int nb = 64;
  if (n == 0) return;
  if (nb >= n) {
    CtaGetrfRec(n, n, a, ipiv, info, 0, lanes, sh, gemm);
    return;
  }
  for (int j = 0; j < n; j += nb) {
    const int jb = min(n - j, nb);
    CtaGetrfRec(n - j, jb, a.sub(j, j), ipiv + j, info, j, lanes, sh, gemm);
    for (int i = j + threadIdx.x; i < j + jb; i += blockDim.x) ipiv[i] += j;
    __syncthreads();
    CtaLaswp(j, a, j + 1, j + jb, ipiv);
    if (j + jb < n) {
      CtaLaswp(n - j - jb, a.sub(0, j + jb), j + 1, j + jb, ipiv);
      CtaTrsmLeft(a.sub(j, j), true, true, jb, n - j - jb, &a(j, j + jb), a.cs, sh.st,
                  sh.sinv, gemm);
      gemm(n - j - jb, n - j - jb, jb, T(-1), a.sub(j + jb, j), a.sub(j, j + jb), T(1),
           a.sub(j + jb, j + jb));
    }
  }
}

// The reference's Getrs: solve op(A) X = B with the LU factors.
template <typename T, typename G>
__device__ void CtaGetrs(bool trans, int n, int nrhs, Mat<T> a, const int* ipiv, T* b,
                         long long ldb, LuShared<T>& sh, const G& gemm) {
  if (n == 0 || nrhs == 0) return;
  const Mat<T> bm = Col(b, ldb);
  if (!trans) {
    CtaLaswp(nrhs, bm, 1, n, ipiv);
    CtaTrsmLeft(a, true, true, n, nrhs, b, ldb, sh.st, sh.sinv, gemm);
    CtaTrsmLeft(a, false, false, n, nrhs, b, ldb, sh.st, sh.sinv, gemm);
  } else {
    // op(T) = T^T: the transposed view, upper <-> lower.
    const Mat<T> at = {a.p, a.cs, a.rs};
    CtaTrsmLeft(at, true, false, n, nrhs, b, ldb, sh.st, sh.sinv, gemm);
    CtaTrsmLeft(at, false, true, n, nrhs, b, ldb, sh.st, sh.sinv, gemm);
    CtaLaswpBack(nrhs, bm, 1, n, ipiv);
  }
}

// ---------------------------------------------------------------------------
// Persistent batched kernels: CTAs take problems from a queue ordered by
// decreasing size until it is empty (no waits).

template <typename T>
struct BatchArgs {
  int count;
  const int* order;      // problem indices, largest first
  unsigned int* next;    // queue head, zero at launch
  const int* m;          // getrf/getrs: n; gemm: m
  const int* n;          // getrs: nrhs; gemm: n
  const int* k;          // gemm: k
  const int* lda;
  const int* ldb;
  const int* ldc;
  T* const* a;
  T* const* b;
  T* const* c;
  int* const* ipiv;
  int* info;
  T alpha, beta;
  int flags;             // getrs: trans; gemm: transa | transb << 1
  int lanes;
};

template <typename T>
__device__ __forceinline__ int NextProblem(const BatchArgs<T>& p, int* slot) {
  if (threadIdx.x == 0) *slot = static_cast<int>(atomicAdd(p.next, 1u));
  __syncthreads();
  const int q = *slot;
  __syncthreads();
  return q < p.count ? p.order[q] : -1;
}

// The three queue loops, each with the GEMM its updates use.
template <typename T, typename G>
__device__ void GetrfProblems(const BatchArgs<T>& p, const G& gemm, LuShared<T>& sh,
                              int* slot) {
  for (int id = NextProblem(p, slot); id >= 0; id = NextProblem(p, slot)) {
    if (threadIdx.x == 0) p.info[id] = 0;
    __syncthreads();
    CtaGetrf(p.m[id], Col(p.a[id], p.lda[id]), p.ipiv[id], &p.info[id], p.lanes, sh, gemm);
  }
}

template <typename T, typename G>
__device__ void GetrsProblems(const BatchArgs<T>& p, const G& gemm, LuShared<T>& sh,
                              int* slot) {
  for (int id = NextProblem(p, slot); id >= 0; id = NextProblem(p, slot)) {
    CtaGetrs(p.flags != 0, p.m[id], p.n[id], Col(p.a[id], p.lda[id]), p.ipiv[id], p.b[id],
             p.ldb[id], sh, gemm);
  }
}

// TRSM (src/trsm.cc:137-180): B := alpha*B first (alpha != 1; B zeroed for
// alpha == 0), then the recursion on op(A). flags: bit 0 right side, bit 1
// lower, bit 2 transposed, bit 3 unit diagonal.
template <typename T, typename G>
__device__ void TrsmProblems(const BatchArgs<T>& p, const G& gemm, LuShared<T>& sh,
                             int* slot) {
  for (int id = NextProblem(p, slot); id >= 0; id = NextProblem(p, slot)) {
    const int m = p.m[id], n = p.n[id];
    if (m == 0 || n == 0) continue;
    const bool right = p.flags & 1, lower = p.flags & 2, trans = p.flags & 4,
               unit = p.flags & 8;
    T* b = p.b[id];
    const long long ldb = p.ldb[id];
    if (p.alpha != T(1)) {
      for (int idx = threadIdx.x; idx < m * n; idx += blockDim.x) {
        T& v = b[idx % m + (idx / m) * ldb];
        v = (p.alpha == T(0)) ? T(0) : v * p.alpha;
      }
      __syncthreads();
      if (p.alpha == T(0)) continue;
    }
    const long long la = p.lda[id];
    const Mat<T> tri = trans ? Mat<T>{p.a[id], la, 1} : Col(p.a[id], la);
    const bool op_lower = trans ? !lower : lower;
    if (right)
      CtaTrsmRight(tri, op_lower, unit, n, m, b, ldb, sh.st, sh.sinv, gemm);
    else
      CtaTrsmLeft(tri, op_lower, unit, m, n, b, ldb, sh.st, sh.sinv, gemm);
  }
}

enum BatchKindDev { kDevGetrf = 0, kDevGetrs = 1, kDevTrsm = 3 };

template <int Kind, typename T, typename G>
__device__ __forceinline__ void RunProblems(const BatchArgs<T>& p, const G& gemm,
                                            LuShared<T>& sh, int* slot) {
  if (Kind == kDevGetrf) GetrfProblems(p, gemm, sh, slot);
  else if (Kind == kDevGetrs) GetrsProblems(p, gemm, sh, slot);
  else TrsmProblems(p, gemm, sh, slot);
}

// Per-element updates (any CTA size up to 256).
template <int Kind, typename T, int Threads, int MinBlocks = 1>
__global__ void __launch_bounds__(Threads, MinBlocks) BatchedLuKernel(BatchArgs<T> p) {
  using Cfg = RegTile<T, Threads>;
  __shared__ LuShared<T> sh;
  __shared__ __align__(16) T sA[Cfg::kKb * Cfg::kSA];
  __shared__ __align__(16) T sB[Cfg::kKb * Cfg::kSB];
  __shared__ int slot;
  RunProblems<Kind>(p, RegGemm<T, Threads>{sA, sB}, sh, &slot);
}

// FP64 updates on the tensor pipe (the CTA has the tile's WM x WN warps).
template <int Kind, int WM, int WN, int NB, int MinBlocks = 1>
__global__ void __launch_bounds__(DmmaTile<WM, WN, NB>::kThreads, MinBlocks)
    BatchedLuDmmaKernel(BatchArgs<double> p) {
  using Cfg = DmmaTile<WM, WN, NB>;
  __shared__ LuShared<double> sh;
  __shared__ double sA[kDmmaKb * Cfg::kSA];
  __shared__ double sB[kDmmaKb * Cfg::kSB];
  __shared__ int slot;
  RunProblems<Kind>(p, TileGemm<WM, WN, NB>{sA, sB}, sh, &slot);
}

template <typename T, int Threads>
__global__ void __launch_bounds__(Threads, 512 / Threads) BatchedGemmKernel(BatchArgs<T> p) {
  using Cfg = RegTile<T, Threads>;
  __shared__ __align__(16) T sA[Cfg::kKb * Cfg::kSA];
  __shared__ __align__(16) T sB[Cfg::kKb * Cfg::kSB];
  __shared__ int slot;
  for (int id = NextProblem(p, &slot); id >= 0; id = NextProblem(p, &slot)) {
    const long long la = p.lda[id], lb = p.ldb[id];
    const Mat<T> a = (p.flags & 1) ? Mat<T>{p.a[id], la, 1} : Col(p.a[id], la);
    const Mat<T> b = (p.flags & 2) ? Mat<T>{p.b[id], lb, 1} : Col(p.b[id], lb);
    const int m = p.m[id], n = p.n[id], k = p.k[id];
    if (m == 0 || n == 0) continue;
    if (k == 0 || p.alpha == T(0)) {
      // Only C := beta*C (C not read for beta == 0), as the single GEMM.
      if (p.beta != T(1)) {
        const Mat<T> c = Col(p.c[id], p.ldc[id]);
        for (int idx = threadIdx.x; idx < m * n; idx += blockDim.x) {
          const int i = idx % m, j = idx / m;
          c(i, j) = (p.beta == T(0)) ? T(0) : c(i, j) * p.beta;
        }
      }
      __syncthreads();
      continue;
    }
    RegGemm<T, Threads>{sA, sB}(m, n, k, p.alpha, a, b, p.beta, Col(p.c[id], p.ldc[id]));
  }
}

// FP64 batched GEMM on the tensor pipe (CtaGemmDmma) for problems with m and n
// of at least 16; smaller ones take the per-element chains of CtaGemm.
template <int WM, int WN, int NB>
__global__ void __launch_bounds__(DmmaTile<WM, WN, NB>::kThreads,
                                  512 / DmmaTile<WM, WN, NB>::kThreads)
    BatchedGemmDmmaKernel(BatchArgs<double> p) {
  using Cfg = DmmaTile<WM, WN, NB>;
  __shared__ double sA[kDmmaKb * Cfg::kSA];
  __shared__ double sB[kDmmaKb * Cfg::kSB];
  __shared__ int slot;
  for (int id = NextProblem(p, &slot); id >= 0; id = NextProblem(p, &slot)) {
    const long long la = p.lda[id], lb = p.ldb[id];
    const Mat<double> a = (p.flags & 1) ? Mat<double>{p.a[id], la, 1} : Col(p.a[id], la);
    const Mat<double> b = (p.flags & 2) ? Mat<double>{p.b[id], lb, 1} : Col(p.b[id], lb);
    const int m = p.m[id], n = p.n[id], k = p.k[id];
    if (m == 0 || n == 0) continue;
    const Mat<double> c = Col(p.c[id], p.ldc[id]);
    if (k == 0 || p.alpha == 0.0) {
      if (p.beta != 1.0) {
        for (int idx = threadIdx.x; idx < m * n; idx += blockDim.x) {
          const int i = idx % m, j = idx / m;
          c(i, j) = (p.beta == 0.0) ? 0.0 : c(i, j) * p.beta;
        }
      }
      __syncthreads();
      continue;
    }
    if (m < 16 || n < 16) {
      CtaGemm<double>(m, n, k, p.alpha, a, b, p.beta, c);
    } else {
      CtaGemmDmma<WM, WN, NB>(m, n, k, p.alpha, a, b, p.beta, c, sA, sB);
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.

namespace {

// Whether [p, p + bytes) lies inside one device allocation (cuMemGetAddressRange
// through the runtime's driver entry point), with the last ranges cached: a
// batch usually carves its problems out of a few allocations.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddressRangeFn RangeFn() {
  static AddressRangeFn fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &ptr, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<AddressRangeFn>(nullptr);
    return reinterpret_cast<AddressRangeFn>(ptr);
  }();
  return fn;
}

struct ExtentChecker {
  std::vector<std::pair<uintptr_t, uintptr_t>> ranges;
  bool Check(const void* p, size_t bytes) {
    if (bytes == 0) return true;
    if (p == nullptr) return false;
    const uintptr_t lo = reinterpret_cast<uintptr_t>(p), hi = lo + bytes;
    for (const auto& r : ranges)
      if (lo >= r.first && hi <= r.second) return true;
    AddressRangeFn fn = RangeFn();
    if (fn == nullptr) return false;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, static_cast<CUdeviceptr>(lo)) != CUDA_SUCCESS) return false;
    const uintptr_t b = static_cast<uintptr_t>(base);
    ranges.emplace_back(b, b + size);
    if (ranges.size() > 64) ranges.erase(ranges.begin());
    return lo >= b && hi <= b + size;
  }
};

// Pinned host staging for a batch's descriptor, copied to the device in one
// transfer.
struct HostStage {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* Get(size_t want) {
    if (bytes < want) {
      if (ptr != nullptr) {
        cudaStreamSynchronize(Ctx().stream);
        cudaFreeHost(ptr);
      }
      ptr = nullptr;
      bytes = 0;
      if (cudaMallocHost(&ptr, want) != cudaSuccess) return nullptr;
      bytes = want;
    }
    return ptr;
  }
};
thread_local HostStage t_stage;

size_t Align8(size_t v) { return (v + 7) / 8 * 8; }

// Lays out the descriptor of a batch: int arrays then pointer arrays.
struct Layout {
  size_t off_order, off_next, off_m, off_n, off_k, off_lda, off_ldb, off_ldc, off_info;
  size_t off_a, off_b, off_c, off_ipiv, total;
  explicit Layout(int count) {
    size_t o = 0;
    const size_t ints = sizeof(int) * static_cast<size_t>(count);
    off_order = o; o = Align8(o + ints);
    off_next = o; o = Align8(o + 64);
    off_m = o; o = Align8(o + ints);
    off_n = o; o = Align8(o + ints);
    off_k = o; o = Align8(o + ints);
    off_lda = o; o = Align8(o + ints);
    off_ldb = o; o = Align8(o + ints);
    off_ldc = o; o = Align8(o + ints);
    off_info = o; o = Align8(o + ints);
    const size_t ptrs = sizeof(void*) * static_cast<size_t>(count);
    off_a = o; o += ptrs;
    off_b = o; o += ptrs;
    off_c = o; o += ptrs;
    off_ipiv = o; o += ptrs;
    total = o;
  }
};

enum BatchKind { kBatchGetrf = 0, kBatchGetrs = 1, kBatchGemm = 2, kBatchTrsm = 3 };

// A launch configuration of the autotuner: the threads per CTA of the
// register-tiled FMA kernels (64, 128, 256; kDense128: 128 threads with
// registers capped for six CTAs an SM), or a tile shape of the FP64
// tensor-pipe GEMM that the routine's products use (kDmma32: 32 x 32 tiles,
// 4 warps; kDmma64: 64 x 64 tiles, 8 warps).
constexpr int kDmma32 = 1001, kDmma64 = 1002, kDense128 = 1128;

int ThreadsOf(int config) {
  return config == kDmma32     ? DmmaTile<2, 2, 2>::kThreads
         : config == kDmma64   ? DmmaTile<4, 2, 4>::kThreads
         : config == kDense128 ? 128
                               : config;
}

template <int Kind, typename T>
void* LuKernelOf(int config) {
  if constexpr (sizeof(T) == 8) {
    if (config == kDmma32) return reinterpret_cast<void*>(BatchedLuDmmaKernel<Kind, 2, 2, 2, 4>);
    if (config == kDmma64) return reinterpret_cast<void*>(BatchedLuDmmaKernel<Kind, 4, 2, 4, 3>);
  }
  if (config == 64) return reinterpret_cast<void*>(BatchedLuKernel<Kind, T, 64, 8>);
  if (config == 128) return reinterpret_cast<void*>(BatchedLuKernel<Kind, T, 128, 4>);
  if (config == kDense128) return reinterpret_cast<void*>(BatchedLuKernel<Kind, T, 128, 6>);
  return reinterpret_cast<void*>(BatchedLuKernel<Kind, T, 256, 3>);
}

template <typename T>
void* KernelOf(int kind, int config) {
  if (kind == kBatchGetrf) return LuKernelOf<kDevGetrf, T>(config);
  if (kind == kBatchGetrs) return LuKernelOf<kDevGetrs, T>(config);
  if (kind == kBatchTrsm) return LuKernelOf<kDevTrsm, T>(config);
  if (sizeof(T) == 8 && config == kDmma32)
    return reinterpret_cast<void*>(BatchedGemmDmmaKernel<2, 2, 2>);
  if (sizeof(T) == 8 && config == kDmma64)
    return reinterpret_cast<void*>(BatchedGemmDmmaKernel<4, 2, 4>);
  if (config == 64) return reinterpret_cast<void*>(BatchedGemmKernel<T, 64>);
  if (config == 128) return reinterpret_cast<void*>(BatchedGemmKernel<T, 128>);
  return reinterpret_cast<void*>(BatchedGemmKernel<T, 256>);
}

// The configurations the autotuner times for a routine and type: in FP64
// every routine also has the tensor-pipe variants for its products.
template <typename T>
std::vector<int> Candidates(int kind) {
  std::vector<int> c = {64, 128, 256};
  if (kind != kBatchGemm) c.push_back(kDense128);
  if (sizeof(T) == 8) {
    c.push_back(kDmma32);
    c.push_back(kDmma64);
  }
  return c;
}

// Threads per CTA for a batch: the autotuner's choice for the batch's size
// bucket (the log2 of the size that splits the batch's work in half),
// measured once per process on a sample of the batch (TunedConfig below).
struct TuneKey {
  int kind, bytes, bucket;
  bool operator<(const TuneKey& o) const {
    return std::tie(kind, bytes, bucket) < std::tie(o.kind, o.bytes, o.bucket);
  }
};

}  // namespace
}  // namespace hb

namespace hb {
namespace {

// Graphs of recent batch shapes (per host thread).
struct GraphKey {
  int kind, bytes, count, config, grid;
  void* dev;
  void* host;
  size_t total;
  double alpha, beta;
  int flags, lanes;
  cudaStream_t stream;
  bool operator==(const GraphKey& o) const {
    return kind == o.kind && bytes == o.bytes && count == o.count && config == o.config &&
           grid == o.grid && dev == o.dev && host == o.host && total == o.total &&
           alpha == o.alpha && beta == o.beta && flags == o.flags && lanes == o.lanes &&
           stream == o.stream;
  }
};
struct GraphEntry {
  GraphKey key;
  cudaGraphExec_t exec;
};
thread_local std::vector<GraphEntry> t_graphs;

// A batch as the host sees it: per-problem sizes and device pointers.
template <typename T>
struct HostBatch {
  int count = 0;
  std::vector<int> m, n, k, lda, ldb, ldc;
  std::vector<T*> a, b, c;
  std::vector<int*> ipiv;
  T alpha = T(1), beta = T(0);
  int flags = 0;
};

// Work of one problem, for the largest-first order.
template <typename T>
double WorkOf(int kind, const HostBatch<T>& bt, int i) {
  const double m = bt.m[i], n = bt.n.empty() ? 0 : bt.n[i];
  if (kind == kBatchGetrf) return m * m * m;
  if (kind == kBatchGetrs) return m * m * (n + 1);
  if (kind == kBatchTrsm) return m * n * (std::max(m, n) + 1);
  return m * n * (bt.k[i] + 1);
}

// Packs the descriptor, copies it to the device, launches the persistent
// kernel with `threads` threads a CTA. Problem info lands in dev_info (if
// non-null) on return of the stream.
template <typename T>
bool LaunchBatch(int kind, const HostBatch<T>& bt, int config, int** dev_info,
                 bool use_graph) {
  Context& ctx = Ctx();
  const int threads = ThreadsOf(config);
  const int count = bt.count;
  const Layout L(count);
  uint8_t* host = static_cast<uint8_t*>(t_stage.Get(L.total));
  uint8_t* dev = static_cast<uint8_t*>(Workspace(kWsBatch, L.total));
  if (host == nullptr || dev == nullptr) {
    Failed(cudaErrorMemoryAllocation, "batched descriptor");
    return false;
  }
  int* order = reinterpret_cast<int*>(host + L.off_order);
  std::iota(order, order + count, 0);
  std::vector<double> work(count);
  for (int i = 0; i < count; ++i) work[i] = WorkOf(kind, bt, i);
  std::stable_sort(order, order + count, [&](int x, int y) { return work[x] > work[y]; });
  std::memset(host + L.off_next, 0, 64);
  auto put_ints = [&](size_t off, const std::vector<int>& v) {
    if (!v.empty()) std::memcpy(host + off, v.data(), sizeof(int) * count);
  };
  put_ints(L.off_m, bt.m);
  put_ints(L.off_n, bt.n);
  put_ints(L.off_k, bt.k);
  put_ints(L.off_lda, bt.lda);
  put_ints(L.off_ldb, bt.ldb);
  put_ints(L.off_ldc, bt.ldc);
  auto put_ptrs = [&](size_t off, const void* src) {
    if (src != nullptr) std::memcpy(host + off, src, sizeof(void*) * count);
  };
  put_ptrs(L.off_a, bt.a.empty() ? nullptr : bt.a.data());
  put_ptrs(L.off_b, bt.b.empty() ? nullptr : bt.b.data());
  put_ptrs(L.off_c, bt.c.empty() ? nullptr : bt.c.data());
  put_ptrs(L.off_ipiv, bt.ipiv.empty() ? nullptr : bt.ipiv.data());
  BatchArgs<T> args;
  args.count = count;
  args.order = reinterpret_cast<const int*>(dev + L.off_order);
  args.next = reinterpret_cast<unsigned int*>(dev + L.off_next);
  args.m = reinterpret_cast<const int*>(dev + L.off_m);
  args.n = reinterpret_cast<const int*>(dev + L.off_n);
  args.k = reinterpret_cast<const int*>(dev + L.off_k);
  args.lda = reinterpret_cast<const int*>(dev + L.off_lda);
  args.ldb = reinterpret_cast<const int*>(dev + L.off_ldb);
  args.ldc = reinterpret_cast<const int*>(dev + L.off_ldc);
  args.a = reinterpret_cast<T* const*>(dev + L.off_a);
  args.b = reinterpret_cast<T* const*>(dev + L.off_b);
  args.c = reinterpret_cast<T* const*>(dev + L.off_c);
  args.ipiv = reinterpret_cast<int* const*>(dev + L.off_ipiv);
  args.info = reinterpret_cast<int*>(dev + L.off_info);
  args.alpha = bt.alpha;
  args.beta = bt.beta;
  args.flags = bt.flags;
  args.lanes = sizeof(T) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  void* fn = KernelOf<T>(kind, config);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0);
  const int grid = std::max(1, std::min(count, ctx.num_sms * std::max(per_sm, 1)));
  void* kargs[] = {&args};
  if (dev_info != nullptr) *dev_info = args.info;
  // The descriptor copy and the launch replay as one CUDA graph when the
  // same batch shape comes again (same workspace, staging buffer and kernel
  // arguments); the legacy default stream cannot be captured.
  if (use_graph && ctx.stream != nullptr) {
    GraphKey key{kind, static_cast<int>(sizeof(T)), count, config, grid, dev, host,
                 L.total, static_cast<double>(args.alpha), static_cast<double>(args.beta),
                 args.flags, args.lanes, ctx.stream};
    for (auto& e : t_graphs) {
      if (e.key == key) {
        if (Failed(cudaGraphLaunch(e.exec, ctx.stream), "batched graph launch")) return false;
        CountLaunch();
        return true;
      }
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal) ==
              cudaSuccess;
    if (ok) {
      cudaMemcpyAsync(dev, host, L.total, cudaMemcpyHostToDevice, ctx.stream);
      cudaLaunchKernel(fn, grid, threads, kargs, 0, ctx.stream);
      ok = cudaStreamEndCapture(ctx.stream, &graph) == cudaSuccess && graph != nullptr &&
           cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
      if (graph != nullptr) cudaGraphDestroy(graph);
    }
    if (ok) {
      if (t_graphs.size() >= 8) {
        cudaGraphExecDestroy(t_graphs.front().exec);
        t_graphs.erase(t_graphs.begin());
      }
      t_graphs.push_back({key, exec});
      if (Failed(cudaGraphLaunch(exec, ctx.stream), "batched graph launch")) return false;
      CountLaunch();
      return true;
    }
    cudaGetLastError();  // capture unavailable: launch directly
  }
  if (Failed(cudaMemcpyAsync(dev, host, L.total, cudaMemcpyHostToDevice, ctx.stream),
             "batched descriptor copy"))
    return false;
  if (Failed(cudaLaunchKernel(fn, grid, threads, kargs, 0, ctx.stream), "batched launch"))
    return false;
  CountLaunch();
  return true;
}

// Uniform values in [-1, 1) from a hash of the index.
template <typename T>
__global__ void FillRandomKernel(T* x, long long count, unsigned seed) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < count; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    unsigned h = static_cast<unsigned>(i) * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    x[i] = static_cast<T>((h & 0xffffff) / 8388608.0 - 1.0);
  }
}

// Adds dim[p] to the diagonal of the dim[p] x dim[p] matrix at base + off[p]
// (leading dimension dim[p]): a triangular factor that stays well conditioned.
template <typename T>
__global__ void BoostDiagonalKernel(T* base, const long long* off, const int* dim, int count) {
  for (int p = blockIdx.x; p < count; p += gridDim.x) {
    T* a = base + off[p];
    const int d = dim[p];
    for (int j = threadIdx.x; j < d; j += blockDim.x)
      a[j + static_cast<long long>(j) * d] += static_cast<T>(d);
  }
}

// The autotuner: for (routine, type, size bucket), the launch configuration
// (Candidates above) that runs a replica of the batch itself fastest: the
// batch's own problem sizes (all of them, or every stride-th in largest-first
// order for a batch too large to copy), on synthetic operands with tight
// leading dimensions. Results do not depend on
// the choice: every problem's arithmetic is the same whichever configuration
// runs it.
// A configuration set by hwyblas_batched_set_config (0: the autotuner's).
std::atomic<int> g_forced_config{0};

template <typename T>
int TunedConfig(int kind, const HostBatch<T>& real, int work_median) {
  const int forced = g_forced_config.load(std::memory_order_relaxed);
  if (forced != 0) {
    for (int c : Candidates<T>(kind))
      if (c == forced) return c;
  }
  static std::mutex mu;
  static std::map<TuneKey, int> cache;
  int bucket = 0;
  while ((2 << bucket) <= std::max(1, work_median)) ++bucket;
  const TuneKey key{kind, static_cast<int>(sizeof(T)), bucket};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  // Per-problem operand shapes with tight leading dimensions: A (rows x
  // cols), B and C (rows x n), and the pivot vector.
  struct Shape {
    int m, n, k, ra, ca, rb, cb, rc, cc, piv;
  };
  const bool right = kind == kBatchTrsm && (real.flags & 1);
  auto shape_of = [&](int i) {
    Shape s{};
    s.m = real.m[i];
    s.n = real.n.empty() ? 0 : real.n[i];
    s.k = real.k.empty() ? 0 : real.k[i];
    if (kind == kBatchGemm) {
      const bool ta = real.flags & 1, tb = real.flags & 2;
      s.ra = ta ? s.k : s.m, s.ca = ta ? s.m : s.k;
      s.rb = tb ? s.n : s.k, s.cb = tb ? s.k : s.n;
      s.rc = s.m, s.cc = s.n;
    } else {
      const int t = right ? s.n : s.m;
      s.ra = t, s.ca = t;
      if (kind != kBatchGetrf) s.rb = s.m, s.cb = s.n;
      if (kind != kBatchTrsm) s.piv = s.m;
    }
    return s;
  };
  auto round_up = [](size_t x) { return (x + 31) / 32 * 32; };  // 256-byte starts
  std::vector<int> order(real.count);
  std::iota(order.begin(), order.end(), 0);
  std::vector<double> work(real.count);
  size_t total = 0;
  for (int i = 0; i < real.count; ++i) {
    work[i] = WorkOf(kind, real, i);
    const Shape s = shape_of(i);
    total += sizeof(T) * (round_up(size_t(s.ra) * s.ca) + round_up(size_t(s.rb) * s.cb) +
                          round_up(size_t(s.rc) * s.cc));
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return work[x] > work[y]; });
  // The whole batch when its operands fit a quarter of the free memory (at
  // most 16 GB): a batch's time is the larger of the throughput bound and
  // the latency of its largest problem on one CTA, and a thinned sample
  // shifts that balance (it keeps the largest problem but not the work
  // around it). Beyond that, every stride-th problem.
  size_t free_bytes = 0, total_bytes = 0;
  if (cudaMemGetInfo(&free_bytes, &total_bytes) != cudaSuccess) free_bytes = size_t(4) << 30;
  const size_t budget = std::max<size_t>(size_t(256) << 20,
                                         std::min<size_t>(free_bytes / 4, size_t(16) << 30));
  const size_t stride = std::max<size_t>(1, (total + budget - 1) / budget);
  std::vector<Shape> sample;
  for (size_t q = 0; q < order.size(); q += stride) sample.push_back(shape_of(order[q]));
  const int S = static_cast<int>(sample.size());
  std::vector<long long> off_a(S), off_b(S), off_c(S), off_p(S);
  std::vector<int> dim_a(S);
  size_t na = 0, nb = 0, nc = 0, np = 0;
  for (int i = 0; i < S; ++i) {
    const Shape& s = sample[i];
    off_a[i] = static_cast<long long>(na), na += round_up(size_t(s.ra) * s.ca);
    off_b[i] = static_cast<long long>(nb), nb += round_up(size_t(s.rb) * s.cb);
    off_c[i] = static_cast<long long>(nc), nc += round_up(size_t(s.rc) * s.cc);
    off_p[i] = static_cast<long long>(np), np += round_up(size_t(s.piv));
    dim_a[i] = s.ra;
  }
  Context& ctx = Ctx();
  T *A = nullptr, *B = nullptr, *C = nullptr;
  int* P = nullptr;
  long long* d_off = nullptr;
  int* d_dim = nullptr;
  int best = 256;
  if (cudaMalloc(&A, sizeof(T) * std::max<size_t>(na, 1)) == cudaSuccess &&
      cudaMalloc(&B, sizeof(T) * std::max<size_t>(nb, 1)) == cudaSuccess &&
      cudaMalloc(&C, sizeof(T) * std::max<size_t>(nc, 1)) == cudaSuccess &&
      cudaMalloc(&P, sizeof(int) * std::max<size_t>(np, 1)) == cudaSuccess &&
      cudaMalloc(&d_off, sizeof(long long) * S) == cudaSuccess &&
      cudaMalloc(&d_dim, sizeof(int) * S) == cudaSuccess) {
    HostBatch<T> bt;
    bt.count = S;
    bt.alpha = real.alpha;
    bt.beta = real.beta;
    bt.flags = real.flags;
    for (int i = 0; i < S; ++i) {
      const Shape& s = sample[i];
      bt.m.push_back(s.m);
      if (!real.n.empty()) bt.n.push_back(s.n);
      if (!real.k.empty()) bt.k.push_back(s.k);
      bt.lda.push_back(std::max(1, s.ra));
      bt.a.push_back(A + off_a[i]);
      if (!real.b.empty()) {
        bt.ldb.push_back(std::max(1, s.rb));
        bt.b.push_back(B + off_b[i]);
      }
      if (!real.c.empty()) {
        bt.ldc.push_back(std::max(1, s.rc));
        bt.c.push_back(C + off_c[i]);
      }
      if (!real.ipiv.empty()) bt.ipiv.push_back(P + off_p[i]);
    }
    if (kind == kBatchGetrs) {
      // Valid pivots for the solve: the identity.
      std::vector<int> ident(std::max<size_t>(np, 1), 1);
      for (int i = 0; i < S; ++i)
        for (int r = 0; r < sample[i].piv; ++r) ident[off_p[i] + r] = r + 1;
      cudaMemcpy(P, ident.data(), sizeof(int) * ident.size(), cudaMemcpyHostToDevice);
    }
    // A once (the solves and products only read it; the LU refills it below).
    FillRandomKernel<<<1024, 256, 0, ctx.stream>>>(A, static_cast<long long>(na), 7u);
    if (kind == kBatchGetrs || kind == kBatchTrsm) {
      cudaMemcpyAsync(d_off, off_a.data(), sizeof(long long) * S, cudaMemcpyHostToDevice,
                      ctx.stream);
      cudaMemcpyAsync(d_dim, dim_a.data(), sizeof(int) * S, cudaMemcpyHostToDevice,
                      ctx.stream);
      BoostDiagonalKernel<<<std::min(S, 4096), 256, 0, ctx.stream>>>(A, d_off, d_dim, S);
    }
    FillRandomKernel<<<1024, 256, 0, ctx.stream>>>(C, static_cast<long long>(nc), 11u);
    // Fresh operands before every run: the LU and the solves work in place,
    // and a factored matrix pivots differently from a random one.
    auto refill = [&]() {
      if (kind == kBatchGetrf)
        FillRandomKernel<<<1024, 256, 0, ctx.stream>>>(A, static_cast<long long>(na), 7u);
      if (kind != kBatchGetrf)
        FillRandomKernel<<<1024, 256, 0, ctx.stream>>>(B, static_cast<long long>(nb), 9u);
    };
    const std::vector<int> configs = Candidates<T>(kind);
    for (int config : configs) {  // untimed: first launches of every kernel
      refill();
      LaunchBatch(kind, bt, config, nullptr, false);
    }
    cudaStreamSynchronize(ctx.stream);
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<float> times(configs.size(), 1e30f);
    for (int rep = 0; rep < 2; ++rep) {
      for (size_t c = 0; c < configs.size(); ++c) {
        refill();
        cudaEventRecord(e0, ctx.stream);
        LaunchBatch(kind, bt, configs[c], nullptr, false);
        cudaEventRecord(e1, ctx.stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        times[c] = std::min(times[c], ms);
        if (ms < best_ms) {
          best_ms = ms;
          best = configs[c];
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // HWYBLAS_TUNE_LOG=1: one line per tuning on stderr (routine, type size,
    // bucket, sample size, each configuration's time, the choice).
    const char* log = getenv("HWYBLAS_TUNE_LOG");
    if (log != nullptr && log[0] != '\0' && log[0] != '0') {
      std::fprintf(stderr, "hwyblas tune: kind %d bytes %d bucket %d sample %d/%d:", kind,
                   static_cast<int>(sizeof(T)), bucket, S, real.count);
      for (size_t c = 0; c < configs.size(); ++c)
        std::fprintf(stderr, " %d=%.3fms", configs[c], times[c]);
      std::fprintf(stderr, " -> %d\n", best);
    }
  }
  cudaStreamSynchronize(ctx.stream);
  cudaFree(A);
  cudaFree(B);
  cudaFree(C);
  cudaFree(P);
  cudaFree(d_off);
  cudaFree(d_dim);
  cudaGetLastError();
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = best;
  return best;
}

// The size that splits the batch's work in half: problems at least this
// large hold half of it. The batch's time follows these problems, so the
// autotuner measures at this size rather than at the median count.
template <typename T>
int WorkMedian(int kind, const HostBatch<T>& bt) {
  std::vector<std::pair<int, double>> w(bt.count);
  double total = 0.0;
  for (int i = 0; i < bt.count; ++i) {
    w[i] = {bt.m[i], WorkOf(kind, bt, i)};
    total += w[i].second;
  }
  std::sort(w.begin(), w.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  double acc = 0.0;
  for (const auto& e : w) {
    acc += e.second;
    if (acc >= 0.5 * total) return e.first;
  }
  return w.empty() ? 0 : w.back().first;
}

}  // namespace
}  // namespace hb

namespace hb {
namespace {

// Runs a validated batch: autotuned launch, then (getrf) the per-problem
// INFO back to the host. Synchronous, like the single-problem routines.
template <typename T>
void RunBatch(int kind, const HostBatch<T>& bt, int* info_out, const char* name) {
  if (bt.count == 0) return;
  const int config = TunedConfig<T>(kind, bt, WorkMedian(kind, bt));
  int* dev_info = nullptr;
  if (!LaunchBatch(kind, bt, config, &dev_info, true)) return;
  LaunchFailed(name);
  if (info_out != nullptr) {
    Failed(cudaMemcpyAsync(info_out, dev_info, sizeof(int) * bt.count,
                           cudaMemcpyDeviceToHost, Ctx().stream),
           "batched info");
  }
  Failed(cudaStreamSynchronize(Ctx().stream), name);
  CheckDeviceStatus(name);
}

template <typename T>
void GetrfBatched(const int* n, T* const* a, const int* lda, int* const* ipiv, int* info,
                  int count, const char* name) {
  if (count < 0) {
    ReportError(name, 6);
    return;
  }
  HostBatch<T> bt;
  bt.count = count;
  ExtentChecker ext;
  for (int i = 0; i < count; ++i) {
    if (n[i] < 0) { ReportError(name, 1); return; }
    if (lda[i] < std::max(1, n[i])) { ReportError(name, 3); return; }
    const size_t elems = n[i] == 0 ? 0 : static_cast<size_t>(lda[i]) * (n[i] - 1) + n[i];
    if (!ext.Check(a[i], sizeof(T) * elems)) { ReportError(name, 2); return; }
    if (!ext.Check(ipiv[i], sizeof(int) * n[i])) { ReportError(name, 4); return; }
  }
  bt.m.assign(n, n + count);
  bt.lda.assign(lda, lda + count);
  bt.a.assign(a, a + count);
  bt.ipiv.assign(ipiv, ipiv + count);
  RunBatch(kBatchGetrf, bt, info, name);
}

template <typename T>
void GetrsBatched(char trans, const int* n, const int* nrhs, T* const* a, const int* lda,
                  int* const* ipiv, T* const* b, const int* ldb, int count, int* info,
                  const char* name) {
  *info = 0;
  const char t = (trans >= 'a' && trans <= 'z') ? static_cast<char>(trans - 32) : trans;
  if (t != 'N' && t != 'T' && t != 'C') *info = -1;
  else if (count < 0) *info = -9;
  HostBatch<T> bt;
  ExtentChecker ext;
  for (int i = 0; *info == 0 && i < count; ++i) {
    if (n[i] < 0) *info = -2;
    else if (nrhs[i] < 0) *info = -3;
    else if (lda[i] < std::max(1, n[i])) *info = -5;
    else if (ldb[i] < std::max(1, n[i])) *info = -8;
    else {
      const size_t ea = n[i] == 0 ? 0 : static_cast<size_t>(lda[i]) * (n[i] - 1) + n[i];
      const size_t eb = (n[i] == 0 || nrhs[i] == 0)
                            ? 0 : static_cast<size_t>(ldb[i]) * (nrhs[i] - 1) + n[i];
      if (!ext.Check(a[i], sizeof(T) * ea)) *info = -4;
      else if (!ext.Check(ipiv[i], sizeof(int) * n[i])) *info = -6;
      else if (!ext.Check(b[i], sizeof(T) * eb)) *info = -7;
    }
  }
  if (*info != 0) {
    ReportError(name, -*info);
    return;
  }
  bt.count = count;
  bt.m.assign(n, n + count);
  bt.n.assign(nrhs, nrhs + count);
  bt.lda.assign(lda, lda + count);
  bt.ldb.assign(ldb, ldb + count);
  bt.a.assign(a, a + count);
  bt.b.assign(b, b + count);
  bt.ipiv.assign(ipiv, ipiv + count);
  bt.flags = (t == 'N') ? 0 : 1;
  RunBatch(kBatchGetrs, bt, nullptr, name);
}

template <typename T>
void TrsmBatched(char side, char uplo, char transa, char diag, const int* m, const int* n,
                 T alpha, T* const* a, const int* lda, T* const* b, const int* ldb,
                 int count, const char* name) {
  auto up = [](char ch) { return (ch >= 'a' && ch <= 'z') ? static_cast<char>(ch - 32) : ch; };
  const char sd = up(side), ul = up(uplo), ta = up(transa), dg = up(diag);
  int pos = 0;
  if (sd != 'L' && sd != 'R') pos = 1;
  else if (ul != 'L' && ul != 'U') pos = 2;
  else if (ta != 'N' && ta != 'T' && ta != 'C') pos = 3;
  else if (dg != 'N' && dg != 'U') pos = 4;
  else if (count < 0) pos = 12;
  ExtentChecker ext;
  for (int i = 0; pos == 0 && i < count; ++i) {
    const int ka = sd == 'L' ? m[i] : n[i];
    if (m[i] < 0) pos = 5;
    else if (n[i] < 0) pos = 6;
    else if (lda[i] < std::max(1, ka)) pos = 9;
    else if (ldb[i] < std::max(1, m[i])) pos = 11;
    else if (m[i] > 0 && n[i] > 0) {
      const size_t ea = alpha == T(0) ? 0 : static_cast<size_t>(lda[i]) * (ka - 1) + ka;
      const size_t eb = static_cast<size_t>(ldb[i]) * (n[i] - 1) + m[i];
      if (!ext.Check(a[i], sizeof(T) * ea)) pos = 8;
      else if (!ext.Check(b[i], sizeof(T) * eb)) pos = 10;
    }
  }
  if (pos != 0) {
    ReportError(name, pos);
    return;
  }
  HostBatch<T> bt;
  bt.count = count;
  bt.m.assign(m, m + count);
  bt.n.assign(n, n + count);
  bt.lda.assign(lda, lda + count);
  bt.ldb.assign(ldb, ldb + count);
  bt.a.assign(a, a + count);
  bt.b.assign(b, b + count);
  bt.alpha = alpha;
  bt.flags = (sd == 'R' ? 1 : 0) | (ul == 'L' ? 2 : 0) | (ta != 'N' ? 4 : 0) |
             (dg == 'U' ? 8 : 0);
  RunBatch(kBatchTrsm, bt, nullptr, name);
}

template <typename T>
void GemmBatched(char transa, char transb, const int* m, const int* n, const int* k,
                 T alpha, T* const* a, const int* lda, T* const* b, const int* ldb, T beta,
                 T* const* c, const int* ldc, int count, const char* name) {
  auto up = [](char ch) { return (ch >= 'a' && ch <= 'z') ? static_cast<char>(ch - 32) : ch; };
  const char ta = up(transa), tb = up(transb);
  int pos = 0;
  if (ta != 'N' && ta != 'T' && ta != 'C') pos = 1;
  else if (tb != 'N' && tb != 'T' && tb != 'C') pos = 2;
  else if (count < 0) pos = 14;
  ExtentChecker ext;
  for (int i = 0; pos == 0 && i < count; ++i) {
    const bool tra = ta != 'N', trb = tb != 'N';
    const int ra = tra ? k[i] : m[i], ca = tra ? m[i] : k[i];
    const int rb = trb ? n[i] : k[i], cb = trb ? k[i] : n[i];
    if (m[i] < 0) pos = 3;
    else if (n[i] < 0) pos = 4;
    else if (k[i] < 0) pos = 5;
    else if (lda[i] < std::max(1, ra)) pos = 8;
    else if (ldb[i] < std::max(1, rb)) pos = 10;
    else if (ldc[i] < std::max(1, m[i])) pos = 13;
    else if (m[i] > 0 && n[i] > 0) {
      const bool compute = k[i] > 0 && alpha != T(0);
      const size_t ea = (!compute || ra == 0 || ca == 0) ? 0
                        : static_cast<size_t>(lda[i]) * (ca - 1) + ra;
      const size_t eb = (!compute || rb == 0 || cb == 0) ? 0
                        : static_cast<size_t>(ldb[i]) * (cb - 1) + rb;
      const size_t ec = static_cast<size_t>(ldc[i]) * (n[i] - 1) + m[i];
      if (!ext.Check(a[i], sizeof(T) * ea)) pos = 7;
      else if (!ext.Check(b[i], sizeof(T) * eb)) pos = 9;
      else if (!ext.Check(c[i], sizeof(T) * ec)) pos = 12;
    }
  }
  if (pos != 0) {
    ReportError(name, pos);
    return;
  }
  HostBatch<T> bt;
  bt.count = count;
  bt.m.assign(m, m + count);
  bt.n.assign(n, n + count);
  bt.k.assign(k, k + count);
  bt.lda.assign(lda, lda + count);
  bt.ldb.assign(ldb, ldb + count);
  bt.ldc.assign(ldc, ldc + count);
  bt.a.assign(a, a + count);
  bt.b.assign(b, b + count);
  bt.c.assign(c, c + count);
  bt.alpha = alpha;
  bt.beta = beta;
  bt.flags = (ta != 'N' ? 1 : 0) | (tb != 'N' ? 2 : 0);
  RunBatch(kBatchGemm, bt, nullptr, name);
}

}  // namespace
}  // namespace hb

extern "C" {

HWYBLAS_API int hwyblas_batched_set_config(int config) {
  return hb::g_forced_config.exchange(config);
}

HWYBLAS_API void hwyblas_dgetrf_batched(const hwyblas_int* n, double* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        hwyblas_int* info, hwyblas_int count) {
  hb::GetrfBatched<double>(n, a, lda, ipiv, info, count, "DGETRF_BATCHED");
}

HWYBLAS_API void hwyblas_sgetrf_batched(const hwyblas_int* n, float* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        hwyblas_int* info, hwyblas_int count) {
  hb::GetrfBatched<float>(n, a, lda, ipiv, info, count, "SGETRF_BATCHED");
}

HWYBLAS_API void hwyblas_dgetrs_batched(char trans, const hwyblas_int* n,
                                        const hwyblas_int* nrhs, double* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        double* const* b, const hwyblas_int* ldb,
                                        hwyblas_int count, hwyblas_int* info) {
  hb::GetrsBatched<double>(trans, n, nrhs, a, lda, ipiv, b, ldb, count, info,
                           "DGETRS_BATCHED");
}

HWYBLAS_API void hwyblas_sgetrs_batched(char trans, const hwyblas_int* n,
                                        const hwyblas_int* nrhs, float* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        float* const* b, const hwyblas_int* ldb,
                                        hwyblas_int count, hwyblas_int* info) {
  hb::GetrsBatched<float>(trans, n, nrhs, a, lda, ipiv, b, ldb, count, info,
                          "SGETRS_BATCHED");
}

HWYBLAS_API void hwyblas_dtrsm_batched(char side, char uplo, char transa, char diag,
                                       const hwyblas_int* m, const hwyblas_int* n,
                                       double alpha, double* const* a,
                                       const hwyblas_int* lda, double* const* b,
                                       const hwyblas_int* ldb, hwyblas_int count) {
  hb::TrsmBatched<double>(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, count,
                          "DTRSM_BATCHED");
}

HWYBLAS_API void hwyblas_strsm_batched(char side, char uplo, char transa, char diag,
                                       const hwyblas_int* m, const hwyblas_int* n,
                                       float alpha, float* const* a,
                                       const hwyblas_int* lda, float* const* b,
                                       const hwyblas_int* ldb, hwyblas_int count) {
  hb::TrsmBatched<float>(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, count,
                         "STRSM_BATCHED");
}

HWYBLAS_API void hwyblas_dgemm_batched(char transa, char transb, const hwyblas_int* m,
                                       const hwyblas_int* n, const hwyblas_int* k,
                                       double alpha, double* const* a,
                                       const hwyblas_int* lda, double* const* b,
                                       const hwyblas_int* ldb, double beta,
                                       double* const* c, const hwyblas_int* ldc,
                                       hwyblas_int count) {
  hb::GemmBatched<double>(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                          count, "DGEMM_BATCHED");
}

HWYBLAS_API void hwyblas_sgemm_batched(char transa, char transb, const hwyblas_int* m,
                                       const hwyblas_int* n, const hwyblas_int* k,
                                       float alpha, float* const* a,
                                       const hwyblas_int* lda, float* const* b,
                                       const hwyblas_int* ldb, float beta,
                                       float* const* c, const hwyblas_int* ldc,
                                       hwyblas_int count) {
  hb::GemmBatched<float>(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                         count, "SGEMM_BATCHED");
}

}  // extern "C"
