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
// The triangle of a base solve in shared memory, in solve order, and the
// reciprocals of its diagonal (the CTA's threads share the loads).
template <typename T>
__device__ void LoadBaseTriangle(View<T> tri, int lower, int unit, int r, T (*st)[33],
                                 T* sinv) {
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
}

// One row of X: loads through L2 only when kCg (rows written by other CTAs
// in an earlier step of a cooperative launch).
template <typename T, bool kCg>
__device__ __forceinline__ T LoadX(const T* p) {
  if constexpr (kCg) return __ldcg(p);
  return *p;
}
template <typename T, bool kCg>
__device__ __forceinline__ void StoreX(T* p, T v) {
  if constexpr (kCg) __stcg(p, v);
  else *p = v;
}

template <typename T, bool kCg>
__device__ __forceinline__ void BaseSolveRow(const T (*st)[33], const T* sinv, int lower,
                                             int unit, int r, T* xr, long long xs_col) {
  T y[32];
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) y[s] = LoadX<T, kCg>(xr + (lower ? r - 1 - s : s) * xs_col);
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
#pragma unroll
  for (int s = 0; s < 32; ++s) {
    if (s < r) StoreX<T, kCg>(xr + (lower ? r - 1 - s : s) * xs_col, y[s]);
  }
}

template <typename T>
__global__ void __launch_bounds__(128)
    TrsmBaseKernel(View<T> tri, int lower, int unit, int r, int rows, T* x,
                   long long xs_row, long long xs_col, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ T st[32][33];  // st[s][u] = T(col(s), col(u)) in solve order
  __shared__ T sinv[32];
  LoadBaseTriangle(tri, lower, unit, r, st, sinv);
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  BaseSolveRow<T, false>(st, sinv, lower, unit, r, x + row * xs_row, xs_col);
}

// Cooperative TRSM of a subtree of the recursion (at most kTcRows rows of
// the triangle, at most TcOther right-hand sides): all of its base solves
// and updates in one launch, in TrsmRec's order, with a bounded grid barrier
// after each step; below that size the recursion is a chain of small
// dependent launches. (n = 16384, one right-hand side: 22 -> 12 ms a
// triangle; 64: 21 -> 12 ms.) A base step solves the `other` rows of X, one a
// thread, with the 32 x 32 triangle in every CTA's shared memory; an update
// step gives each thread C elements, each the reference's FMA chain over k
// restarted every KC and merged in order (alpha -1, beta 1), as the GEMM
// kernels compute it. X is read and written through L2 only: its rows
// change owner between steps.
constexpr int kTcRows = 512, kTcThreads = 256;
// Right-hand sides of the cooperative path: up to 64 on the staged FMA
// chains; in FP64 up to 1024, with the updates on the tensor pipe from 32.
template <typename T>
constexpr int TcOther() { return sizeof(T) == 8 ? 1024 : 64; }

template <typename T>
struct KcOf {
  static constexpr int value = sizeof(T) == 8 ? 256 : 384;
};

template <typename T>
__device__ __forceinline__ View<T> SubView(View<T> v, long long i, long long j) {
  v.data += i * v.rs + j * v.cs;
  return v;
}

template <typename T>
struct TrsmCoopArgs {
  View<T> tri;
  int left, lower, unit, r, other;
  T* b;
  long long ldb;
  unsigned int* barrier;
  int* timeout_flag;
  const int* guard;
};

// C (mm x nn) -= A (mm x kk) B (kk x nn), kk <= 2 KC (all strided views;
// element (i, j) of a view at data[i rs + j cs]). Each element's chain is
// sequential, so its operands are staged first: a CTA takes blocks of
// kTcRowsCta rows by kTcColsCta columns of C, copies those rows of A and
// columns of B (all kk) into shared memory, then each thread runs its
// elements' chains from there. The staging is wide and independent of the
// chains, which then wait on no memory.
constexpr int kTcRowsCta = 32, kTcColsCta = 16;
constexpr int kTcKMax = 512;  // update depth within a subtree of kTcRows rows
template <typename T>
__device__ void CoopUpdate(int mm, int nn, int kk, View<T> a, View<T> bv, View<T> cv_,
                           T* sa, T* sb) {
  constexpr int KC = KcOf<T>::value;
  const int rgroups = (mm + kTcRowsCta - 1) / kTcRowsCta;
  const int items = rgroups * ((nn + kTcColsCta - 1) / kTcColsCta);
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int i0 = (item % rgroups) * kTcRowsCta, rows = min(kTcRowsCta, mm - i0);
    const int j0 = (item / rgroups) * kTcColsCta, cols = min(kTcColsCta, nn - j0);
    __syncthreads();  // the previous block's reads are done
    // sa[q * 32 + il] = A(i0 + il, q); sb[q * 16 + jl] = B(q, j0 + jl)
    for (int idx = threadIdx.x; idx < kk * kTcRowsCta; idx += blockDim.x) {
      const int il = idx % kTcRowsCta, q = idx / kTcRowsCta;
      sa[idx] = il < rows ? __ldcg(a.data + (i0 + il) * a.rs + q * a.cs) : T(0);
    }
    for (int idx = threadIdx.x; idx < kk * kTcColsCta; idx += blockDim.x) {
      const int jl = idx % kTcColsCta, q = idx / kTcColsCta;
      sb[idx] = jl < cols ? __ldcg(bv.data + q * bv.rs + (j0 + jl) * bv.cs) : T(0);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
      const int il = e % rows, jl = e / rows;
      T* cij = const_cast<T*>(cv_.data) + (i0 + il) * cv_.rs + (j0 + jl) * cv_.cs;
      T cv = __ldcg(cij);
      for (int pc = 0; pc < kk; pc += KC) {
        const int pe = min(kk, pc + KC);
        T acc = T(0);
        for (int q = pc; q < pe; ++q)
          acc = fma(sa[q * kTcRowsCta + il], sb[q * kTcColsCta + jl], acc);
        const T r = T(-1) * acc;
        cv = r + cv;
      }
      __stcg(cij, cv);
    }
  }
}

// The same update on the FP64 tensor pipe for many right-hand sides: blocks
// of 32 x 32 of C, the CTA's 8 warps one 16 x 8 tile each, k staged in
// 64-deep chunks (A and B padded to 36 doubles a row, conflict-free
// fragments) and each tile's m16n8k8 chain restarted every KC = 256 and
// merged in order: every element's chain and merges are CoopUpdate's.
constexpr int kTcDmmaB = 32, kTcDmmaKb = 64, kTcDmmaLd = kTcDmmaB + 4;
__device__ void CoopUpdateDmma(int mm, int nn, int kk, View<double> a, View<double> bv,
                               View<double> cv_, double* sa, double* sb) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp % 2, wc = warp / 2;  // tile rows 16 wr, columns 8 wc
  const int rgroups = (mm + kTcDmmaB - 1) / kTcDmmaB;
  const int items = rgroups * ((nn + kTcDmmaB - 1) / kTcDmmaB);
  for (int item = blockIdx.x; item < items; item += gridDim.x) {
    const int i0 = (item % rgroups) * kTcDmmaB, j0 = (item / rgroups) * kTcDmmaB;
    // This thread's four elements (the m16n8 accumulator layout) and their C.
    double cv[4], acc[4] = {0.0, 0.0, 0.0, 0.0};
    bool in[4];
    double* cp[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = i0 + wr * 16 + g + (e >> 1) * 8, j = j0 + wc * 8 + 2 * t + (e & 1);
      in[e] = i < mm && j < nn;
      cp[e] = const_cast<double*>(cv_.data) + i * cv_.rs + j * cv_.cs;
      cv[e] = in[e] ? __ldcg(cp[e]) : 0.0;
    }
    for (int k0 = 0; k0 < kk; k0 += kTcDmmaKb) {
      __syncthreads();  // the previous chunk's fragments are read
      // sa[q * 36 + il] = A(i0 + il, k0 + q); sb[q * 36 + jl] = B(k0 + q, j0 + jl)
      for (int idx = threadIdx.x; idx < kTcDmmaKb * kTcDmmaB; idx += blockDim.x) {
        const int l = idx % kTcDmmaB, q = idx / kTcDmmaB;
        const bool kq = k0 + q < kk;
        sa[q * kTcDmmaLd + l] = (kq && i0 + l < mm)
                                    ? __ldcg(a.data + (i0 + l) * a.rs + (k0 + q) * a.cs)
                                    : 0.0;
        sb[q * kTcDmmaLd + l] = (kq && j0 + l < nn)
                                    ? __ldcg(bv.data + (k0 + q) * bv.rs + (j0 + l) * bv.cs)
                                    : 0.0;
      }
      __syncthreads();
      const int steps = (min(kTcDmmaKb, kk - k0) + 7) / 8;
      for (int ks = 0; ks < steps; ++ks) {
        const double* pa = sa + (ks * 8 + t) * kTcDmmaLd + wr * 16 + g;
        const double* pb = sb + (ks * 8 + t) * kTcDmmaLd + wc * 8 + g;
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
            "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
            : "+d"(acc[0]), "+d"(acc[1]), "+d"(acc[2]), "+d"(acc[3])
            : "d"(pa[0]), "d"(pa[8]), "d"(pa[4 * kTcDmmaLd]), "d"(pa[4 * kTcDmmaLd + 8]),
              "d"(pb[0]), "d"(pb[4 * kTcDmmaLd]));
      }
      // End of a KC chunk (or of k): merge alpha * acc = -acc, restart.
      if ((k0 + kTcDmmaKb) % 256 == 0 || k0 + kTcDmmaKb >= kk) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double r = -1.0 * acc[e];
          cv[e] = r + cv[e];
          acc[e] = 0.0;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (in[e]) __stcg(cp[e], cv[e]);
  }
}

// The update of a cooperative step: the tensor-pipe tiles in FP64 when the
// right-hand sides fill them, else the staged FMA chains.
template <typename T>
__device__ __forceinline__ void CoopStep(int mm, int nn, int kk, View<T> a, View<T> bv,
                                         View<T> c, T* sa, T* sb) {
  if constexpr (sizeof(T) == 8) {
    if (nn >= kTcDmmaB) {
      CoopUpdateDmma(mm, nn, kk, a, bv, c, sa, sb);
      return;
    }
  }
  CoopUpdate(mm, nn, kk, a, bv, c, sa, sb);
}

template <typename T>
__global__ void __launch_bounds__(kTcThreads) TrsmCoopKernel(TrsmCoopArgs<T> p) {
  if (p.guard != nullptr && *p.guard != 0) return;
  __shared__ T st[32][33];
  __shared__ T sinv[32];
  extern __shared__ __align__(16) unsigned char tc_smem[];
  T* sa = reinterpret_cast<T*>(tc_smem);   // kTcKMax x kTcRowsCta
  T* sb = sa + kTcKMax * kTcRowsCta;       // kTcKMax x kTcColsCta
  const long long tid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long nth = static_cast<long long>(gridDim.x) * blockDim.x;
  const auto col = [&](T* x, long long ld) {  // column-major, element (i, j) at x[i + j ld]
    View<T> v;
    v.data = x;
    v.rs = 1;
    v.cs = ld;
    return v;
  };
  const auto row = [&](T* x, long long ld) {  // its transpose, element (i, j) at x[j + i ld]
    View<T> v;
    v.data = x;
    v.rs = ld;
    v.cs = 1;
    return v;
  };
  // Which half TrsmRec solves first: t11 for left-lower and right-upper.
  const bool first11 = (p.left != 0) == (p.lower != 0);
  int s_off[8], s_r[8], s_ph[8];
  int sp = 0;
  s_off[0] = 0;
  s_r[0] = p.r;
  s_ph[0] = 0;
  unsigned int gen = 0;
  while (sp >= 0) {
    const int off = s_off[sp], rr = s_r[sp];
    if (rr <= 32) {
      View<T> t = SubView(p.tri, off, off);
      int lo = p.lower;
      long long xs_row, xs_col;
      T* xb;
      if (p.left) {  // T X = B as X^T T^T = B^T: rows of X^T are B's columns
        const long long rs = t.rs;
        t.rs = t.cs;
        t.cs = rs;
        lo = !lo;
        xs_row = p.ldb;
        xs_col = 1;
        xb = p.b + off;
      } else {
        xs_row = 1;
        xs_col = p.ldb;
        xb = p.b + static_cast<long long>(off) * p.ldb;
      }
      LoadBaseTriangle(t, lo, p.unit, rr, st, sinv);
      for (long long row = tid; row < p.other; row += nth)
        BaseSolveRow<T, true>(st, sinv, lo, p.unit, rr, xb + row * xs_row, xs_col);
      --sp;
      if (!GridBarrier(p.barrier, gridDim.x, ++gen, p.timeout_flag)) return;
      continue;
    }
    const int r1 = max(32, (rr / 2) / 32 * 32), r2 = rr - r1;
    const int ph = s_ph[sp]++;
    if (ph == 2) {
      --sp;
      continue;
    }
    if (ph == 1) {
      const View<T> toff =
          p.lower ? SubView(p.tri, off + r1, off) : SubView(p.tri, off, off + r1);
      if (p.left) {
        T* b1 = p.b + off;
        T* b2 = p.b + off + r1;
        if (p.lower)
          CoopStep(r2, p.other, r1, toff, col(b1, p.ldb), col(b2, p.ldb), sa, sb);
        else
          CoopStep(r1, p.other, r2, toff, col(b2, p.ldb), col(b1, p.ldb), sa, sb);
      } else {
        // X op(T) = B: the update C -= X_k toff, computed transposed,
        // C^T -= toff^T X_k^T (each product's factors swap, which leaves
        // every FMA's value unchanged), so that the few right-hand sides are
        // the columns.
        T* b1 = p.b + static_cast<long long>(off) * p.ldb;
        T* b2 = p.b + static_cast<long long>(off + r1) * p.ldb;
        View<T> tt = toff;
        tt.rs = toff.cs;
        tt.cs = toff.rs;
        if (p.lower)
          CoopStep(r1, p.other, r2, tt, row(b2, p.ldb), row(b1, p.ldb), sa, sb);
        else
          CoopStep(r2, p.other, r1, tt, row(b1, p.ldb), row(b2, p.ldb), sa, sb);
      }
      if (!GridBarrier(p.barrier, gridDim.x, ++gen, p.timeout_flag)) return;
    }
    // ph 0: the first half; ph 1: the second.
    const bool take11 = (ph == 0) == first11;
    ++sp;
    s_off[sp] = take11 ? off : off + r1;
    s_r[sp] = take11 ? r1 : r2;
    s_ph[sp] = 0;
  }
}

template <typename T>
bool TrsmCoop(bool left, View<T> tri, bool lower, bool unit, int r, int other, T* b,
              int ldb) {
  Context& ctx = Ctx();
  static int per_sm[2] = {-1, -1};
  int& occ = per_sm[sizeof(T) == 8 ? 0 : 1];
  constexpr int kSmem = static_cast<int>(sizeof(T)) * kTcKMax * (kTcRowsCta + kTcColsCta);
  if (occ < 0) {
    int v = 0;
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(TrsmCoopKernel<T>),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, TrsmCoopKernel<T>, kTcThreads,
                                                      kSmem) != cudaSuccess) {
      cudaGetLastError();
      v = 0;
    }
    occ = v;
  }
  if (occ <= 0) return false;
  // One CTA per block of the largest update, at most one an SM (fewer CTAs
  // make cheaper barriers).
  const int blocks =
      (sizeof(T) == 8 && other >= kTcDmmaB)
          ? ((r - 32 + kTcDmmaB - 1) / kTcDmmaB) * ((other + kTcDmmaB - 1) / kTcDmmaB)
          : ((r - 32 + kTcRowsCta - 1) / kTcRowsCta) * ((other + kTcColsCta - 1) / kTcColsCta);
  const int grid = std::max(1, std::min(blocks, std::min(ctx.num_sms, ctx.num_sms * occ)));
  unsigned int* bar = static_cast<unsigned int*>(Workspace(kWsTrsmBarrier, 256));
  if (bar == nullptr) return false;
  cudaMemsetAsync(bar, 0, sizeof(unsigned int), ctx.stream);
  TrsmCoopArgs<T> a;
  a.tri = tri;
  a.left = left ? 1 : 0;
  a.lower = lower ? 1 : 0;
  a.unit = unit ? 1 : 0;
  a.r = r;
  a.other = other;
  a.b = b;
  a.ldb = ldb;
  a.barrier = bar;
  a.timeout_flag = ctx.dev_status;
  a.guard = ctx.guard;
  void* args[] = {&a};
  if (cudaLaunchCooperativeKernel(reinterpret_cast<void*>(TrsmCoopKernel<T>), grid,
                                  kTcThreads, args, kSmem, ctx.stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  CountLaunch();
  LaunchFailed("trsm cooperative");
  return true;
}

// Left-side FP64 TRSM subtree (at most kTcRows rows) with many right-hand
// sides: the columns of X are independent, so each CTA owns kTsCols of them
// and walks the whole recursion for those columns alone, with block
// barriers only (no grid barrier, no cooperative launch). Base solves are
// the base kernel's code (one thread a column); an update C -= A X of the
// CTA's columns gives each warp 16-row strips of C and runs the element's
// m16n8k8 chain over k, restarted every KC = 256 and merged in order (alpha
// -1, beta 1): every element's FMA chain and merges are those of the
// cooperative kernel's updates, so X comes out the same.
constexpr int kTsCols = 8;       // right-hand sides a CTA owns: one n8 fragment
constexpr int kTsMinOther = 256;  // the column-owned path from this many
// ... and from this many rows: a shallower subtree is a short chain of
// launches already, and the LU's 64-row panel solves over thousands of
// columns measured slower column-owned (dgesv n = 16384 251 -> 278 ms).
constexpr int kTsMinRows = 256;

// C (mm x w) -= A (mm x kk) X (kk x w); X and C column-major with leading
// dimension ld, A a strided view. Fragments come from L2 four k8 steps at a
// time (zero past kk, mm and w: fma(0, 0, acc) = acc for a chain started at
// +0).
__device__ void ColsUpdate(int mm, int kk, View<double> a, const double* x, double* c,
                           long long ld, int w) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane >> 2, t = lane & 3;
  const int warps = blockDim.x / 32;
  for (int i0 = warp * 16; i0 < mm; i0 += warps * 16) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0}, cv[4];
    bool in[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = i0 + g + (e >> 1) * 8, j = 2 * t + (e & 1);
      in[e] = i < mm && j < w;
      cv[e] = in[e] ? __ldcg(c + i + j * ld) : 0.0;
    }
    const int ra = i0 + g, rb = i0 + g + 8;
    for (int k0 = 0; k0 < kk; k0 += 32) {
      double fa[4][4], fb[4][2];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int q0 = k0 + 8 * s + t, q1 = q0 + 4;
        fa[s][0] = (ra < mm && q0 < kk) ? __ldcg(a.data + ra * a.rs + q0 * a.cs) : 0.0;
        fa[s][1] = (rb < mm && q0 < kk) ? __ldcg(a.data + rb * a.rs + q0 * a.cs) : 0.0;
        fa[s][2] = (ra < mm && q1 < kk) ? __ldcg(a.data + ra * a.rs + q1 * a.cs) : 0.0;
        fa[s][3] = (rb < mm && q1 < kk) ? __ldcg(a.data + rb * a.rs + q1 * a.cs) : 0.0;
        fb[s][0] = (g < w && q0 < kk) ? __ldcg(x + q0 + g * ld) : 0.0;
        fb[s][1] = (g < w && q1 < kk) ? __ldcg(x + q1 + g * ld) : 0.0;
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
            "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
            : "+d"(acc[0]), "+d"(acc[1]), "+d"(acc[2]), "+d"(acc[3])
            : "d"(fa[s][0]), "d"(fa[s][1]), "d"(fa[s][2]), "d"(fa[s][3]), "d"(fb[s][0]),
              "d"(fb[s][1]));
      }
      // End of a KC chunk (or of k): merge alpha * acc = -acc, restart.
      if ((k0 + 32) % 256 == 0 || k0 + 32 >= kk) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double r = -1.0 * acc[e];
          cv[e] = r + cv[e];
          acc[e] = 0.0;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = i0 + g + (e >> 1) * 8, j = 2 * t + (e & 1);
      if (in[e]) __stcg(c + i + j * ld, cv[e]);
    }
  }
}

__global__ void __launch_bounds__(kTcThreads) TrsmColsKernel(TrsmCoopArgs<double> p) {
  if (p.guard != nullptr && *p.guard != 0) return;
  __shared__ double st[32][33];
  __shared__ double sinv[32];
  const int j0 = blockIdx.x * kTsCols;
  const int w = min(kTsCols, p.other - j0);
  if (w <= 0) return;
  double* xb = p.b + static_cast<long long>(j0) * p.ldb;  // this CTA's columns
  // Which half TrsmRec solves first: t11 for left-lower.
  const bool first11 = p.lower != 0;
  int s_off[8], s_r[8], s_ph[8];
  int sp = 0;
  s_off[0] = 0;
  s_r[0] = p.r;
  s_ph[0] = 0;
  while (sp >= 0) {
    const int off = s_off[sp], rr = s_r[sp];
    if (rr <= 32) {
      // T X = B as X^T T^T = B^T: rows of X^T are B's columns.
      View<double> t = SubView(p.tri, off, off);
      const long long rs = t.rs;
      t.rs = t.cs;
      t.cs = rs;
      const int lo = !p.lower;
      LoadBaseTriangle(t, lo, p.unit, rr, st, sinv);
      if (threadIdx.x < w)
        BaseSolveRow<double, true>(st, sinv, lo, p.unit, rr,
                                   xb + off + threadIdx.x * p.ldb, 1);
      --sp;
      __syncthreads();
      continue;
    }
    const int r1 = max(32, (rr / 2) / 32 * 32), r2 = rr - r1;
    const int ph = s_ph[sp]++;
    if (ph == 2) {
      --sp;
      continue;
    }
    if (ph == 1) {
      if (p.lower)
        ColsUpdate(r2, r1, SubView(p.tri, off + r1, off), xb + off, xb + off + r1, p.ldb, w);
      else
        ColsUpdate(r1, r2, SubView(p.tri, off, off + r1), xb + off + r1, xb + off, p.ldb, w);
      __syncthreads();
    }
    // ph 0: the first half; ph 1: the second.
    const bool take11 = (ph == 0) == first11;
    ++sp;
    s_off[sp] = take11 ? off : off + r1;
    s_r[sp] = take11 ? r1 : r2;
    s_ph[sp] = 0;
  }
}

bool TrsmCols(View<double> tri, bool lower, bool unit, int r, int other, double* b, int ldb) {
  Context& ctx = Ctx();
  TrsmCoopArgs<double> a;
  a.tri = tri;
  a.left = 1;
  a.lower = lower ? 1 : 0;
  a.unit = unit ? 1 : 0;
  a.r = r;
  a.other = other;
  a.b = b;
  a.ldb = ldb;
  a.barrier = nullptr;
  a.timeout_flag = ctx.dev_status;
  a.guard = ctx.guard;
  TrsmColsKernel<<<(other + kTsCols - 1) / kTsCols, kTcThreads, 0, ctx.stream>>>(a);
  CountLaunch();
  return !LaunchFailed("trsm column-owned");
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
  if constexpr (sizeof(T) == 8) {
    if (left && r <= kTcRows && r >= kTsMinRows && other >= kTsMinOther) {
      TrsmCols(tri, lower, unit, r, other, b, ldb);
      return;
    }
  }
  if (r <= kTcRows && other <= TcOther<T>() &&
      TrsmCoop<T>(left, tri, lower, unit, r, other, b, ldb))
    return;
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
