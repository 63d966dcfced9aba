// Oracle BLAS (TEST INFRASTRUCTURE ONLY; the product never loads this file's
// library). CPU restatement of the reference's level-3 BLAS hot path with the
// reference's exact per-element rounding:
//
//   GEMM   src/gemm-inl.h:153-232 (KC chunks, beta only on the first chunk),
//          src/gemm_kernel-inl.h:161-176 (acc = fma(a, b, acc) over k),
//          src/gemm_kernel-inl.h:182-224 (r = alpha*acc; r + C, or fma(C, beta, r))
//          src/gemm-inl.h:91-130 (triangular C: tiles crossing the diagonal
//          are merged element-wise as v + beta*C, two roundings)
//          src/gemm.cc:73-132 (argument checks and quick returns)
//   TRSM   src/trsm.cc:87-180 (recursive split at max(32, (r/2)/32*32))
//          src/trsm-inl.h:43-71, 107-174, 277-325 (base solve, dot form,
//          two columns per pass, reciprocal diagonal)
//   SYRK   src/level3.cc:84-139
//   IAMAX  src/level1.cc:383-402, src/level1-inl.h:343-423
//
// The restatement is vectorised with AVX2 along M only (each lane owns one C
// element, so the per-element order is the reference's) and threaded over
// column blocks of C (std::thread), which also leaves every element's order unchanged.
#include <immintrin.h>
#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

int g_lanes = 8;
int g_threads = 1;

// ---------------------------------------------------------------------------
// Vector helpers (AVX2 + FMA): one register of T.
template <typename T>
struct Vec;
template <>
struct Vec<double> {
  using V = __m256d;
  static constexpr int kL = 4;
  static V zero() { return _mm256_setzero_pd(); }
  static V load(const double* p) { return _mm256_loadu_pd(p); }
  static V set(double x) { return _mm256_set1_pd(x); }
  static V fma(V a, V b, V c) { return _mm256_fmadd_pd(a, b, c); }
  static void store(double* p, V v) { _mm256_storeu_pd(p, v); }
};
template <>
struct Vec<float> {
  using V = __m256;
  static constexpr int kL = 8;
  static V zero() { return _mm256_setzero_ps(); }
  static V load(const float* p) { return _mm256_loadu_ps(p); }
  static V set(float x) { return _mm256_set1_ps(x); }
  static V fma(V a, V b, V c) { return _mm256_fmadd_ps(a, b, c); }
  static void store(float* p, V v) { _mm256_storeu_ps(p, v); }
};

// ---------------------------------------------------------------------------
// Reference micro-tile geometry for triangular C (SYRK): MR = 2 * lanes rows,
// NR = 12 columns with 32 vector registers (AVX-512) or 6 with 16 (AVX2);
// MC = 96 (double) / 144 (float) rounded to MR, NC = 4080 rounded to NR
// (src/gemm_kernel-inl.h:64-74).
template <typename T>
struct RefTiles {
  size_t mr, nr, mc, nc;
  RefTiles() {
    const size_t lanes = sizeof(T) == 8 ? g_lanes : 2 * g_lanes;
    mr = 2 * lanes;
    nr = g_lanes >= 8 ? 12 : 6;
    mc = (sizeof(T) == 4 ? 144 : 96) / mr * mr;
    nc = 4080 / nr * nr;
  }
};

// Whether element (i, j) of an m x n triangular C lies in a reference
// micro-tile that crosses the diagonal (src/gemm-inl.h:93-106, 195-199).
template <typename T>
static bool InCrossingTile(const RefTiles<T>& t, Part part, size_t m, size_t n,
                           size_t i, size_t j) {
  const size_t ic = i / t.mc * t.mc, mcb = std::min(t.mc, m - ic);
  const size_t ir = (i - ic) / t.mr * t.mr, mr = std::min(t.mr, mcb - ir);
  const size_t jc = j / t.nc * t.nc, ncb = std::min(t.nc, n - jc);
  const size_t jr = (j - jc) / t.nr * t.nr, nr = std::min(t.nr, ncb - jr);
  const size_t i0 = ic + ir, j0 = jc + jr;
  const size_t i_last = i0 + mr - 1, j_last = j0 + nr - 1;
  if (part == kLower) return !(i0 > j_last);
  return !(i_last < j0);
}

// One KC chunk's contribution merged into C(i, j): `first` selects beta.
// Inside tiles: r = alpha*acc, then C = r (beta 0), r + C (beta 1) or
// fma(C, beta, r). Crossing tiles: v = alpha*acc, then v + beta*C.
template <typename T>
static inline T Merge(T acc, T alpha, T beta, T c, bool crossing) {
  const T r = alpha * acc;
  if (beta == T(0)) return r;
  if (crossing) {
    const T bc = beta * c;
    return r + bc;
  }
  if (beta == T(1)) return r + c;
  return std::fma(c, beta, r);
}

template <typename T>
constexpr size_t KcOf() {
  return sizeof(T) == 4 ? 384 : 256;
}

// C := alpha * op(A) * op(B) + beta * C (or one triangle of it). Requires
// m, n, k > 0 (callers handle trivial cases, as RunGemm's callers do).
template <typename T>
void Gemm(size_t m, size_t n, size_t k, T alpha, Opnd<T> a, Opnd<T> b, T beta,
          T* c, size_t ldc, Part part) {
  using VT = Vec<T>;
  using V = typename VT::V;
  constexpr size_t L = VT::kL;
  constexpr size_t MR = 2 * L, NR = 6;
  constexpr size_t KC = KcOf<T>();
  constexpr size_t MC = 96 / MR * MR * (sizeof(T) == 4 ? 2 : 1);
  constexpr size_t NCB = 96;  // columns per parallel block
  const RefTiles<T> tiles;
  const size_t nblocks = (n + NCB - 1) / NCB;

  const auto run_block = [&](size_t blk) {
    const size_t jc = blk * NCB, nc = std::min(NCB, n - jc);
    std::vector<T> pa(MC * KC + MR), pb(((nc + NR - 1) / NR) * NR * KC + NR);
    T tmp[MR * NR];
    for (size_t pc = 0; pc < k; pc += KC) {
      const size_t kc = std::min(KC, k - pc);
      const bool first = (pc == 0);
      // Pack op(B)[pc:pc+kc, jc:jc+nc] into NR-column panels (k-major).
      for (size_t c0 = 0; c0 < nc; c0 += NR) {
        T* dst = pb.data() + c0 * kc;
        for (size_t p = 0; p < kc; ++p)
          for (size_t cc = 0; cc < NR; ++cc)
            dst[p * NR + cc] =
                (c0 + cc < nc) ? b.at(pc + p, jc + c0 + cc) : T(0);
      }
      for (size_t ic = 0; ic < m; ic += MC) {
        const size_t mc = std::min(MC, m - ic);
        // Skip row blocks entirely outside the triangle.
        if (part == kLower && ic + mc - 1 < jc) continue;
        if (part == kUpper && ic > jc + nc - 1) continue;
        for (size_t r0 = 0; r0 < mc; r0 += MR) {
          T* dst = pa.data() + r0 * kc;
          for (size_t p = 0; p < kc; ++p)
            for (size_t rr = 0; rr < MR; ++rr)
              dst[p * MR + rr] =
                  (r0 + rr < mc) ? a.at(ic + r0 + rr, pc + p) : T(0);
        }
        for (size_t c0 = 0; c0 < nc; c0 += NR) {
          const size_t ncols = std::min(NR, nc - c0);
          for (size_t r0 = 0; r0 < mc; r0 += MR) {
            const size_t nrows = std::min(MR, mc - r0);
            const size_t gi0 = ic + r0, gj0 = jc + c0;
            if (part == kLower && gi0 + nrows - 1 < gj0) continue;
            if (part == kUpper && gi0 > gj0 + ncols - 1) continue;
            const T* ap = pa.data() + r0 * kc;
            const T* bp = pb.data() + c0 * kc;
            V acc[NR][2];
            for (size_t cc = 0; cc < NR; ++cc) acc[cc][0] = acc[cc][1] = VT::zero();
            for (size_t p = 0; p < kc; ++p) {
              const V a0 = VT::load(ap + p * MR), a1 = VT::load(ap + p * MR + L);
              for (size_t cc = 0; cc < NR; ++cc) {
                const V bv = VT::set(bp[p * NR + cc]);
                acc[cc][0] = VT::fma(a0, bv, acc[cc][0]);
                acc[cc][1] = VT::fma(a1, bv, acc[cc][1]);
              }
            }
            for (size_t cc = 0; cc < NR; ++cc) {
              VT::store(tmp + cc * MR, acc[cc][0]);
              VT::store(tmp + cc * MR + L, acc[cc][1]);
            }
            const T beta_eff = first ? beta : T(1);
            for (size_t cc = 0; cc < ncols; ++cc) {
              const size_t gj = gj0 + cc;
              T* cj = c + gj * ldc;
              for (size_t rr = 0; rr < nrows; ++rr) {
                const size_t gi = gi0 + rr;
                bool crossing = false;
                if (part != kAll) {
                  if (part == kLower ? (gi < gj) : (gi > gj)) continue;
                  crossing = InCrossingTile(tiles, part, m, n, gi, gj);
                }
                cj[gi] = Merge(tmp[cc * MR + rr], alpha, beta_eff,
                               beta_eff == T(0) ? T(0) : cj[gi], crossing);
              }
            }
          }
        }
      }
    }
  };
  // Column blocks of C are independent; threads take them in turn.
  const size_t nthreads = std::min<size_t>(g_threads, nblocks);
  if (nthreads <= 1 || m * n * k < (size_t(1) << 21)) {
    for (size_t blk = 0; blk < nblocks; ++blk) run_block(blk);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  for (size_t t = 0; t < nthreads; ++t) {
    pool.emplace_back([&] {
      for (size_t blk; (blk = next.fetch_add(1)) < nblocks;) run_block(blk);
    });
  }
  for (auto& th : pool) th.join();
}

template <typename T>
void ScaleMatrix(size_t m, size_t n, T beta, T* c, size_t ldc, Part part) {
  for (size_t j = 0; j < n; ++j) {
    T* cj = c + j * ldc;
    const size_t begin = (part == kLower) ? std::min(j, m) : 0;
    const size_t end = (part == kUpper) ? std::min(j + 1, m) : m;
    if (beta == T(0)) {
      for (size_t i = begin; i < end; ++i) cj[i] = T(0);
    } else {
      for (size_t i = begin; i < end; ++i) cj[i] *= beta;
    }
  }
}

static char Up(char ch) { return (ch >= 'a' && ch <= 'z') ? ch - 32 : ch; }
bool DecodeOp(char ch, bool* trans) {
  ch = Up(ch);
  *trans = (ch == 'T' || ch == 'C');
  return ch == 'N' || ch == 'T' || ch == 'C';
}

template <typename T>
Opnd<T> General(bool trans, const T* x, int ld) {
  Opnd<T> o;
  o.data = x;
  o.rs = trans ? ld : 1;
  o.cs = trans ? 1 : ld;
  return o;
}

template <typename T>
int GemmF(char transa, char transb, int m, int n, int k, T alpha, const T* a,
          int lda, const T* b, int ldb, T beta, T* c, int ldc) {
  bool ta, tb;
  const bool va = DecodeOp(transa, &ta), vb = DecodeOp(transb, &tb);
  const int rows_a = ta ? k : m, rows_b = tb ? n : k;
  int info = 0;
  if (!va) info = 1;
  else if (!vb) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, m)) info = 13;
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  if ((k == 0 || alpha == T(0)) && beta == T(1)) return 0;
  if (k == 0 || alpha == T(0)) {
    ScaleMatrix<T>(m, n, beta, c, ldc, kAll);
    return 0;
  }
  Gemm<T>(m, n, k, alpha, General(ta, a, lda), General(tb, b, ldb), beta, c,
          ldc, kAll);
  return 0;
}

// ---------------------------------------------------------------------------
// TRSM (src/trsm.cc, src/trsm-inl.h).

// Solves X T = B for `rows` independent rows. Element (row i, column q) of B
// is at b[i * xs_row + q * xs_col]; T(q, j) is tri.at(q, j).
template <typename T>
static void SolveBase(const Opnd<T>& tri, bool lower, bool unit, size_t r,
                      size_t rows, T* b, ptrdiff_t xs_row, ptrdiff_t xs_col) {
  T inv[32];
  for (size_t j = 0; j < r; ++j) inv[j] = unit ? T(1) : T(1) / tri.at(j, j);
  const auto col = [&](size_t s) { return lower ? r - 1 - s : s; };
  for (size_t i = 0; i < rows; ++i) {
    T* bi = b + static_cast<ptrdiff_t>(i) * xs_row;
    const auto X = [&](size_t q) -> T& {
      return bi[static_cast<ptrdiff_t>(q) * xs_col];
    };
    size_t step = 0;
    for (; step + 2 <= r; step += 2) {
      const size_t j0 = col(step), j1 = col(step + 1);
      T acc0 = X(j0), acc1 = X(j1);
      for (size_t s = 0; s < step; ++s) {
        const size_t q = col(s);
        const T x = X(q);
        acc0 = std::fma(-x, tri.at(q, j0), acc0);
        acc1 = std::fma(-x, tri.at(q, j1), acc1);
      }
      if (!unit) acc0 = acc0 * inv[j0];
      X(j0) = acc0;
      acc1 = std::fma(-acc0, tri.at(j0, j1), acc1);
      if (!unit) acc1 = acc1 * inv[j1];
      X(j1) = acc1;
    }
    if (step < r) {
      const size_t j = col(step);
      T acc = X(j);
      for (size_t s = 0; s < step; ++s) {
        const size_t q = col(s);
        acc = std::fma(-X(q), tri.at(q, j), acc);
      }
      if (!unit) acc = acc * inv[j];
      X(j) = acc;
    }
  }
}

template <typename T>
static void TrsmRec(bool left, const Opnd<T>& tri, bool lower, bool unit,
                    size_t r, size_t other, T* b, size_t ldb) {
  if (r <= 32) {
    if (!left) {
      SolveBase(tri, lower, unit, r, other, b, 1, static_cast<ptrdiff_t>(ldb));
    } else {
      // T X = B  <=>  X^T T^T = B^T (src/trsm-inl.h:306-324).
      Opnd<T> tt = tri;
      tt.rs = tri.cs;
      tt.cs = tri.rs;
      SolveBase(tt, !lower, unit, r, other, b, static_cast<ptrdiff_t>(ldb), 1);
    }
    return;
  }
  const size_t r1 = std::max<size_t>(32, (r / 2) / 32 * 32);
  const size_t r2 = r - r1;
  const Opnd<T> t11 = tri;
  const Opnd<T> t22 = tri.sub(r1, r1);
  const Opnd<T> toff = lower ? tri.sub(r1, 0) : tri.sub(0, r1);
  const auto colmajor = [&](T* blk) {
    Opnd<T> o;
    o.data = blk;
    o.rs = 1;
    o.cs = static_cast<ptrdiff_t>(ldb);
    return o;
  };
  const T minus1 = T(-1), one = T(1);
  if (left) {
    T* b1 = b;
    T* b2 = b + r1;
    if (lower) {
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
      Gemm<T>(r2, other, r1, minus1, toff, colmajor(b1), one, b2, ldb, kAll);
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
    } else {
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
      Gemm<T>(r1, other, r2, minus1, toff, colmajor(b2), one, b1, ldb, kAll);
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
    }
  } else {
    T* b1 = b;
    T* b2 = b + r1 * ldb;
    if (lower) {
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
      Gemm<T>(other, r1, r2, minus1, colmajor(b2), toff, one, b1, ldb, kAll);
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
    } else {
      TrsmRec(left, t11, lower, unit, r1, other, b1, ldb);
      Gemm<T>(other, r2, r1, minus1, colmajor(b1), toff, one, b2, ldb, kAll);
      TrsmRec(left, t22, lower, unit, r2, other, b2, ldb);
    }
  }
}

template <typename T>
int TrsmF(char side, char uplo, char transa, char diag, int m, int n, T alpha,
          const T* a, int lda, T* b, int ldb) {
  const char s = Up(side), u = Up(uplo), d = Up(diag);
  bool trans;
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const bool vt = DecodeOp(transa, &trans), vd = (d == 'U' || d == 'N');
  const bool left = (s == 'L'), lower = (u == 'L'), unit = (d == 'U');
  const int rows_a = left ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (!vt) info = 3;
  else if (!vd) info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, rows_a)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  if (alpha != T(1)) ScaleMatrix<T>(m, n, alpha, b, ldb, kAll);
  if (alpha == T(0)) return 0;
  const Opnd<T> tri = General(trans, a, lda);
  const bool op_lower = trans ? !lower : lower;
  TrsmRec<T>(left, tri, op_lower, unit, left ? m : n, left ? n : m, b, ldb);
  return 0;
}

// ---------------------------------------------------------------------------
// SYRK (src/level3.cc:84-139), real only; the reference's ssyrk_/dsyrk_
// (level3.cc:410-421) are the same template at float and double.
template <typename T>
int Syrk(char uplo, char trans, int n, int k, T alpha, const T* a, int lda, T beta, T* c,
         int ldc) {
  const char u = Up(uplo);
  bool t;
  const bool vu = (u == 'L' || u == 'U');
  const bool vt = DecodeOp(trans, &t);
  const int rows_a = t ? k : n;
  int info = 0;
  if (!vu) info = 1;
  else if (!vt) info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, rows_a)) info = 7;
  else if (ldc < std::max(1, n)) info = 10;
  if (info) return info;
  const Part part = (u == 'L') ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return 0;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return 0;
  }
  Gemm<T>(n, n, k, alpha, General(t, a, lda), General(!t, a, lda), beta, c, ldc, part);
  return 0;
}
template int Syrk<double>(char, char, int, int, double, const double*, int, double, double*,
                          int);
template int Syrk<float>(char, char, int, int, float, const float*, int, float, float*, int);
int SyrkD(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
          double beta, double* c, int ldc) {
  return Syrk<double>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}

// ---------------------------------------------------------------------------
// SYMM (src/level3.cc:26-76): the reference packs the stored triangle
// mirrored (Structure::kSymmetric, src/pack-inl.h:99-160), i.e. the values of
// the full symmetric matrix; the other triangle is never read.
template <typename T>
int Symm(char side, char uplo, int m, int n, T alpha, const T* a, int lda, const T* b,
         int ldb, T beta, T* c, int ldc) {
  const char s = Up(side), u = Up(uplo);
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const bool left = (s == 'L'), lower = (u == 'L');
  const int ka = left ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (lda < std::max(1, ka)) info = 7;
  else if (ldb < std::max(1, m)) info = 9;
  else if (ldc < std::max(1, m)) info = 12;
  if (info) return info;
  if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return 0;
  if (alpha == T(0)) {
    ScaleMatrix<T>(m, n, beta, c, ldc, kAll);
    return 0;
  }
  std::vector<T> full(static_cast<size_t>(ka) * ka);
  for (int j = 0; j < ka; ++j)
    for (int i = 0; i < ka; ++i) {
      const bool stored = lower ? (i >= j) : (i <= j);
      full[i + static_cast<size_t>(j) * ka] =
          stored ? a[i + static_cast<ptrdiff_t>(j) * lda] : a[j + static_cast<ptrdiff_t>(i) * lda];
    }
  const Opnd<T> sym = General(false, full.data(), ka);
  const Opnd<T> gen = General(false, b, ldb);
  Gemm<T>(m, n, ka, alpha, left ? sym : gen, left ? gen : sym, beta, c, ldc, kAll);
  return 0;
}

// SYR2K (src/level3.cc:153-221): alpha op(A) op(B)^T + beta C, then
// + alpha op(B) op(A)^T with beta 1, each a GEMM problem on the uplo triangle.
template <typename T>
int Syr2k(char uplo, char trans, int n, int k, T alpha, const T* a, int lda, const T* b,
          int ldb, T beta, T* c, int ldc) {
  const char u = Up(uplo);
  bool t;
  const bool vu = (u == 'L' || u == 'U');
  const bool vt = DecodeOp(trans, &t);
  const int rows = t ? k : n;
  int info = 0;
  if (!vu) info = 1;
  else if (!vt) info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, rows)) info = 7;
  else if (ldb < std::max(1, rows)) info = 9;
  else if (ldc < std::max(1, n)) info = 12;
  if (info) return info;
  const Part part = (u == 'L') ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return 0;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return 0;
  }
  Gemm<T>(n, n, k, alpha, General(t, a, lda), General(!t, b, ldb), beta, c, ldc, part);
  Gemm<T>(n, n, k, alpha, General(t, b, ldb), General(!t, a, lda), T(1), c, ldc, part);
  return 0;
}

// GEMMTR and its alias GEMMT (src/level3.cc:226-280): op(A) n x k times
// op(B) k x n on the uplo triangle of C.
template <typename T>
int Gemmtr(char uplo, char transa, char transb, int n, int k, T alpha, const T* a, int lda,
           const T* b, int ldb, T beta, T* c, int ldc) {
  const char u = Up(uplo);
  bool ta, tb;
  const bool vu = (u == 'L' || u == 'U');
  const bool va = DecodeOp(transa, &ta), vb = DecodeOp(transb, &tb);
  const int rows_a = ta ? k : n, rows_b = tb ? n : k;
  int info = 0;
  if (!vu) info = 1;
  else if (!va) info = 2;
  else if (!vb) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, n)) info = 13;
  if (info) return info;
  const Part part = (u == 'L') ? kLower : kUpper;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return 0;
  if (alpha == T(0) || k == 0) {
    ScaleMatrix<T>(n, n, beta, c, ldc, part);
    return 0;
  }
  Gemm<T>(n, n, k, alpha, General(ta, a, lda), General(tb, b, ldb), beta, c, ldc, part);
  return 0;
}

// TRMM (src/level3.cc:284-342), element by element: B(i, j) is the GEMM
// problem's chain over the k range that the reference multiplies for the
// micro-tile holding (i, j) (NonZeroRange, src/gemm-inl.h:62-85), restarted
// every KC; a chunk outside that range is skipped, except the first, which
// still applies beta = 0 (src/gemm-inl.h:176-209). The triangular operand has
// explicit zeros outside its triangle and ones on a unit diagonal
// (src/pack-inl.h:99-160); op(A) is lower when A is lower xor transposed
// (src/api.h:133-140). B is read from a copy of its input.
template <typename T>
int Trmm(char side, char uplo, char transa, char diag, int m, int n, T alpha, const T* a,
         int lda, T* b, int ldb) {
  const char s = Up(side), u = Up(uplo), d = Up(diag);
  bool trans;
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const bool vt = DecodeOp(transa, &trans), vd = (d == 'U' || d == 'N');
  const bool left = (s == 'L'), lower = (u == 'L'), unit = (d == 'U');
  const int ka = left ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (!vt) info = 3;
  else if (!vd) info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, ka)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  if (alpha == T(0)) {
    ScaleMatrix<T>(m, n, T(0), b, ldb, kAll);
    return 0;
  }
  const size_t K = static_cast<size_t>(ka);
  std::vector<T> tri(K * K);  // op(A), dense
  for (int j = 0; j < ka; ++j)
    for (int i = 0; i < ka; ++i) {
      T v = T(0);
      if (i == j) v = unit ? T(1) : a[i + static_cast<ptrdiff_t>(i) * lda];
      else if (lower ? i > j : i < j) v = a[i + static_cast<ptrdiff_t>(j) * lda];
      if (trans) tri[j + i * K] = v;
      else tri[i + j * K] = v;
    }
  std::vector<T> copy(static_cast<size_t>(m) * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i)
      copy[i + static_cast<size_t>(j) * m] = b[i + static_cast<ptrdiff_t>(j) * ldb];
  const bool op_lower = (lower != trans);
  const RefTiles<T> t;
  constexpr size_t KC = KcOf<T>();
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      const size_t ic = i / t.mc * t.mc, mcb = std::min(t.mc, m - ic);
      const size_t ir = (i - ic) / t.mr * t.mr, mr = std::min(t.mr, mcb - ir);
      const size_t jc = j / t.nc * t.nc, ncb = std::min(t.nc, n - jc);
      const size_t jr = (j - jc) / t.nr * t.nr, nr = std::min(t.nr, ncb - jr);
      const size_t i0 = ic + ir, j0 = jc + jr;
      size_t kb = 0, ke = K;
      if (left) {
        if (op_lower) ke = std::min(ke, i0 + mr);
        else kb = i0;
      } else {
        if (op_lower) kb = j0;
        else ke = std::min(ke, j0 + nr);
      }
      T cv = T(0);
      for (size_t pc = 0; pc < K; pc += KC) {
        const size_t lo = std::max(kb, pc), hi = std::max(lo, std::min(ke, pc + KC));
        if (lo == hi && pc != 0) continue;
        T acc = T(0);
        for (size_t q = lo; q < hi; ++q) {
          const T av = left ? tri[i + q * K] : copy[i + q * m];
          const T bv = left ? copy[q + static_cast<size_t>(j) * m] : tri[q + j * K];
          acc = std::fma(av, bv, acc);
        }
        cv = (pc == 0) ? Merge(acc, alpha, T(0), T(0), false)
                       : Merge(acc, alpha, T(1), cv, false);
      }
      b[i + static_cast<ptrdiff_t>(j) * ldb] = cv;
    }
  return 0;
}

// ---------------------------------------------------------------------------
// TRMV, op N, contiguous x (src/trmv-inl.h:44-80): x := A x. The product
// collects in a zeroed y, in strips of 4 columns: the strip's diagonal block
// element by element as y += v * x (product and sum rounded separately, the
// reference being built without contraction), then the rectangle below
// (lower) or above (upper) it by the axpy GEMV kernel, which chains an fma
// per column in column order for each row (src/gemv-inl.h:54-84, 280-292).
template <typename T>
void TrmvN(bool lower, bool unit, int n, const T* a, int lda, T* x) {
  if (n <= 0) return;
  std::vector<T> y(n, T(0));
  const auto A = [&](int i, int j) { return a[i + static_cast<ptrdiff_t>(j) * lda]; };
  for (int j = 0; j < n; j += 4) {
    const int cols = std::min(4, n - j);
    for (int jj = j; jj < j + cols; ++jj)
      for (int ii = j; ii < j + cols; ++ii) {
        if (lower ? ii < jj : ii > jj) continue;
        const T v = (ii == jj && unit) ? T(1) : A(ii, jj);
        const T prod = v * x[jj];
        y[ii] = y[ii] + prod;
      }
    const int row0 = lower ? j + cols : 0;
    const int rows = lower ? n - row0 : j;
    for (int c = j; c < j + cols; ++c)
      for (int i = row0; i < row0 + rows; ++i) y[i] = std::fma(A(i, c), x[c], y[i]);
  }
  std::copy(y.begin(), y.end(), x);
}

// GEMV, op N, contiguous x and y (src/gemv.cc:48-77; src/gemv-inl.h:40-52,
// 280-292, 318-333): y := beta y (beta 0 writes zeros), then with
// t = alpha * x, y(i) = fma(A(i, j), t(j), y(i)) for j in order.
template <typename T>
void GemvN(int m, int n, T alpha, const T* a, int lda, const T* x, T beta, T* y) {
  if (m <= 0 || n <= 0 || (alpha == T(0) && beta == T(1))) return;
  if (beta != T(1)) {
    for (int i = 0; i < m; ++i) y[i] = (beta == T(0)) ? T(0) : y[i] * beta;
  }
  if (alpha == T(0)) return;
  for (int j = 0; j < n; ++j) {
    const T t = alpha * x[j];
    const T* col = a + static_cast<ptrdiff_t>(j) * lda;
    for (int i = 0; i < m; ++i) y[i] = std::fma(col[i], t, y[i]);
  }
}

// Vector lanes of the reference's SIMD target: 8 doubles / 16 floats
// (AVX-512) or 4 / 8 (AVX2).
template <typename T>
static size_t RefLanes() {
  return sizeof(T) == 8 ? g_lanes : 2 * g_lanes;
}

// The lane sum of a vector (ReduceSum): halves added lane-wise until one
// lane is left, i.e. ((v0+v4)+(v2+v6)) + ((v1+v5)+(v3+v7)) for 8 lanes.
template <typename T>
static T ReduceSumLanes(std::vector<T> v) {
  for (size_t h = v.size() / 2; h >= 1; h /= 2)
    for (size_t i = 0; i < h; ++i) v[i] = v[i] + v[i + h];
  return v[0];
}

// GEMV, op T, contiguous x and y (src/gemv-inl.h:163-196, 294-307, 318-333):
// y := beta y, then y(c) += alpha * (lane sum of the dot product of column c
// with x), lane l holding the fma chain over the rows i = l mod N in order
// (zero products past the end of the last vector).
template <typename T>
void GemvT(int m, int n, T alpha, const T* a, int lda, const T* x, T beta, T* y) {
  if (m <= 0 || n <= 0 || (alpha == T(0) && beta == T(1))) return;
  if (beta != T(1)) {
    for (int j = 0; j < n; ++j) y[j] = (beta == T(0)) ? T(0) : y[j] * beta;
  }
  if (alpha == T(0)) return;
  const size_t N = RefLanes<T>();
  const size_t full = static_cast<size_t>(m) / N * N;
  for (int c = 0; c < n; ++c) {
    const T* col = a + static_cast<ptrdiff_t>(c) * lda;
    std::vector<T> s(N, T(0));
    for (size_t i = 0; i < full; ++i) s[i % N] = std::fma(col[i], x[i], s[i % N]);
    if (full < static_cast<size_t>(m)) {
      for (size_t l = 0; l < N; ++l) {
        const size_t i = full + l;
        s[l] = (i < static_cast<size_t>(m)) ? std::fma(col[i], x[i], s[l])
                                            : std::fma(T(0), T(0), s[l]);
      }
    }
    const T prod = alpha * ReduceSumLanes(s);
    y[c] = y[c] + prod;
  }
}

// ASUM, contiguous (src/level1.cc:357-368; src/level1-inl.h:186-217): four
// accumulator vectors over blocks of 4 vectors, remaining whole vectors into
// the first, the zero-padded tail into the second, then (s0+s1)+(s2+s3) and
// the lane sum.
template <typename T>
T AbsSum(int n, const T* x) {
  if (n < 1) return T(0);
  const size_t N = RefLanes<T>(), len = static_cast<size_t>(n);
  std::vector<T> s0(N, T(0)), s1(N, T(0)), s2(N, T(0)), s3(N, T(0));
  size_t i = 0;
  for (; i + 4 * N <= len; i += 4 * N)
    for (size_t l = 0; l < N; ++l) {
      s0[l] = std::fabs(x[i + l]) + s0[l];
      s1[l] = std::fabs(x[i + N + l]) + s1[l];
      s2[l] = std::fabs(x[i + 2 * N + l]) + s2[l];
      s3[l] = std::fabs(x[i + 3 * N + l]) + s3[l];
    }
  for (; i + N <= len; i += N)
    for (size_t l = 0; l < N; ++l) s0[l] = std::fabs(x[i + l]) + s0[l];
  if (i < len)
    for (size_t l = 0; l < N; ++l) s1[l] = (i + l < len ? std::fabs(x[i + l]) : T(0)) + s1[l];
  std::vector<T> sum(N);
  for (size_t l = 0; l < N; ++l) sum[l] = (s0[l] + s1[l]) + (s2[l] + s3[l]);
  return ReduceSumLanes(sum);
}

// AXPY, contiguous (src/level1.cc:120-128; src/level1-inl.h:37-76): blocks
// of two vectors as fma(alpha, x, y), the rest as y + alpha * x.
template <typename T>
void AxpyRef(int n, T alpha, const T* x, T* y) {
  if (n <= 0 || alpha == T(0)) return;
  const size_t N = RefLanes<T>(), len = static_cast<size_t>(n);
  size_t i = 0;
  for (; i + 2 * N <= len; i += 2 * N)
    for (size_t l = 0; l < 2 * N; ++l) y[i + l] = std::fma(alpha, x[i + l], y[i + l]);
  for (; i < len; ++i) {
    const T prod = x[i] * alpha;
    y[i] = y[i] + prod;
  }
}

template void GemvT<double>(int, int, double, const double*, int, const double*, double,
                            double*);
template void GemvT<float>(int, int, float, const float*, int, const float*, float, float*);
template double AbsSum<double>(int, const double*);
template float AbsSum<float>(int, const float*);
template void AxpyRef<double>(int, double, const double*, double*);
template void AxpyRef<float>(int, float, const float*, float*);
template void TrmvN<double>(bool, bool, int, const double*, int, double*);
template void TrmvN<float>(bool, bool, int, const float*, int, float*);
template void GemvN<double>(int, int, double, const double*, int, const double*, double,
                            double*);
template void GemvN<float>(int, int, float, const float*, int, const float*, float, float*);
template int Trmm<double>(char, char, char, char, int, int, double, const double*, int,
                          double*, int);
template int Trmm<float>(char, char, char, char, int, int, float, const float*, int, float*,
                         int);

// ---------------------------------------------------------------------------
// Complex GEMM (src/gemm.cc:67-123; src/gemm_kernel-inl.h:226-428;
// src/gemm-inl.h:152-232), element by element. Arrays interleave (re, im);
// op 'C' conjugates while packing. Per KC = 256 chunk of k, four fma chains
// rr = sum ar*br, ir = sum ai*br, ri = sum ar*bi, ii = sum ai*bi give
// ab = (rr - ii, ir + ri) and r = alpha * ab as (ab.re*al.re - ab.im*al.im,
// ab.im*al.re + ab.re*al.im), every product and sum rounded; the first chunk
// merges r, r + C or r + beta*C (beta 0, 1, other), the later ones r + C.
// A complex operand: element (i, p) has its real part at
// data[2 * (i * rs + p * cs)]; conj negates the imaginary part.
template <typename R>
struct ZOp {
  const R* data;
  ptrdiff_t rs, cs;
  bool conj;
  void at(ptrdiff_t i, ptrdiff_t p, R* re, R* im) const {
    const R* e = data + 2 * (i * rs + p * cs);
    *re = e[0];
    *im = conj ? -e[1] : e[1];
  }
  ZOp sub(ptrdiff_t i0, ptrdiff_t p0) const {
    ZOp o = *this;
    o.data += 2 * (i0 * rs + p0 * cs);
    return o;
  }
};

// The complex GEMM problem (m, n, k > 0, alpha != 0) on operand views.
template <typename R>
void ZGemmCore(int m, int n, int k, const R* alpha, ZOp<R> a, ZOp<R> b, const R* beta, R* c,
               int ldc) {
  const bool beta_zero = beta[0] == R(0) && beta[1] == R(0);
  const bool beta_one = beta[0] == R(1) && beta[1] == R(0);
  const auto C = [&](int i, int j) { return c + 2 * (i + static_cast<ptrdiff_t>(j) * ldc); };
  constexpr int KC = 256;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      R cre = R(0), cim = R(0);
      for (int pc = 0; pc < k; pc += KC) {
        const int pe = std::min(k, pc + KC);
        R rr = R(0), ir = R(0), ri = R(0), ii = R(0);
        for (int p = pc; p < pe; ++p) {
          R ar, ai, br, bi;
          a.at(i, p, &ar, &ai);
          b.at(p, j, &br, &bi);
          rr = std::fma(ar, br, rr);
          ir = std::fma(ai, br, ir);
          ri = std::fma(ar, bi, ri);
          ii = std::fma(ai, bi, ii);
        }
        const R ab_re = rr - ii, ab_im = ir + ri;
        const R q0 = ab_re * alpha[0], q1 = ab_im * alpha[1];
        const R q2 = ab_im * alpha[0], q3 = ab_re * alpha[1];
        const R t_re = q0 - q1, t_im = q2 + q3;
        if (pc != 0) {
          cre = t_re + cre;
          cim = t_im + cim;
        } else if (beta_zero) {
          cre = t_re;
          cim = t_im;
        } else {
          const R c0 = C(i, j)[0], c1 = C(i, j)[1];
          if (beta_one) {
            cre = t_re + c0;
            cim = t_im + c1;
          } else {
            const R s0 = c0 * beta[0], s1 = c1 * beta[1], s2 = c1 * beta[0], s3 = c0 * beta[1];
            const R b_re = s0 - s1, b_im = s2 + s3;
            cre = t_re + b_re;
            cim = t_im + b_im;
          }
        }
      }
      C(i, j)[0] = cre;
      C(i, j)[1] = cim;
    }
}

template <typename R>
int ZgemmF(char transa, char transb, int m, int n, int k, const R* alpha, const R* a, int lda,
           const R* b, int ldb, const R* beta, R* c, int ldc) {
  const auto op = [](char ch) {
    ch = Up(ch);
    return ch == 'N' ? 0 : ch == 'T' ? 1 : ch == 'C' ? 2 : -1;
  };
  const int ta = op(transa), tb = op(transb);
  const int rows_a = ta == 0 ? m : k, rows_b = tb == 0 ? k : n;
  int info = 0;
  if (ta < 0) info = 1;
  else if (tb < 0) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, m)) info = 13;
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  const bool alpha_zero = alpha[0] == R(0) && alpha[1] == R(0);
  const bool beta_zero = beta[0] == R(0) && beta[1] == R(0);
  const bool beta_one = beta[0] == R(1) && beta[1] == R(0);
  if ((k == 0 || alpha_zero) && beta_one) return 0;
  const auto C = [&](int i, int j) { return c + 2 * (i + static_cast<ptrdiff_t>(j) * ldc); };
  if (k == 0 || alpha_zero) {
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) {
        R* e = C(i, j);
        if (beta_zero) {
          e[0] = e[1] = R(0);
        } else {
          const R c0 = e[0], c1 = e[1];
          const R p0 = c0 * beta[0], p1 = c1 * beta[1], p2 = c0 * beta[1], p3 = c1 * beta[0];
          e[0] = p0 - p1;
          e[1] = p2 + p3;
        }
      }
    return 0;
  }
  const ZOp<R> va = ta == 0 ? ZOp<R>{a, 1, lda, false} : ZOp<R>{a, lda, 1, ta == 2};
  const ZOp<R> vb = tb == 0 ? ZOp<R>{b, 1, ldb, false} : ZOp<R>{b, ldb, 1, tb == 2};
  ZGemmCore<R>(m, n, k, alpha, va, vb, beta, c, ldc);
  return 0;
}
// ---------------------------------------------------------------------------
// Complex TRSM (src/trsm.cc:87-180; src/trsm-inl.h:40-70, 175-214, 277-325).
// The recursion and its GEMM updates (alpha -1, beta 1) are the real ones.
// The base solves X T = B row by row (T X = B through the transposed
// triangle): column j in solve order is b_j - sum_q x_q t(q, j) over the
// solved q in increasing q, the sum kept as the four fma chains
// (xr*tr, xi*tr, xr*ti, xi*ti) combined as (rr - ii, ir + ri), then
// multiplied by inv_j = 1 / t(j, j) as (xr*vr - xi*vi, xi*vr + xr*vi). inv_j
// is the C++ complex quotient, which is what the reference computes.
template <typename R>
static void ZTrsmBase(bool left, ZOp<R> tri, bool lower, bool unit, int r, int other, R* b,
                      int ldb) {
  if (left) {  // T X = B  <=>  X^T T^T = B^T
    std::swap(tri.rs, tri.cs);
    lower = !lower;
  }
  std::vector<R> inv_re(r), inv_im(r);
  for (int j = 0; j < r; ++j) {
    R dr, di;
    tri.at(j, j, &dr, &di);
    const std::complex<R> v = unit ? std::complex<R>(1) : std::complex<R>(1) / std::complex<R>(dr, di);
    inv_re[j] = v.real();
    inv_im[j] = v.imag();
  }
  // Row `row` of X: element (row, j) at b + 2 * (row * xr + j * xc).
  const ptrdiff_t xr = left ? ldb : 1, xc = left ? 1 : ldb;
  for (int row = 0; row < other; ++row) {
    R* x = b + 2 * (static_cast<ptrdiff_t>(row) * xr);
    for (int step = 0; step < r; ++step) {
      const int j = lower ? r - 1 - step : step;
      const int qb = lower ? j + 1 : 0, qe = lower ? r : j;
      R s_rr = R(0), s_ir = R(0), s_ri = R(0), s_ii = R(0);
      for (int q = qb; q < qe; ++q) {
        R tr, ti;
        tri.at(q, j, &tr, &ti);
        const R yr = x[2 * q * xc], yi = x[2 * q * xc + 1];
        s_rr = std::fma(yr, tr, s_rr);
        s_ir = std::fma(yi, tr, s_ir);
        s_ri = std::fma(yr, ti, s_ri);
        s_ii = std::fma(yi, ti, s_ii);
      }
      const R p_re = s_rr - s_ii, p_im = s_ir + s_ri;
      R vr = x[2 * j * xc] - p_re, vi = x[2 * j * xc + 1] - p_im;
      if (!unit) {
        const R a0 = vr * inv_re[j], a1 = vi * inv_im[j], a2 = vi * inv_re[j], a3 = vr * inv_im[j];
        vr = a0 - a1;
        vi = a2 + a3;
      }
      x[2 * j * xc] = vr;
      x[2 * j * xc + 1] = vi;
    }
  }
}

template <typename R>
static void ZTrsmRec(bool left, ZOp<R> tri, bool lower, bool unit, int r, int other, R* b,
                     int ldb) {
  constexpr int kBase = 32;
  if (r <= kBase) {
    ZTrsmBase<R>(left, tri, lower, unit, r, other, b, ldb);
    return;
  }
  const int r1 = std::max(kBase, (r / 2) / kBase * kBase), r2 = r - r1;
  const ZOp<R> t11 = tri, t22 = tri.sub(r1, r1);
  const ZOp<R> toff = lower ? tri.sub(r1, 0) : tri.sub(0, r1);
  const R m1[2] = {R(-1), R(0)}, one[2] = {R(1), R(0)};
  const auto col = [&](R* p) { return ZOp<R>{p, 1, ldb, false}; };
  if (left) {
    R* b1 = b;
    R* b2 = b + 2 * r1;
    if (lower) {
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
      ZGemmCore<R>(r2, other, r1, m1, toff, col(b1), one, b2, ldb);
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
    } else {
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
      ZGemmCore<R>(r1, other, r2, m1, toff, col(b2), one, b1, ldb);
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
    }
  } else {
    R* b1 = b;
    R* b2 = b + 2 * static_cast<ptrdiff_t>(r1) * ldb;
    if (lower) {
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
      ZGemmCore<R>(other, r1, r2, m1, col(b2), toff, one, b1, ldb);
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
    } else {
      ZTrsmRec<R>(left, t11, lower, unit, r1, other, b1, ldb);
      ZGemmCore<R>(other, r2, r1, m1, col(b1), toff, one, b2, ldb);
      ZTrsmRec<R>(left, t22, lower, unit, r2, other, b2, ldb);
    }
  }
}

template <typename R>
int ZtrsmF(char side, char uplo, char transa, char diag, int m, int n, const R* alpha,
           const R* a, int lda, R* b, int ldb) {
  const char s = Up(side), u = Up(uplo), d = Up(diag), t = Up(transa);
  const int op = t == 'N' ? 0 : t == 'T' ? 1 : t == 'C' ? 2 : -1;
  const bool left = (s == 'L');
  const int ka = left ? m : n;
  int info = 0;
  if (s != 'L' && s != 'R') info = 1;
  else if (u != 'L' && u != 'U') info = 2;
  else if (op < 0) info = 3;
  else if (d != 'U' && d != 'N') info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, ka)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info) return info;
  if (m == 0 || n == 0) return 0;
  const bool alpha_one = alpha[0] == R(1) && alpha[1] == R(0);
  const bool alpha_zero = alpha[0] == R(0) && alpha[1] == R(0);
  if (!alpha_one) {
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) {
        R* e = b + 2 * (i + static_cast<ptrdiff_t>(j) * ldb);
        if (alpha_zero) {
          e[0] = e[1] = R(0);
        } else {
          const R c0 = e[0], c1 = e[1];
          const R p0 = c0 * alpha[0], p1 = c1 * alpha[1], p2 = c0 * alpha[1], p3 = c1 * alpha[0];
          e[0] = p0 - p1;
          e[1] = p2 + p3;
        }
      }
  }
  if (alpha_zero) return 0;
  const ZOp<R> tri = op == 0 ? ZOp<R>{a, 1, lda, false} : ZOp<R>{a, lda, 1, op == 2};
  const bool op_lower = (u == 'L') != (op != 0);
  ZTrsmRec<R>(left, tri, op_lower, d == 'U', ka, left ? n : m, b, ldb);
  return 0;
}
// Complex HERK (src/level3.cc:85-140) through the GEMM problem model: every
// element of the triangle is the complex GEMM's (four FMA chains per KC
// chunk, ab = (rr - ii, ir + ri), t = alpha ab), merged as the micro-kernel
// merges in tiles wholly inside the triangle and as MergeTile does in tiles
// that cross the diagonal (src/gemm-inl.h:86-130): there the diagonal keeps
// only its real part and v += beta * c is the C++ runtime's complex product
// and sum (beta 1 after the first chunk). The complex micro-tile is
// lanes / 2 complex rows per vector, two vectors per column, and 6 columns
// (3 with 16 vector registers): src/gemm_kernel-inl.h:243-257. The quick
// path (alpha 0 or k 0) is ScaleMatrix with real_diagonal (src/gemm.cc:48-64).
template <typename R>
int ZherkF(char uplo, char trans, int n, int k, R alpha, const R* a, int lda, R beta, R* c,
           int ldc) {
  using T = std::complex<R>;
  const char u = Up(uplo), t = Up(trans);
  const bool lower = (u == 'L');
  int info = 0;
  if (u != 'L' && u != 'U') info = 1;
  else if (t != 'N' && t != 'C') info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, t == 'N' ? n : k)) info = 7;
  else if (ldc < std::max(1, n)) info = 10;
  if (info != 0) return info;
  T* C = reinterpret_cast<T*>(c);
  const auto at = [&](int i, int j) -> T& { return C[i + static_cast<ptrdiff_t>(j) * ldc]; };
  const auto is_zero = [](T v) { return v.real() == R(0) && v.imag() == R(0); };
  const T be = T(beta);
  if (n == 0 || ((alpha == R(0) || k == 0) && beta == R(1))) return 0;
  if (alpha == R(0) || k == 0) {
    for (int j = 0; j < n; ++j) {
      const int begin = lower ? j : 0, end = lower ? n : j + 1;
      at(j, j) = T(std::real(at(j, j)));
      for (int i = begin; i < end; ++i) {
        if (is_zero(be)) at(i, j) = T(0);
        else at(i, j) *= be;
      }
    }
    return 0;
  }
  const ZOp<R> plain{a, 1, lda, false}, herm{a, lda, 1, true};
  const ZOp<R> va = t == 'N' ? plain : herm, vb = t == 'N' ? herm : plain;
  const int mr = sizeof(R) == 8 ? g_lanes : 2 * g_lanes, nr = g_lanes >= 8 ? 6 : 3;
  constexpr int KC = 256;
  for (int j = 0; j < n; ++j) {
    for (int i = lower ? j : 0; i < (lower ? n : j + 1); ++i) {
      const int i0 = i / mr * mr, j0 = j / nr * nr;
      const int il = std::min(i0 + mr, n) - 1, jl = std::min(j0 + nr, n) - 1;
      const bool inside = lower ? i0 > jl : il < j0;
      for (int pc = 0; pc < k; pc += KC) {
        const int pe = std::min(k, pc + KC);
        R rr = R(0), ir = R(0), ri = R(0), ii = R(0);
        for (int p = pc; p < pe; ++p) {
          R ar, ai, br, bi;
          va.at(i, p, &ar, &ai);
          vb.at(p, j, &br, &bi);
          rr = std::fma(ar, br, rr);
          ir = std::fma(ai, br, ir);
          ri = std::fma(ar, bi, ri);
          ii = std::fma(ai, bi, ii);
        }
        const R ab_re = rr - ii, ab_im = ir + ri;
        const R q0 = ab_re * alpha, q1 = ab_im * R(0), q2 = ab_im * alpha, q3 = ab_re * R(0);
        const R t_re = q0 - q1, t_im = q2 + q3;
        const T cij = at(i, j);
        if (inside) {
          if (pc == 0 && beta == R(0)) {
            at(i, j) = T(t_re, t_im);
          } else if (pc != 0 || beta == R(1)) {
            at(i, j) = T(t_re + cij.real(), t_im + cij.imag());
          } else {
            const R s0 = cij.real() * beta, s1 = cij.imag() * R(0);
            const R s2 = cij.imag() * beta, s3 = cij.real() * R(0);
            at(i, j) = T(t_re + (s0 - s1), t_im + (s2 + s3));
          }
        } else {
          const T bc = pc == 0 ? be : T(1);
          T v(t_re, t_im);
          if (i == j) {
            v = T(std::real(v));
            if (!is_zero(bc)) v += bc * T(std::real(cij));
          } else if (!is_zero(bc)) {
            v += bc * cij;
          }
          at(i, j) = v;
        }
      }
    }
  }
  return 0;
}
template int ZherkF<double>(char, char, int, int, double, const double*, int, double, double*,
                            int);
template int ZherkF<float>(char, char, int, int, float, const float*, int, float, float*, int);

template int ZtrsmF<double>(char, char, char, char, int, int, const double*, const double*,
                            int, double*, int);
template int ZtrsmF<float>(char, char, char, char, int, int, const float*, const float*, int,
                           float*, int);

template int ZgemmF<double>(char, char, int, int, int, const double*, const double*, int,
                            const double*, int, const double*, double*, int);
template int ZgemmF<float>(char, char, int, int, int, const float*, const float*, int,
                           const float*, int, const float*, float*, int);

// ---------------------------------------------------------------------------
// IAMAX (src/level1.cc:383-402; src/level1-inl.h:343-423): 1-based index of
// the first element of largest |x|; NaNs never compare larger, so one is only
// returned when it is x[0].
template <typename T>
int Iamax(int n, const T* x, int incx) {
  if (n < 1 || incx <= 0) return 0;
  if (n == 1) return 1;
  int best = 1;
  T bv = std::fabs(x[0]);
  if (std::isnan(bv)) return 1;
  for (int i = 1; i < n; ++i) {
    const T v = std::fabs(x[static_cast<ptrdiff_t>(i) * incx]);
    if (v > bv) {
      best = i + 1;
      bv = v;
    }
  }
  return best;
}

template void Gemm<double>(size_t, size_t, size_t, double, Opnd<double>,
                           Opnd<double>, double, double*, size_t, Part);
template void Gemm<float>(size_t, size_t, size_t, float, Opnd<float>,
                          Opnd<float>, float, float*, size_t, Part);
template int GemmF<double>(char, char, int, int, int, double, const double*,
                           int, const double*, int, double, double*, int);
template int GemmF<float>(char, char, int, int, int, float, const float*, int,
                          const float*, int, float, float*, int);
template int TrsmF<double>(char, char, char, char, int, int, double,
                           const double*, int, double*, int);
template int TrsmF<float>(char, char, char, char, int, int, float,
                          const float*, int, float*, int);
template int Iamax<double>(int, const double*, int);
template int Iamax<float>(int, const float*, int);

}  // namespace orc

extern "C" {
void orc_set_lanes(int lanes) { orc::g_lanes = (lanes >= 8) ? 8 : 4; }
int orc_get_lanes(void) { return orc::g_lanes; }
void orc_set_threads(int threads) { orc::g_threads = threads < 1 ? 1 : threads; }

int orc_dgemm(char ta, char tb, int m, int n, int k, double alpha,
              const double* a, int lda, const double* b, int ldb, double beta,
              double* c, int ldc) {
  return orc::GemmF<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c,
                            ldc);
}
int orc_sgemm(char ta, char tb, int m, int n, int k, float alpha,
              const float* a, int lda, const float* b, int ldb, float beta,
              float* c, int ldc) {
  return orc::GemmF<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c,
                           ldc);
}
int orc_dtrsm(char side, char uplo, char transa, char diag, int m, int n,
              double alpha, const double* a, int lda, double* b, int ldb) {
  return orc::TrsmF<double>(side, uplo, transa, diag, m, n, alpha, a, lda, b,
                            ldb);
}
int orc_strsm(char side, char uplo, char transa, char diag, int m, int n,
              float alpha, const float* a, int lda, float* b, int ldb) {
  return orc::TrsmF<float>(side, uplo, transa, diag, m, n, alpha, a, lda, b,
                           ldb);
}
int orc_dsyrk(char uplo, char trans, int n, int k, double alpha,
              const double* a, int lda, double beta, double* c, int ldc) {
  return orc::SyrkD(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_ssyrk(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
              float beta, float* c, int ldc) {
  return orc::Syrk<float>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_zgemm(char ta, char tb, int m, int n, int k, const double* alpha, const double* a,
              int lda, const double* b, int ldb, const double* beta, double* c, int ldc) {
  return orc::ZgemmF<double>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
int orc_cgemm(char ta, char tb, int m, int n, int k, const float* alpha, const float* a,
              int lda, const float* b, int ldb, const float* beta, float* c, int ldc) {
  return orc::ZgemmF<float>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

int orc_zherk(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
              double beta, double* c, int ldc) {
  return orc::ZherkF<double>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_cherk(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
              float beta, float* c, int ldc) {
  return orc::ZherkF<float>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}
int orc_ztrsm(char side, char uplo, char ta, char diag, int m, int n, const double* alpha,
              const double* a, int lda, double* b, int ldb) {
  return orc::ZtrsmF<double>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
int orc_ctrsm(char side, char uplo, char ta, char diag, int m, int n, const float* alpha,
              const float* a, int lda, float* b, int ldb) {
  return orc::ZtrsmF<float>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
}
// The complex reciprocal as the C++ runtime computes it, for pinning the
// device's restatement (Smith's method for double; float in double).
void orc_zrecip(int n, const double* c, double* out) {
  for (int i = 0; i < n; ++i) {
    const std::complex<double> v = std::complex<double>(1) / std::complex<double>(c[2 * i], c[2 * i + 1]);
    out[2 * i] = v.real();
    out[2 * i + 1] = v.imag();
  }
}
void orc_crecip(int n, const float* c, float* out) {
  for (int i = 0; i < n; ++i) {
    const std::complex<float> v = std::complex<float>(1) / std::complex<float>(c[2 * i], c[2 * i + 1]);
    out[2 * i] = v.real();
    out[2 * i + 1] = v.imag();
  }
}

#define ORC_L3(P, T)                                                                       \
  int orc_##P##symm(char side, char uplo, int m, int n, T alpha, const T* a, int lda,       \
                    const T* b, int ldb, T beta, T* c, int ldc) {                            \
    return orc::Symm<T>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);             \
  }                                                                                          \
  int orc_##P##syr2k(char uplo, char trans, int n, int k, T alpha, const T* a, int lda,     \
                     const T* b, int ldb, T beta, T* c, int ldc) {                           \
    return orc::Syr2k<T>(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);           \
  }                                                                                          \
  int orc_##P##gemmtr(char uplo, char ta, char tb, int n, int k, T alpha, const T* a,       \
                      int lda, const T* b, int ldb, T beta, T* c, int ldc) {                 \
    return orc::Gemmtr<T>(uplo, ta, tb, n, k, alpha, a, lda, b, ldb, beta, c, ldc);         \
  }                                                                                          \
  int orc_##P##trmm(char side, char uplo, char transa, char diag, int m, int n, T alpha,    \
                    const T* a, int lda, T* b, int ldb) {                                    \
    return orc::Trmm<T>(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb);             \
  }
ORC_L3(d, double)
ORC_L3(s, float)
#undef ORC_L3

int orc_idamax(int n, const double* x, int incx) {
  return orc::Iamax<double>(n, x, incx);
}
int orc_isamax(int n, const float* x, int incx) {
  return orc::Iamax<float>(n, x, incx);
}
}  // extern "C"
