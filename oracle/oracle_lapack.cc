// Oracle LAPACK (TEST INFRASTRUCTURE ONLY; the product never loads this
// file's library). CPU restatement of the reference's LU and Cholesky drivers
// on top of the oracle BLAS, with the reference's operation order:
//
//   GetrfLeaf  src/lapack/factor_kernels.cc:79-183 (pivot as IAMAX, row swap
//              across the leaf, 1/pivot unless |pivot| < sfmin, AXPY updates;
//              columns shorter than one vector use y + alpha*x with two
//              roundings, longer ones fma(x, alpha, y))
//   PotrfLeaf  src/lapack/factor_kernels.cc:187-221
//   Laswp      src/lapack/getrf.cc:28-81
//   Getrf2     src/lapack/getrf.cc:112-207 (leaf at min(m, n) <= 16)
//              (the same templates at std::complex: the leaf's pivot is the
//              first largest |re| + |im|, src/level1-inl.h:343-411, and its
//              complex AXPY src/lapack/factor_kernels.cc:33-72)
//   Getrf      src/lapack/getrf.cc:216-280 (nb = 64, src/lapack/environment.cc:86-88)
//   Getrs/Gesv src/lapack/getrf.cc:287-374
//   Potrf2     src/lapack/potrf.cc:48-119 (leaf at n <= 32)
//   Potrf      src/lapack/potrf.cc:128-199 (nb = 64, environment.cc:110-111)
//   Potrs/Posv src/lapack/posv.cc:31-114
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <limits>
#include <type_traits>
#include <utility>

#include "oracle.h"
#include "oracle_internal.h"

namespace orc {

template <typename T>
static T Sfmin() {
  return sizeof(T) == 8 ? static_cast<T>(DBL_MIN) : static_cast<T>(FLT_MIN);
}

// Lanes of the reference's vectors of T.
template <typename T>
static size_t LanesOf() {
  return sizeof(T) == 8 ? g_lanes : 2 * g_lanes;
}

// y[0:n] += alpha * x[0:n] (src/lapack/factor_kernels.cc:79-118).
template <typename T>
static void AxpyColumn(size_t n, T alpha, const T* x, T* y) {
  if (n < LanesOf<T>()) {
    for (size_t i = 0; i < n; ++i) {
      const T p = alpha * x[i];
      y[i] = y[i] + p;
    }
    return;
  }
  for (size_t i = 0; i < n; ++i) y[i] = std::fma(x[i], alpha, y[i]);
}

template <typename T>
struct IsCplx : std::false_type {};
template <typename R>
struct IsCplx<std::complex<R>> : std::true_type {};
template <typename T>
struct RealOf {
  using type = T;
};
template <typename R>
struct RealOf<std::complex<R>> {
  using type = R;
};

// y[0:n] += alpha * x[0:n] for complex elements (src/lapack/factor_kernels.cc:
// 33-72): fewer reals than one vector, the complex product and sum of the
// C++ runtime; otherwise per element re: fma(xi, -ai, fma(xr, ar, yr)),
// im: fma(xr, ai, fma(xi, ar, yi)).
template <typename R>
static void AxpyColumn(size_t n, std::complex<R> alpha, const std::complex<R>* x,
                       std::complex<R>* y) {
  if (2 * n < LanesOf<R>()) {
    for (size_t i = 0; i < n; ++i) y[i] += alpha * x[i];
    return;
  }
  const R ar = alpha.real(), ai = alpha.imag();
  for (size_t i = 0; i < n; ++i) {
    const R xr = x[i].real(), xi = x[i].imag();
    const R tr = std::fma(xr, ar, y[i].real()), ti = std::fma(xi, ar, y[i].imag());
    y[i] = std::complex<R>(std::fma(xi, -ai, tr), std::fma(xr, ai, ti));
  }
}

// 0-based index of the first element of largest |re| + |im| (NaNs never
// win; a NaN first element is returned: src/level1-inl.h:343-411).
template <typename R>
static size_t ArgMaxMagnitude(size_t n, const std::complex<R>* x) {
  const R first = std::fabs(x[0].real()) + std::fabs(x[0].imag());
  if (std::isnan(first)) return 0;
  R best = first;
  size_t bi = 0;
  for (size_t i = 1; i < n; ++i) {
    const R v = std::fabs(x[i].real()) + std::fabs(x[i].imag());
    if (v > best) {
      best = v;
      bi = i;
    }
  }
  return bi;
}

template <typename T>
int GetrfLeaf(int m_, int n_, T* a, int lda, int* ipiv) {
  using R = typename RealOf<T>::type;
  const size_t m = m_, n = n_;
  const auto at = [&](size_t i, size_t j) -> T& { return a[i + j * lda]; };
  const R sfmin = Sfmin<R>();
  int info = 0;
  for (size_t j = 0; j < std::min(m, n); ++j) {
    size_t p;
    if constexpr (IsCplx<T>::value) {
      p = j + ArgMaxMagnitude<R>(m - j, &at(j, j));
    } else {
      p = j + static_cast<size_t>(Iamax<T>(m - j, &at(j, j), 1) - 1);
    }
    ipiv[j] = static_cast<int>(p + 1);
    const T pivot = at(p, j);
    if (pivot != T(0)) {
      if (p != j) {
        for (size_t k = 0; k < n; ++k) std::swap(at(j, k), at(p, k));
      }
      if (std::abs(pivot) >= sfmin) {
        const T r = T(1) / pivot;
        for (size_t i = j + 1; i < m; ++i) at(i, j) = at(i, j) * r;
      } else {
        for (size_t i = j + 1; i < m; ++i) at(i, j) = at(i, j) / pivot;
      }
    } else if (info == 0) {
      info = static_cast<int>(j + 1);
    }
    for (size_t k = j + 1; k < n; ++k) {
      AxpyColumn(m - j - 1, -at(j, k), &at(j + 1, j), &at(j + 1, k));
    }
  }
  return info;
}

template <typename T>
static T ConjOf(T v) {
  if constexpr (IsCplx<T>::value) {
    return std::conj(v);
  } else {
    return v;
  }
}

// For complex T (src/lapack/factor_kernels.cc:141-175): only the real part
// of the diagonal is tested; it becomes (sqrt, 0), and rows (upper) or
// columns (lower) are scaled part by part by the real 1 / sqrt.
template <typename T>
int PotrfLeaf(bool upper, int n_, T* a, int lda) {
  using R = typename RealOf<T>::type;
  const size_t n = n_;
  const auto at = [&](size_t i, size_t j) -> T& { return a[i + j * lda]; };
  T row[64];
  for (size_t j = 0; j < n; ++j) {
    R ajj = std::real(at(j, j));
    if (ajj <= R(0) || std::isnan(ajj)) return static_cast<int>(j + 1);
    ajj = std::sqrt(ajj);
    at(j, j) = T(ajj);
    const R rinv = R(1) / ajj;
    if (upper) {
      for (size_t k = j + 1; k < n; ++k) {
        at(j, k) = at(j, k) * rinv;
        row[k] = ConjOf(at(j, k));
      }
      for (size_t k = j + 1; k < n; ++k) {
        AxpyColumn(k - j, -at(j, k), &row[j + 1], &at(j + 1, k));
      }
    } else {
      for (size_t i = j + 1; i < n; ++i) at(i, j) = at(i, j) * rinv;
      for (size_t k = j + 1; k < n; ++k) {
        AxpyColumn(n - k, -ConjOf(at(k, j)), &at(k, j), &at(k, k));
      }
    }
  }
  return 0;
}

// TRSM and GEMM of the drivers: the restated real routines, or the complex
// ones on interleaved (re, im) arrays.
template <typename T>
static int TrsmAny(char side, char uplo, char ta, char diag, int m, int n, T alpha, const T* a,
                   int lda, T* b, int ldb) {
  if constexpr (IsCplx<T>::value) {
    using R = typename RealOf<T>::type;
    return ZtrsmF<R>(side, uplo, ta, diag, m, n, reinterpret_cast<const R*>(&alpha),
                     reinterpret_cast<const R*>(a), lda, reinterpret_cast<R*>(b), ldb);
  } else {
    return TrsmF<T>(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb);
  }
}
template <typename T>
static int SyrkAny(char uplo, char trans, int n, int k, typename RealOf<T>::type alpha,
                   const T* a, int lda, typename RealOf<T>::type beta, T* c, int ldc) {
  if constexpr (IsCplx<T>::value) {
    using R = typename RealOf<T>::type;
    return ZherkF<R>(uplo, trans, n, k, alpha, reinterpret_cast<const R*>(a), lda, beta,
                     reinterpret_cast<R*>(c), ldc);
  } else {
    return Syrk<T>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
  }
}
template <typename T>
static int GemmAny(char ta, char tb, int m, int n, int k, T alpha, const T* a, int lda,
                   const T* b, int ldb, T beta, T* c, int ldc) {
  if constexpr (IsCplx<T>::value) {
    using R = typename RealOf<T>::type;
    return ZgemmF<R>(ta, tb, m, n, k, reinterpret_cast<const R*>(&alpha),
                     reinterpret_cast<const R*>(a), lda, reinterpret_cast<const R*>(b), ldb,
                     reinterpret_cast<const R*>(&beta), reinterpret_cast<R*>(c), ldc);
  } else {
    return GemmF<T>(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
  }
}

// Row interchanges, 1-based k1..k2 and ipiv (src/lapack/getrf.cc:28-81).
// Blocking by columns does not change any column's result, so this applies
// the interchanges column by column.
template <typename T>
void Laswp(int n, T* a, int lda, int k1, int k2, const int* ipiv, int incx) {
  int i1, i2, inc, ix0;
  if (incx > 0) {
    ix0 = k1; i1 = k1; i2 = k2; inc = 1;
  } else if (incx < 0) {
    ix0 = k1 + (k1 - k2) * incx; i1 = k2; i2 = k1; inc = -1;
  } else {
    return;
  }
  for (int col = 0; col < n; ++col) {
    T* ac = a + static_cast<ptrdiff_t>(col) * lda;
    int ix = ix0;
    for (int i = i1; inc > 0 ? i <= i2 : i >= i2; i += inc) {
      const int ip = ipiv[ix - 1];
      if (ip != i) std::swap(ac[i - 1], ac[ip - 1]);
      ix += incx;
    }
  }
}

template <typename T>
int Getrf2(int m, int n, T* a, int lda, int* ipiv) {
  if (m < 0) return -1;
  if (n < 0) return -2;
  if (lda < std::max(1, m)) return -4;
  if (m == 0 || n == 0) return 0;
  if (std::min(m, n) <= 16) return GetrfLeaf<T>(m, n, a, lda, ipiv);
  int info = 0;
  const int n1 = std::min(m, n) / 2;
  const int n2 = n - n1;
  const auto A = [&](int i, int j) { return a + i + static_cast<ptrdiff_t>(j) * lda; };
  int iinfo = Getrf2<T>(m, n1, a, lda, ipiv);
  if (info == 0 && iinfo > 0) info = iinfo;
  Laswp<T>(n2, A(0, n1), lda, 1, n1, ipiv, 1);
  TrsmAny<T>('L', 'L', 'N', 'U', n1, n2, T(1), a, lda, A(0, n1), lda);
  GemmAny<T>('N', 'N', m - n1, n2, n1, T(-1), A(n1, 0), lda, A(0, n1), lda, T(1),
           A(n1, n1), lda);
  iinfo = Getrf2<T>(m - n1, n2, A(n1, n1), lda, ipiv + n1);
  if (info == 0 && iinfo > 0) info = iinfo + n1;
  for (int i = n1; i < std::min(m, n); ++i) ipiv[i] += n1;
  Laswp<T>(n1, a, lda, n1 + 1, std::min(m, n), ipiv, 1);
  return info;
}

template <typename T>
int Getrf(int m, int n, T* a, int lda, int* ipiv) {
  if (m < 0) return -1;
  if (n < 0) return -2;
  if (lda < std::max(1, m)) return -4;
  if (m == 0 || n == 0) return 0;
  const int nb = 64;
  const int mn = std::min(m, n);
  if (nb >= mn) return Getrf2<T>(m, n, a, lda, ipiv);
  const auto A = [&](int i, int j) { return a + i + static_cast<ptrdiff_t>(j) * lda; };
  int info = 0;
  for (int j = 0; j < mn; j += nb) {
    const int jb = std::min(mn - j, nb);
    const int iinfo = Getrf2<T>(m - j, jb, A(j, j), lda, ipiv + j);
    if (info == 0 && iinfo > 0) info = iinfo + j;
    for (int i = j; i < std::min(m, j + jb); ++i) ipiv[i] += j;
    Laswp<T>(j, a, lda, j + 1, j + jb, ipiv, 1);
    if (j + jb < n) {
      Laswp<T>(n - j - jb, A(0, j + jb), lda, j + 1, j + jb, ipiv, 1);
      TrsmAny<T>('L', 'L', 'N', 'U', jb, n - j - jb, T(1), A(j, j), lda,
               A(j, j + jb), lda);
      if (j + jb < m) {
        GemmAny<T>('N', 'N', m - j - jb, n - j - jb, jb, T(-1), A(j + jb, j),
                 lda, A(j, j + jb), lda, T(1), A(j + jb, j + jb), lda);
      }
    }
  }
  return info;
}

template <typename T>
int Getrs(char trans, int n, int nrhs, const T* a, int lda, const int* ipiv,
          T* b, int ldb) {
  const char t = (trans >= 'a' && trans <= 'z') ? trans - 32 : trans;
  const bool notran = (t == 'N');
  if (!notran && t != 'T' && t != 'C') return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (ldb < std::max(1, n)) return -8;
  if (n == 0 || nrhs == 0) return 0;
  if (notran) {
    Laswp<T>(nrhs, b, ldb, 1, n, ipiv, 1);
    TrsmAny<T>('L', 'L', 'N', 'U', n, nrhs, T(1), a, lda, b, ldb);
    TrsmAny<T>('L', 'U', 'N', 'N', n, nrhs, T(1), a, lda, b, ldb);
  } else {
    TrsmAny<T>('L', 'U', t, 'N', n, nrhs, T(1), a, lda, b, ldb);
    TrsmAny<T>('L', 'L', t, 'U', n, nrhs, T(1), a, lda, b, ldb);
    Laswp<T>(nrhs, b, ldb, 1, n, ipiv, -1);
  }
  return 0;
}

template <typename T>
int Potrf2(char uplo, int n, T* a, int lda) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;
  const bool upper = (u == 'U');
  if (!upper && u != 'L') return -1;
  if (n < 0) return -2;
  if (lda < std::max(1, n)) return -4;
  if (n == 0) return 0;
  if (n <= 32) return PotrfLeaf<T>(upper, n, a, lda);
  const int n1 = n / 2, n2 = n - n1;
  const auto A = [&](int i, int j) { return a + i + static_cast<ptrdiff_t>(j) * lda; };
  int iinfo = Potrf2<T>(uplo, n1, a, lda);
  if (iinfo != 0) return iinfo;
  if (upper) {
    TrsmAny<T>('L', 'U', 'C', 'N', n1, n2, T(1), a, lda, A(0, n1), lda);
    SyrkAny<T>('U', 'C', n2, n1, -1, A(0, n1), lda, 1, A(n1, n1), lda);
  } else {
    TrsmAny<T>('R', 'L', 'C', 'N', n2, n1, T(1), a, lda, A(n1, 0), lda);
    SyrkAny<T>('L', 'N', n2, n1, -1, A(n1, 0), lda, 1, A(n1, n1), lda);
  }
  iinfo = Potrf2<T>(uplo, n2, A(n1, n1), lda);
  if (iinfo != 0) return iinfo + n1;
  return 0;
}

template <typename T>
int Potrf(char uplo, int n, T* a, int lda) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;
  const bool upper = (u == 'U');
  if (!upper && u != 'L') return -1;
  if (n < 0) return -2;
  if (lda < std::max(1, n)) return -4;
  if (n == 0) return 0;
  const int nb = 64;
  if (nb >= n) return Potrf2<T>(uplo, n, a, lda);
  const auto A = [&](int i, int j) { return a + i + static_cast<ptrdiff_t>(j) * lda; };
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    if (upper) {
      SyrkAny<T>('U', 'C', jb, j, -1, A(0, j), lda, 1, A(j, j), lda);
      const int info = Potrf2<T>('U', jb, A(j, j), lda);
      if (info != 0) return info + j;
      if (j + jb < n) {
        GemmAny<T>('C', 'N', jb, n - j - jb, j, T(-1), A(0, j), lda,
                      A(0, j + jb), lda, T(1), A(j, j + jb), lda);
        TrsmAny<T>('L', 'U', 'C', 'N', jb, n - j - jb, T(1), A(j, j), lda,
                      A(j, j + jb), lda);
      }
    } else {
      SyrkAny<T>('L', 'N', jb, j, -1, A(j, 0), lda, 1, A(j, j), lda);
      const int info = Potrf2<T>('L', jb, A(j, j), lda);
      if (info != 0) return info + j;
      if (j + jb < n) {
        GemmAny<T>('N', 'C', n - j - jb, jb, j, T(-1), A(j + jb, 0), lda,
                      A(j, 0), lda, T(1), A(j + jb, j), lda);
        TrsmAny<T>('R', 'L', 'C', 'N', n - j - jb, jb, T(1), A(j, j), lda,
                      A(j + jb, j), lda);
      }
    }
  }
  return 0;
}

template <typename T>
int Potrs(char uplo, int n, int nrhs, const T* a, int lda, T* b, int ldb) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;
  const bool upper = (u == 'U');
  if (!upper && u != 'L') return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (ldb < std::max(1, n)) return -7;
  if (n == 0 || nrhs == 0) return 0;
  if (upper) {
    TrsmAny<T>('L', 'U', 'C', 'N', n, nrhs, T(1), a, lda, b, ldb);
    TrsmAny<T>('L', 'U', 'N', 'N', n, nrhs, T(1), a, lda, b, ldb);
  } else {
    TrsmAny<T>('L', 'L', 'N', 'N', n, nrhs, T(1), a, lda, b, ldb);
    TrsmAny<T>('L', 'L', 'C', 'N', n, nrhs, T(1), a, lda, b, ldb);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Triangular inverse and GETRI (src/lapack/triangular.cc:18-166;
// src/lapack/getrf.cc:369-483), in the reference's call order: TRTI2 column
// by column (an exact reciprocal of the diagonal, then TRMV of the finished
// part and a scaling by -A(j, j)), TRTRI in blocks of 64 with TRMM, TRSM and
// TRTI2, and GETRI solving inv(A) L = inv(U) block column by block column
// from the right (GEMM and TRSM; GEMV unblocked) before undoing the column
// interchanges.

static char UpC(char c) { return (c >= 'a' && c <= 'z') ? c - 32 : c; }

template <typename T>
int Trti2(char uplo, char diag, int n, T* a, int lda) {
  const bool upper = UpC(uplo) == 'U', nounit = UpC(diag) == 'N';
  if (!upper && UpC(uplo) != 'L') return -1;
  if (!nounit && UpC(diag) != 'U') return -2;
  if (n < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  const auto A = [&](int i, int j) -> T& { return a[i + static_cast<ptrdiff_t>(j) * lda]; };
  const auto scal = [](int len, T alpha, T* x) {
    if (len <= 0 || alpha == T(1)) return;
    for (int i = 0; i < len; ++i) x[i] *= alpha;
  };
  if (upper) {
    for (int j = 0; j < n; ++j) {
      T ajj = T(-1);
      if (nounit) {
        A(j, j) = T(1) / A(j, j);
        ajj = -A(j, j);
      }
      TrmvN<T>(false, !nounit, j, a, lda, &A(0, j));
      scal(j, ajj, &A(0, j));
    }
  } else {
    for (int j = n - 1; j >= 0; --j) {
      T ajj = T(-1);
      if (nounit) {
        A(j, j) = T(1) / A(j, j);
        ajj = -A(j, j);
      }
      if (j < n - 1) {
        TrmvN<T>(true, !nounit, n - j - 1, &A(j + 1, j + 1), lda, &A(j + 1, j));
        scal(n - j - 1, ajj, &A(j + 1, j));
      }
    }
  }
  return 0;
}

template <typename T>
int Trtri(char uplo, char diag, int n, T* a, int lda) {
  const bool upper = UpC(uplo) == 'U', nounit = UpC(diag) == 'N';
  if (!upper && UpC(uplo) != 'L') return -1;
  if (!nounit && UpC(diag) != 'U') return -2;
  if (n < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (n == 0) return 0;
  const auto A = [&](int i, int j) { return a + i + static_cast<ptrdiff_t>(j) * lda; };
  if (nounit) {
    for (int i = 0; i < n; ++i)
      if (*A(i, i) == T(0)) return i + 1;
  }
  const char d = nounit ? 'N' : 'U';
  constexpr int nb = 64;  // ILAENV(1, xTRTRI) (src/lapack/environment.cc:134-137)
  if (nb >= n) return Trti2<T>(uplo, d, n, a, lda);
  if (upper) {
    for (int j = 0; j < n; j += nb) {
      const int jb = std::min(nb, n - j);
      Trmm<T>('L', 'U', 'N', d, j, jb, T(1), a, lda, A(0, j), lda);
      TrsmAny<T>('R', 'U', 'N', d, j, jb, T(-1), A(j, j), lda, A(0, j), lda);
      Trti2<T>('U', d, jb, A(j, j), lda);
    }
  } else {
    const int nn = ((n - 1) / nb) * nb;
    for (int j = nn; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      if (j + jb < n) {
        Trmm<T>('L', 'L', 'N', d, n - j - jb, jb, T(1), A(j + jb, j + jb), lda, A(j + jb, j),
                lda);
        TrsmAny<T>('R', 'L', 'N', d, n - j - jb, jb, T(-1), A(j, j), lda, A(j + jb, j), lda);
      }
      Trti2<T>('L', d, jb, A(j, j), lda);
    }
  }
  return 0;
}

// work/lwork as LAPACK's: lwork = -1 queries; the block width falls to
// lwork / n (unblocked below 2) when lwork < 64 n. work[0] returns the size
// used.
template <typename T>
int Getri(int n, T* a, int lda, const int* ipiv, T* work, int lwork) {
  int nb = 64;  // ILAENV(1, xGETRI) (src/lapack/environment.cc:105-106)
  const int lwkopt = std::max(1, n * nb);
  work[0] = static_cast<T>(lwkopt);
  const bool lquery = (lwork == -1);
  if (n < 0) return -1;
  if (lda < std::max(1, n)) return -3;
  if (lwork < std::max(1, n) && !lquery) return -6;
  if (lquery || n == 0) return 0;
  const int info = Trtri<T>('U', 'N', n, a, lda);
  if (info > 0) return info;
  const auto A = [&](int i, int j) -> T& { return a[i + static_cast<ptrdiff_t>(j) * lda]; };
  int nbmin = 2;
  const int ldwork = n;
  int iws;
  if (nb > 1 && nb < n) {
    iws = std::max(ldwork * nb, 1);
    if (lwork < iws) {
      nb = lwork / ldwork;
      nbmin = 2;  // ILAENV(2, xGETRI)
    }
  } else {
    iws = n;
  }
  if (nb < nbmin || nb >= n) {
    for (int j = n - 1; j >= 0; --j) {
      for (int i = j + 1; i < n; ++i) {
        work[i] = A(i, j);
        A(i, j) = T(0);
      }
      if (j < n - 1) GemvN<T>(n, n - j - 1, T(-1), &A(0, j + 1), lda, work + j + 1, T(1), &A(0, j));
    }
  } else {
    const int nn = ((n - 1) / nb) * nb;
    for (int j = nn; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      for (int jj = j; jj < j + jb; ++jj)
        for (int i = jj + 1; i < n; ++i) {
          work[i + static_cast<ptrdiff_t>(jj - j) * ldwork] = A(i, jj);
          A(i, jj) = T(0);
        }
      if (j + jb < n)
        GemmAny<T>('N', 'N', n, jb, n - j - jb, T(-1), &A(0, j + jb), lda, work + j + jb, ldwork,
                 T(1), &A(0, j), lda);
      TrsmAny<T>('R', 'L', 'N', 'U', n, jb, T(1), work + j, ldwork, &A(0, j), lda);
    }
  }
  for (int j = n - 2; j >= 0; --j) {
    const int jp = ipiv[j] - 1;
    if (jp != j)
      for (int i = 0; i < n; ++i) std::swap(A(i, j), A(i, jp));
  }
  work[0] = static_cast<T>(iws);
  return 0;
}

// ---------------------------------------------------------------------------
// GERFS (src/lapack/gesvx.cc:319-456) with its condition estimator xLACN2
// (src/lapack/trsen.cc:2243-2366), real types. Reverse communication as in
// LAPACK: kase 1 asks for x := op(A) x, kase 2 for x := op(A)^T x.

template <typename T>
static T MaxRef(T a, T b) {
  return a > b ? a : b;  // src/lapack/lapack_common.h:145-152
}

template <typename T>
void Lacn2(int n, T* v, T* x, int* isgn, T* est, int* kase, int* isave) {
  constexpr int itmax = 5;
  const auto sign_vector = [&]() {
    for (int i = 0; i < n; ++i) {
      x[i] = (x[i] >= T(0)) ? T(1) : T(-1);
      isgn[i] = static_cast<int>(std::lround(x[i]));
    }
  };
  const auto unit_vector = [&]() {
    for (int i = 0; i < n; ++i) x[i] = T(0);
    x[isave[1] - 1] = T(1);
    *kase = 1;
    isave[0] = 3;
  };
  const auto final_stage = [&]() {
    T altsgn = T(1);
    for (int i = 0; i < n; ++i) {
      x[i] = altsgn * (T(1) + T(i) / T(n - 1));
      altsgn = -altsgn;
    }
    *kase = 1;
    isave[0] = 5;
  };
  if (*kase == 0) {
    for (int i = 0; i < n; ++i) x[i] = T(1) / T(n);
    *kase = 1;
    isave[0] = 1;
    return;
  }
  switch (isave[0]) {
    default:  // an out-of-range state runs the first iteration's step
    case 1:  // x = A x, first iteration
      if (n == 1) {
        v[0] = x[0];
        *est = std::fabs(v[0]);
        *kase = 0;
        return;
      }
      *est = AbsSum<T>(n, x);
      sign_vector();
      *kase = 2;
      isave[0] = 2;
      return;
    case 2:  // x = A^T x, first iteration
      isave[1] = Iamax<T>(n, x, 1);
      isave[2] = 2;
      unit_vector();
      return;
    case 3: {  // x = A x
      for (int i = 0; i < n; ++i) v[i] = x[i];
      const T estold = *est;
      *est = AbsSum<T>(n, v);
      bool same = true;
      for (int i = 0; i < n && same; ++i) {
        const T xs = (x[i] >= T(0)) ? T(1) : T(-1);
        if (static_cast<int>(std::lround(xs)) != isgn[i]) same = false;
      }
      if (same || *est <= estold) {
        final_stage();
        return;
      }
      sign_vector();
      *kase = 2;
      isave[0] = 4;
      return;
    }
    case 4: {  // x = A^T x
      const int jlast = isave[1];
      isave[1] = Iamax<T>(n, x, 1);
      if (x[jlast - 1] != std::fabs(x[isave[1] - 1]) && isave[2] < itmax) {
        isave[2] = isave[2] + 1;
        unit_vector();
        return;
      }
      final_stage();
      return;
    }
    case 5: {  // x = A x, final stage
      const T temp = T(2) * (AbsSum<T>(n, x) / T(3 * n));
      if (temp > *est) {
        for (int i = 0; i < n; ++i) v[i] = x[i];
        *est = temp;
      }
      *kase = 0;
      return;
    }
  }
}

template <typename T>
int Gerfs(char trans, int n, int nrhs, const T* a, int lda, const T* af, int ldaf,
          const int* ipiv, const T* b, int ldb, T* x, int ldx, T* ferr, T* berr, T* work,
          int* iwork) {
  constexpr int itmax = 5;
  const char t = UpC(trans);
  const bool notran = (t == 'N');
  if (!notran && t != 'T' && t != 'C') return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (ldaf < std::max(1, n)) return -7;
  if (ldb < std::max(1, n)) return -10;
  if (ldx < std::max(1, n)) return -12;
  if (n == 0 || nrhs == 0) {
    for (int j = 0; j < nrhs; ++j) ferr[j] = berr[j] = T(0);
    return 0;
  }
  const char transn = notran ? 'N' : 'C', transt = notran ? 'C' : 'N';
  const int nz = n + 1;
  const T eps = std::numeric_limits<T>::epsilon() * T(0.5);
  const T safmin = std::numeric_limits<T>::min();
  const T safe1 = T(nz) * safmin;
  const T safe2 = safe1 / eps;
  T* rw = work;       // abs(op(A))*abs(X) + abs(B)
  T* wk = work + n;   // residual, then the estimator's x
  T* vv = work + 2 * n;
  const auto A = [&](int i, int k) { return a[i + static_cast<ptrdiff_t>(k) * lda]; };
  for (int j = 0; j < nrhs; ++j) {
    T* xj = x + static_cast<ptrdiff_t>(j) * ldx;
    const T* bj = b + static_cast<ptrdiff_t>(j) * ldb;
    int count = 1;
    T lstres = T(3);
    for (;;) {
      for (int i = 0; i < n; ++i) wk[i] = bj[i];
      if (notran) GemvN<T>(n, n, T(-1), a, lda, xj, T(1), wk);
      else GemvT<T>(n, n, T(-1), a, lda, xj, T(1), wk);
      for (int i = 0; i < n; ++i) rw[i] = std::fabs(bj[i]);
      if (notran) {
        for (int k = 0; k < n; ++k) {
          const T xk = std::fabs(xj[k]);
          for (int i = 0; i < n; ++i) {
            const T prod = std::fabs(A(i, k)) * xk;
            rw[i] = rw[i] + prod;
          }
        }
      } else {
        for (int k = 0; k < n; ++k) {
          T sum = T(0);
          for (int i = 0; i < n; ++i) {
            const T prod = std::fabs(A(i, k)) * std::fabs(xj[i]);
            sum = sum + prod;
          }
          rw[k] = rw[k] + sum;
        }
      }
      T sm = T(0);
      for (int i = 0; i < n; ++i) {
        if (rw[i] > safe2) {
          sm = MaxRef(sm, std::fabs(wk[i]) / rw[i]);
        } else {
          sm = MaxRef(sm, (std::fabs(wk[i]) + safe1) / (rw[i] + safe1));
        }
      }
      berr[j] = sm;
      if (berr[j] > eps && T(2) * berr[j] <= lstres && count <= itmax) {
        Getrs<T>(t, n, 1, af, ldaf, ipiv, wk, n);
        AxpyRef<T>(n, T(1), wk, xj);
        lstres = berr[j];
        count = count + 1;
        continue;
      }
      break;
    }
    for (int i = 0; i < n; ++i) {
      const T scaled = T(nz) * eps * rw[i];
      if (rw[i] > safe2) {
        rw[i] = std::fabs(wk[i]) + scaled;
      } else {
        rw[i] = std::fabs(wk[i]) + scaled + safe1;
      }
    }
    int kase = 0;
    int isave[3] = {0, 0, 0};
    for (;;) {
      Lacn2<T>(n, vv, wk, iwork, &ferr[j], &kase, isave);
      if (kase == 0) break;
      if (kase == 1) {
        Getrs<T>(transt, n, 1, af, ldaf, ipiv, wk, n);
        for (int i = 0; i < n; ++i) wk[i] = rw[i] * wk[i];
      } else {
        for (int i = 0; i < n; ++i) wk[i] = rw[i] * wk[i];
        Getrs<T>(transn, n, 1, af, ldaf, ipiv, wk, n);
      }
    }
    T lx = T(0);
    for (int i = 0; i < n; ++i) lx = MaxRef(lx, std::fabs(xj[i]));
    if (lx != T(0)) ferr[j] = ferr[j] / lx;
  }
  return 0;
}

int PotrfD(char uplo, int n, double* a, int lda) { return Potrf<double>(uplo, n, a, lda); }
int Potrf2D(char uplo, int n, double* a, int lda) { return Potrf2<double>(uplo, n, a, lda); }
int PotrsD(char uplo, int n, int nrhs, const double* a, int lda, double* b, int ldb) {
  return Potrs<double>(uplo, n, nrhs, a, lda, b, ldb);
}

template int GetrfLeaf<double>(int, int, double*, int, int*);
template int GetrfLeaf<float>(int, int, float*, int, int*);
template int GetrfLeaf<std::complex<double>>(int, int, std::complex<double>*, int, int*);
template int GetrfLeaf<std::complex<float>>(int, int, std::complex<float>*, int, int*);
template int PotrfLeaf<double>(bool, int, double*, int);
template int PotrfLeaf<float>(bool, int, float*, int);
template int PotrfLeaf<std::complex<double>>(bool, int, std::complex<double>*, int);
template int PotrfLeaf<std::complex<float>>(bool, int, std::complex<float>*, int);

}  // namespace orc

extern "C" {
void orc_dlaswp(int n, double* a, int lda, int k1, int k2, const int* ipiv,
                int incx) {
  orc::Laswp<double>(n, a, lda, k1, k2, ipiv, incx);
}
int orc_dtrti2(char uplo, char diag, int n, double* a, int lda) {
  return orc::Trti2<double>(uplo, diag, n, a, lda);
}
int orc_strti2(char uplo, char diag, int n, float* a, int lda) {
  return orc::Trti2<float>(uplo, diag, n, a, lda);
}
int orc_dtrtri(char uplo, char diag, int n, double* a, int lda) {
  return orc::Trtri<double>(uplo, diag, n, a, lda);
}
int orc_strtri(char uplo, char diag, int n, float* a, int lda) {
  return orc::Trtri<float>(uplo, diag, n, a, lda);
}
int orc_dgetri(int n, double* a, int lda, const int* ipiv, double* work, int lwork) {
  return orc::Getri<double>(n, a, lda, ipiv, work, lwork);
}
int orc_sgetri(int n, float* a, int lda, const int* ipiv, float* work, int lwork) {
  return orc::Getri<float>(n, a, lda, ipiv, work, lwork);
}
int orc_dgerfs(char trans, int n, int nrhs, const double* a, int lda, const double* af,
               int ldaf, const int* ipiv, const double* b, int ldb, double* x, int ldx,
               double* ferr, double* berr, double* work, int* iwork) {
  return orc::Gerfs<double>(trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, berr,
                            work, iwork);
}
int orc_sgerfs(char trans, int n, int nrhs, const float* a, int lda, const float* af,
               int ldaf, const int* ipiv, const float* b, int ldb, float* x, int ldx,
               float* ferr, float* berr, float* work, int* iwork) {
  return orc::Gerfs<float>(trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, berr,
                           work, iwork);
}
int orc_dgetrf(int m, int n, double* a, int lda, int* ipiv) {
  return orc::Getrf<double>(m, n, a, lda, ipiv);
}
int orc_dgetrf2(int m, int n, double* a, int lda, int* ipiv) {
  return orc::Getrf2<double>(m, n, a, lda, ipiv);
}
int orc_sgetrf(int m, int n, float* a, int lda, int* ipiv) {
  return orc::Getrf<float>(m, n, a, lda, ipiv);
}
/* The reference's s-prefixed LU family is the same template at float
 * (src/lapack/getrf.cc:507-546). */
int orc_sgetrf2(int m, int n, float* a, int lda, int* ipiv) {
  return orc::Getrf2<float>(m, n, a, lda, ipiv);
}
void orc_slaswp(int n, float* a, int lda, int k1, int k2, const int* ipiv, int incx) {
  orc::Laswp<float>(n, a, lda, k1, k2, ipiv, incx);
}
int orc_sgesv(int n, int nrhs, float* a, int lda, int* ipiv, float* b, int ldb) {
  if (n < 0) return -1;
  if (nrhs < 0) return -2;
  if (lda < std::max(1, n)) return -4;
  if (ldb < std::max(1, n)) return -7;
  int info = orc::Getrf<float>(n, n, a, lda, ipiv);
  if (info == 0) info = orc::Getrs<float>('N', n, nrhs, a, lda, ipiv, b, ldb);
  return info;
}
int orc_dgetrs(char trans, int n, int nrhs, const double* a, int lda,
               const int* ipiv, double* b, int ldb) {
  return orc::Getrs<double>(trans, n, nrhs, a, lda, ipiv, b, ldb);
}
int orc_sgetrs(char trans, int n, int nrhs, const float* a, int lda,
               const int* ipiv, float* b, int ldb) {
  return orc::Getrs<float>(trans, n, nrhs, a, lda, ipiv, b, ldb);
}
int orc_dgesv(int n, int nrhs, double* a, int lda, int* ipiv, double* b,
              int ldb) {
  if (n < 0) return -1;
  if (nrhs < 0) return -2;
  if (lda < std::max(1, n)) return -4;
  if (ldb < std::max(1, n)) return -7;
  int info = orc::Getrf<double>(n, n, a, lda, ipiv);
  if (info == 0) info = orc::Getrs<double>('N', n, nrhs, a, lda, ipiv, b, ldb);
  return info;
}
int orc_dpotrf(char uplo, int n, double* a, int lda) {
  return orc::PotrfD(uplo, n, a, lda);
}
int orc_dpotrf2(char uplo, int n, double* a, int lda) {
  return orc::Potrf2D(uplo, n, a, lda);
}
int orc_dpotrs(char uplo, int n, int nrhs, const double* a, int lda, double* b,
               int ldb) {
  return orc::PotrsD(uplo, n, nrhs, a, lda, b, ldb);
}
/* The reference's s-prefixed Cholesky family is the same template at float
 * (src/lapack/potrf.cc:747-773, posv.cc). */
int orc_spotrf(char uplo, int n, float* a, int lda) {
  return orc::Potrf<float>(uplo, n, a, lda);
}
int orc_spotrf2(char uplo, int n, float* a, int lda) {
  return orc::Potrf2<float>(uplo, n, a, lda);
}
int orc_spotrs(char uplo, int n, int nrhs, const float* a, int lda, float* b, int ldb) {
  return orc::Potrs<float>(uplo, n, nrhs, a, lda, b, ldb);
}
int orc_sposv(char uplo, int n, int nrhs, float* a, int lda, float* b, int ldb) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;
  if (u != 'U' && u != 'L') return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (ldb < std::max(1, n)) return -7;
  int info = orc::Potrf<float>(uplo, n, a, lda);
  if (info == 0) info = orc::Potrs<float>(uplo, n, nrhs, a, lda, b, ldb);
  return info;
}
int orc_dposv(char uplo, int n, int nrhs, double* a, int lda, double* b,
              int ldb) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;
  if (u != 'U' && u != 'L') return -1;
  if (n < 0) return -2;
  if (nrhs < 0) return -3;
  if (lda < std::max(1, n)) return -5;
  if (ldb < std::max(1, n)) return -7;
  int info = orc::PotrfD(uplo, n, a, lda);
  if (info == 0) info = orc::PotrsD(uplo, n, nrhs, a, lda, b, ldb);
  return info;
}
/* The complex LU family: the same templates at std::complex (src/lapack/
 * getrf.cc:548-549), interleaved (re, im) arrays. */
#define ORC_ZLU(P, R)                                                                      \
  int orc_##P##getrf(int m, int n, R* a, int lda, int* ipiv) {                            \
    return orc::Getrf<std::complex<R>>(m, n, reinterpret_cast<std::complex<R>*>(a), lda, ipiv); \
  }                                                                                        \
  int orc_##P##getrf2(int m, int n, R* a, int lda, int* ipiv) {                           \
    return orc::Getrf2<std::complex<R>>(m, n, reinterpret_cast<std::complex<R>*>(a), lda, ipiv); \
  }                                                                                        \
  void orc_##P##laswp(int n, R* a, int lda, int k1, int k2, const int* ipiv, int incx) {  \
    orc::Laswp<std::complex<R>>(n, reinterpret_cast<std::complex<R>*>(a), lda, k1, k2, ipiv, \
                                incx);                                                     \
  }                                                                                        \
  int orc_##P##getrs(char trans, int n, int nrhs, const R* a, int lda, const int* ipiv,   \
                     R* b, int ldb) {                                                      \
    return orc::Getrs<std::complex<R>>(trans, n, nrhs,                                     \
                                       reinterpret_cast<const std::complex<R>*>(a), lda,   \
                                       ipiv, reinterpret_cast<std::complex<R>*>(b), ldb);  \
  }                                                                                        \
  int orc_##P##gesv(int n, int nrhs, R* a, int lda, int* ipiv, R* b, int ldb) {           \
    if (n < 0) return -1;                                                                  \
    if (nrhs < 0) return -2;                                                               \
    if (lda < std::max(1, n)) return -4;                                                   \
    if (ldb < std::max(1, n)) return -7;                                                   \
    int info = orc_##P##getrf(n, n, a, lda, ipiv);                                         \
    if (info == 0) info = orc_##P##getrs('N', n, nrhs, a, lda, ipiv, b, ldb);              \
    return info;                                                                           \
  }
#define ORC_ZCHOL(P, R)                                                                    \
  int orc_##P##potrf(char uplo, int n, R* a, int lda) {                                    \
    return orc::Potrf<std::complex<R>>(uplo, n, reinterpret_cast<std::complex<R>*>(a), lda); \
  }                                                                                        \
  int orc_##P##potrf2(char uplo, int n, R* a, int lda) {                                   \
    return orc::Potrf2<std::complex<R>>(uplo, n, reinterpret_cast<std::complex<R>*>(a), lda); \
  }                                                                                        \
  int orc_##P##potrs(char uplo, int n, int nrhs, const R* a, int lda, R* b, int ldb) {     \
    return orc::Potrs<std::complex<R>>(uplo, n, nrhs,                                      \
                                       reinterpret_cast<const std::complex<R>*>(a), lda,   \
                                       reinterpret_cast<std::complex<R>*>(b), ldb);        \
  }                                                                                        \
  int orc_##P##posv(char uplo, int n, int nrhs, R* a, int lda, R* b, int ldb) {            \
    const char u = (uplo >= 'a' && uplo <= 'z') ? uplo - 32 : uplo;                        \
    if (u != 'U' && u != 'L') return -1;                                                   \
    if (n < 0) return -2;                                                                  \
    if (nrhs < 0) return -3;                                                               \
    if (lda < std::max(1, n)) return -5;                                                   \
    if (ldb < std::max(1, n)) return -7;                                                   \
    int info = orc_##P##potrf(uplo, n, a, lda);                                            \
    if (info == 0) info = orc_##P##potrs(uplo, n, nrhs, a, lda, b, ldb);                   \
    return info;                                                                           \
  }
ORC_ZCHOL(z, double)
ORC_ZCHOL(c, float)
#undef ORC_ZCHOL
ORC_ZLU(z, double)
ORC_ZLU(c, float)
#undef ORC_ZLU
int orc_dgetrf_leaf(int m, int n, double* a, int lda, int* ipiv) {
  return orc::GetrfLeaf<double>(m, n, a, lda, ipiv);
}
int orc_dpotrf_leaf(int upper, int n, double* a, int lda) {
  return orc::PotrfLeaf<double>(upper != 0, n, a, lda);
}
}  // extern "C"
