// LU and Cholesky drivers on device data. They follow the reference's
// blocked/recursive structure call for call, because the rounding of every
// element depends on how the updates are split:
//   Getrf2  src/lapack/getrf.cc:112-207 (leaf at min(m, n) <= 16,
//           src/lapack/factor_kernels.h:27)
//   Getrf   src/lapack/getrf.cc:216-280 (nb = 64, src/lapack/environment.cc:86-88)
//   Getrs   src/lapack/getrf.cc:287-339
//   Potrf2  src/lapack/potrf.cc:48-119 (leaf at n <= 32)
//   Potrf   src/lapack/potrf.cc:128-199 (nb = 64, environment.cc:110-111)
//   Potrs   src/lapack/posv.cc:31-76
// Every step is a kernel launch on the context's stream; pivots and INFO stay
// on the device until the C ABI copies them back.
#include <algorithm>

#include "internal.h"

namespace hb {

namespace {
template <typename T>
T* At(T* a, int lda, int i, int j) {
  return a + i + static_cast<long long>(j) * lda;
}
}  // namespace

// Getrf2's recursion; col0 is the global column of the block's first column
// (for INFO: columns are factored left to right, so each leaf sets the device
// INFO only while it is still 0, to col0 + its own first zero pivot).
template <typename T>
void GetrfRec(int m, int n, T* a, int lda, int* ipiv, int* info, int col0) {
  if (m == 0 || n == 0) return;
  if (std::min(m, n) <= 16) {
    GetrfLeaf<T>(m, n, a, lda, ipiv, info, col0);
    return;
  }
  const int n1 = std::min(m, n) / 2;
  const int n2 = n - n1;
  GetrfRec<T>(m, n1, a, lda, ipiv, info, col0);
  Laswp<T>(n2, At(a, lda, 0, n1), lda, 1, n1, ipiv, 1);
  TrsmFull<T>(true, true, false, true, n1, n2, T(1), a, lda, At(a, lda, 0, n1),
              lda);
  GemmFull<T>(false, false, m - n1, n2, n1, T(-1), At(a, lda, n1, 0), lda,
              At(a, lda, 0, n1), lda, T(1), At(a, lda, n1, n1), lda);
  GetrfRec<T>(m - n1, n2, At(a, lda, n1, n1), lda, ipiv + n1, info, col0 + n1);
  AdjustPivots(ipiv, n1, std::min(m, n), n1);
  Laswp<T>(n1, a, lda, n1 + 1, std::min(m, n), ipiv, 1);
}

template <typename T>
void Getrf2(int m, int n, T* a, int lda, int* ipiv, int* info) {
  GetrfRec<T>(m, n, a, lda, ipiv, info, 0);
}

template <typename T>
void Getrf(int m, int n, T* a, int lda, int* ipiv, int* info) {
  if (m == 0 || n == 0) return;
  const int nb = 64;
  const int mn = std::min(m, n);
  if (nb >= mn) {
    GetrfRec<T>(m, n, a, lda, ipiv, info, 0);
    return;
  }
  for (int j = 0; j < mn; j += nb) {
    const int jb = std::min(mn - j, nb);
    GetrfRec<T>(m - j, jb, At(a, lda, j, j), lda, ipiv + j, info, j);
    AdjustPivots(ipiv, j, std::min(m, j + jb), j);
    Laswp<T>(j, a, lda, j + 1, j + jb, ipiv, 1);
    if (j + jb < n) {
      Laswp<T>(n - j - jb, At(a, lda, 0, j + jb), lda, j + 1, j + jb, ipiv, 1);
      TrsmFull<T>(true, true, false, true, jb, n - j - jb, T(1), At(a, lda, j, j),
                  lda, At(a, lda, j, j + jb), lda);
      if (j + jb < m) {
        GemmFull<T>(false, false, m - j - jb, n - j - jb, jb, T(-1),
                    At(a, lda, j + jb, j), lda, At(a, lda, j, j + jb), lda, T(1),
                    At(a, lda, j + jb, j + jb), lda);
      }
    }
  }
}

template <typename T>
void Getrs(bool trans, int n, int nrhs, const T* a, int lda, const int* ipiv,
           T* b, int ldb) {
  if (n == 0 || nrhs == 0) return;
  if (!trans) {
    Laswp<T>(nrhs, b, ldb, 1, n, ipiv, 1);
    TrsmFull<T>(true, true, false, true, n, nrhs, T(1), a, lda, b, ldb);
    TrsmFull<T>(true, false, false, false, n, nrhs, T(1), a, lda, b, ldb);
  } else {
    TrsmFull<T>(true, false, true, false, n, nrhs, T(1), a, lda, b, ldb);
    TrsmFull<T>(true, true, true, true, n, nrhs, T(1), a, lda, b, ldb);
    Laswp<T>(nrhs, b, ldb, 1, n, ipiv, -1);
  }
}

// Cholesky: the device INFO doubles as the guard that turns every later
// kernel of the call into a no-op once a leaf has found a non-positive minor
// (the reference returns at that point, src/lapack/potrf.cc:86-87, 173).
namespace {
template <typename T>
void Potrf2Rec(bool upper, int n, T* a, int lda, int* info, int col0) {
  if (n == 0) return;
  if (n <= 32) {
    PotrfLeaf<T>(upper, n, a, lda, info, col0);
    return;
  }
  const int n1 = n / 2, n2 = n - n1;
  Potrf2Rec<T>(upper, n1, a, lda, info, col0);
  if (upper) {
    TrsmFull<T>(true, false, true, false, n1, n2, T(1), a, lda,
                     At(a, lda, 0, n1), lda);
    SyrkFull<T>(false, true, n2, n1, T(-1), At(a, lda, 0, n1), lda, 1.0,
             At(a, lda, n1, n1), lda);
  } else {
    TrsmFull<T>(false, true, true, false, n2, n1, T(1), a, lda,
                     At(a, lda, n1, 0), lda);
    SyrkFull<T>(true, false, n2, n1, T(-1), At(a, lda, n1, 0), lda, 1.0,
             At(a, lda, n1, n1), lda);
  }
  Potrf2Rec<T>(upper, n2, At(a, lda, n1, n1), lda, info, col0 + n1);
}
}  // namespace

template <typename T>
void Potrf2(bool upper, int n, T* a, int lda, int* info) {
  Context& ctx = Ctx();
  const int* saved = ctx.guard;
  ctx.guard = info;
  Potrf2Rec<T>(upper, n, a, lda, info, 0);
  ctx.guard = saved;
}

void PotrfPanel(bool upper, int n, double* a, int lda, int* info, int col0) {
  Context& ctx = Ctx();
  const int* saved = ctx.guard;
  ctx.guard = info;
  Potrf2Rec(upper, n, a, lda, info, col0);
  ctx.guard = saved;
}

template <typename T>
void Potrf(bool upper, int n, T* a, int lda, int* info) {
  if (n == 0) return;
  const int nb = 64;
  if (nb >= n) {
    Potrf2<T>(upper, n, a, lda, info);
    return;
  }
  Context& ctx = Ctx();
  const int* saved = ctx.guard;
  ctx.guard = info;
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    if (upper) {
      SyrkFull<T>(false, true, jb, j, T(-1), At(a, lda, 0, j), lda, 1.0,
               At(a, lda, j, j), lda);
      Potrf2Rec<T>(true, jb, At(a, lda, j, j), lda, info, j);
      if (j + jb < n) {
        GemmFull<T>(true, false, jb, n - j - jb, j, T(-1), At(a, lda, 0, j),
                         lda, At(a, lda, 0, j + jb), lda, 1.0,
                         At(a, lda, j, j + jb), lda);
        TrsmFull<T>(true, false, true, false, jb, n - j - jb, 1.0,
                         At(a, lda, j, j), lda, At(a, lda, j, j + jb), lda);
      }
    } else {
      SyrkFull<T>(true, false, jb, j, T(-1), At(a, lda, j, 0), lda, 1.0,
               At(a, lda, j, j), lda);
      Potrf2Rec<T>(false, jb, At(a, lda, j, j), lda, info, j);
      if (j + jb < n) {
        GemmFull<T>(false, true, n - j - jb, jb, j, -1.0,
                         At(a, lda, j + jb, 0), lda, At(a, lda, j, 0), lda, 1.0,
                         At(a, lda, j + jb, j), lda);
        TrsmFull<T>(false, true, true, false, n - j - jb, jb, 1.0,
                         At(a, lda, j, j), lda, At(a, lda, j + jb, j), lda);
      }
    }
  }
  ctx.guard = saved;
}

template <typename T>
void Potrs(bool upper, int n, int nrhs, const T* a, int lda, T* b, int ldb) {
  if (n == 0 || nrhs == 0) return;
  if (upper) {
    TrsmFull<T>(true, false, true, false, n, nrhs, T(1), a, lda, b, ldb);
    TrsmFull<T>(true, false, false, false, n, nrhs, T(1), a, lda, b, ldb);
  } else {
    TrsmFull<T>(true, true, false, false, n, nrhs, T(1), a, lda, b, ldb);
    TrsmFull<T>(true, true, true, false, n, nrhs, T(1), a, lda, b, ldb);
  }
}

template void Potrf2<double>(bool, int, double*, int, int*);
template void Potrf2<float>(bool, int, float*, int, int*);
template void Potrf<double>(bool, int, double*, int, int*);
template void Potrf<float>(bool, int, float*, int, int*);
template void Potrs<double>(bool, int, int, const double*, int, double*, int);
template void Potrs<float>(bool, int, int, const float*, int, float*, int);
template void Getrf2<double>(int, int, double*, int, int*, int*);
template void Getrf2<float>(int, int, float*, int, int*, int*);
template void Getrf<double>(int, int, double*, int, int*, int*);
template void Getrf<float>(int, int, float*, int, int*, int*);
template void Getrs<double>(bool, int, int, const double*, int, const int*,
                            double*, int);
template void Getrs<float>(bool, int, int, const float*, int, const int*,
                           float*, int);

}  // namespace hb
