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
// SMs left to the side stream while the context stream's persistent GEMMs
// run (look-ahead): enough for a 16-CTA panel leaf and its small kernels.
constexpr int kSideSms = 20;

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

// Blocked LU with a look-ahead of one panel. The reference's sequence of
// calls per panel j (getrf.cc:243-276) is kept, and so is every element's
// arithmetic; only the order of calls that touch disjoint columns changes:
// on the side stream, panel j's interchanges, triangular solve and update
// are applied to the next panel's columns first and the next panel is
// factored, while the context's stream applies them to the columns left of
// the panel and to the rest of the trailing matrix. Events order the
// streams: the side stream's step j waits for the context stream's step
// j - 1 (which updated the next panel's columns), and the context stream's
// step j waits for the side stream's panel j. Splitting the triangular solve
// and the update by columns leaves every element's operations unchanged.
template <typename T>
void Getrf(int m, int n, T* a, int lda, int* ipiv, int* info) {
  if (m == 0 || n == 0) return;
  const int nb = 64;
  const int mn = std::min(m, n);
  if (nb >= mn) {
    GetrfRec<T>(m, n, a, lda, ipiv, info, 0);
    return;
  }
  Context& ctx = Ctx();
  SideStream& side = Side();
  const cudaStream_t main = ctx.stream;
  const cudaStream_t look = side.ok ? side.stream : main;
  // The context stream's persistent GEMMs leave kSideSms SMs free, so that
  // the side stream's panel runs beside them rather than after them.
  const int cap = side.ok ? std::max(1, ctx.num_sms - kSideSms) : 0;
  // The trailing work of panel j on columns [c0, c0 + nc).
  const auto update = [&](int j, int jb, int c0, int nc) {
    Laswp<T>(nc, At(a, lda, 0, c0), lda, j + 1, j + jb, ipiv, 1);
    TrsmFull<T>(true, true, false, true, jb, nc, T(1), At(a, lda, j, j), lda,
                At(a, lda, j, c0), lda);
    if (j + jb < m) {
      GemmFull<T>(false, false, m - j - jb, nc, jb, T(-1), At(a, lda, j + jb, j), lda,
                  At(a, lda, j, c0), lda, T(1), At(a, lda, j + jb, c0), lda);
    }
  };
  StreamAfter(side.to_side, main, look);
  OnSide([&] { GetrfRec<T>(m, std::min(nb, mn), a, lda, ipiv, info, 0); });
  for (int j = 0; j < mn; j += nb) {
    const int jb = std::min(mn - j, nb);
    const int right = n - j - jb;               // columns right of the panel
    const int next = std::min(nb, right);       // the next panel's columns
    const int jb2 = std::min(mn - j - jb, nb);  // the next panel's width
    StreamAfter(side.to_side, main, look);
    OnSide([&] { AdjustPivots(ipiv, j, std::min(m, j + jb), j); });
    StreamAfter(side.to_main, look, main);
    if (next > 0) {
      OnSide([&] {
        ctx.side_leaf = side.ok;
        update(j, jb, j + jb, next);
        if (jb2 > 0) GetrfRec<T>(m - j - jb, jb2, At(a, lda, j + jb, j + jb), lda,
                                 ipiv + j + jb, info, j + jb);
        ctx.side_leaf = false;
      });
    }
    Laswp<T>(j, a, lda, j + 1, j + jb, ipiv, 1);
    if (right > next) {
      ctx.sm_cap = cap;
      update(j, jb, j + jb + next, right - next);
      ctx.sm_cap = 0;
    }
  }
  StreamAfter(side.to_main, look, main);
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

// Blocked Cholesky (potrf.cc:160-197) with a look-ahead of one block. Step j
// updates and factors the diagonal block (SYRK, POTRF2), then updates and
// solves the block beside it (GEMM, TRSM). The GEMM and TRSM act on each row
// (lower; each column, upper) of that block independently, so they are split:
// on the side stream, the part that the next diagonal block reads (its jb
// rows) is done first and the next diagonal block is updated and factored;
// the context's stream does the rest. The side stream's step j waits for
// the context stream's step j - 1; the context stream's step j waits for
// the side stream's diagonal block j. Every element's operations are the
// reference's.
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
  SideStream& side = Side();
  const cudaStream_t main = ctx.stream;
  const cudaStream_t look = side.ok ? side.stream : main;
  const int cap = side.ok ? std::max(1, ctx.num_sms - kSideSms) : 0;
  // The split GEMMs' partial buffers at their largest, reserved before the
  // first launch (growing one in the loop would synchronize the device).
  size_t bytes_main = 0, bytes_side = 0;
  for (int j = nb; j < n; j += nb) {
    const int jb = std::min(nb, n - j), rest = n - j - jb, next = std::min(nb, rest);
    const auto split = [&](int rows) {
      return upper ? DgemmSplitBytes(jb, rows, j) : DgemmSplitBytes(rows, jb, j);
    };
    bytes_side = std::max(bytes_side, split(next));
    if (rest > next) bytes_main = std::max(bytes_main, split(rest - next));
  }
  if (sizeof(T) == 8) {
    if (bytes_main > 0) Workspace(kWsSplitK, bytes_main);
    if (bytes_side > 0) OnSide([&] { Workspace(kWsSplitK, bytes_side); });
  }
  // Diagonal block j: its update by the finished columns, then POTRF2.
  const auto diag = [&](int j, int jb) {
    if (upper) {
      SyrkFull<T>(false, true, jb, j, T(-1), At(a, lda, 0, j), lda, 1.0, At(a, lda, j, j),
                  lda);
      Potrf2Rec<T>(true, jb, At(a, lda, j, j), lda, info, j);
    } else {
      SyrkFull<T>(true, false, jb, j, T(-1), At(a, lda, j, 0), lda, 1.0, At(a, lda, j, j),
                  lda);
      Potrf2Rec<T>(false, jb, At(a, lda, j, j), lda, info, j);
    }
  };
  // Block j's off-diagonal part, restricted to rows (lower; columns, upper)
  // [r0, r0 + nr).
  const auto beside = [&](int j, int jb, int r0, int nr) {
    if (upper) {
      if (j > 0)
        GemmFull<T>(true, false, jb, nr, j, T(-1), At(a, lda, 0, j), lda, At(a, lda, 0, r0),
                    lda, 1.0, At(a, lda, j, r0), lda);
      TrsmFull<T>(true, false, true, false, jb, nr, 1.0, At(a, lda, j, j), lda,
                  At(a, lda, j, r0), lda);
    } else {
      if (j > 0)
        GemmFull<T>(false, true, nr, jb, j, -1.0, At(a, lda, r0, 0), lda, At(a, lda, j, 0),
                    lda, 1.0, At(a, lda, r0, j), lda);
      TrsmFull<T>(false, true, true, false, nr, jb, 1.0, At(a, lda, j, j), lda,
                  At(a, lda, r0, j), lda);
    }
  };
  StreamAfter(side.to_side, main, look);
  OnSide([&] { diag(0, nb); });
  for (int j = 0; j < n; j += nb) {
    const int jb = std::min(nb, n - j);
    const int rest = n - j - jb;
    if (rest <= 0) break;
    const int next = std::min(nb, rest);
    StreamAfter(side.to_side, main, look);
    StreamAfter(side.to_main, look, main);
    OnSide([&] {
      beside(j, jb, j + jb, next);
      diag(j + jb, next);
    });
    if (rest > next) {
      ctx.sm_cap = cap;
      beside(j, jb, j + jb + next, rest - next);
      ctx.sm_cap = 0;
    }
  }
  StreamAfter(side.to_main, look, main);
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
