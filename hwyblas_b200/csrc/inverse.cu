// Triangular inverse (xTRTI2, xTRTRI) and the inverse of a matrix from its
// LU factorization (xGETRI), in the reference's call order and rounding
// (src/lapack/triangular.cc:18-166; src/lapack/getrf.cc:369-483):
//
//   TRTI2   one column at a time: the diagonal becomes its exact reciprocal,
//           the finished part of the inverse multiplies the column (TRMV in
//           the reference kernel's order: strips of 4 columns, the strip's
//           diagonal block as a rounded product plus a rounded sum, the rest
//           as a chain of fmas in column order, src/trmv-inl.h:44-80), then
//           the column is scaled by -A(j, j). One CTA; the columns depend on
//           each other, so a block of 64 costs 64 short steps.
//   TRTRI   blocks of 64 (ILAENV): TRMM and TRSM of the block column (the
//           library's bit-exact level 3), TRTI2 of the diagonal block.
//   GETRI   inv(U) by TRTRI, then inv(A) L = inv(U) for one block column of
//           64 at a time from the right: the block column of L moves to a
//           workspace, GEMM subtracts the finished columns, TRSM with the
//           unit lower block finishes it (GEMV per column when unblocked);
//           finally the column interchanges are undone in reverse order.
#include <algorithm>
#include <climits>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

template <typename T>
__device__ __forceinline__ T MulRn(T x, T y) {
  if constexpr (sizeof(T) == 8) return __dmul_rn(x, y);
  else return __fmul_rn(x, y);
}
template <typename T>
__device__ __forceinline__ T AddRn(T x, T y) {
  if constexpr (sizeof(T) == 8) return __dadd_rn(x, y);
  else return __fadd_rn(x, y);
}
template <typename T>
__device__ __forceinline__ T Fma(T x, T y, T z) {
  if constexpr (sizeof(T) == 8) return fma(x, y, z);
  else return fmaf(x, y, z);
}

constexpr int kTrti2Threads = 256;

// TRTI2 of the n x n triangle of a (upper or lower, unit or not), in place.
// tmp (n elements) holds a column's new values between the block's reads of
// the old ones and its writes.
template <typename T>
__global__ void __launch_bounds__(kTrti2Threads)
    Trti2Kernel(int n, T* a, long long lda, int upper, int unit, T* tmp, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  const auto A = [&](int i, int j) -> T& { return a[i + j * lda]; };
  for (int step = 0; step < n; ++step) {
    const int j = upper ? step : n - 1 - step;
    T ajj = T(-1), dinv = T(0);
    if (!unit) {
      dinv = T(1) / A(j, j);
      ajj = -dinv;
    }
    if (upper) {
      // x = A(0:j, j) := inv(U)(0:j, 0:j) x, rows i < j.
      for (int i = threadIdx.x; i < j; i += blockDim.x) {
        const int send = min((i & ~3) + 4, j);
        T y = T(0);
        for (int jj = i; jj < send; ++jj) {
          const T v = (jj == i && unit) ? T(1) : A(i, jj);
          y = AddRn(y, MulRn(v, A(jj, j)));
        }
        for (int c = send; c < j; ++c) y = Fma(A(i, c), A(c, j), y);
        tmp[i] = MulRn(y, ajj);
      }
    } else {
      // x = A(j+1:n, j) := inv(L)(j+1:n, j+1:n) x, local row li = i - r0.
      const int r0 = j + 1;
      for (int i = r0 + threadIdx.x; i < n; i += blockDim.x) {
        const int li = i - r0, s0 = li & ~3;
        T y = T(0);
        for (int lc = 0; lc < s0; ++lc) y = Fma(A(i, r0 + lc), A(r0 + lc, j), y);
        for (int lc = s0; lc <= li; ++lc) {
          const T v = (lc == li && unit) ? T(1) : A(i, r0 + lc);
          y = AddRn(y, MulRn(v, A(r0 + lc, j)));
        }
        tmp[i] = MulRn(y, ajj);
      }
    }
    __syncthreads();
    if (upper) {
      for (int i = threadIdx.x; i < j; i += blockDim.x) A(i, j) = tmp[i];
    } else {
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A(i, j) = tmp[i];
    }
    if (threadIdx.x == 0 && !unit) A(j, j) = dinv;
    __syncthreads();
  }
}

// TRTI2 of the diagonal blocks of order nb (the last one n - (nblk-1) nb) of
// an n x n triangle, one CTA per block, the block in shared memory; each
// block's arithmetic is Trti2Kernel's. orig receives the blocks as they were
// (leading dimension nb), for the TRSMs that divide by them.
template <typename T>
__global__ void __launch_bounds__(64)
    Trti2BlocksKernel(int n, int nb, T* a, long long lda, int upper, int unit, T* orig,
                      const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ T s[64][65];
  const int j0 = blockIdx.x * nb, jb = min(nb, n - j0), t = threadIdx.x;
  T* blk = a + j0 + static_cast<long long>(j0) * lda;
  T* saved = orig + static_cast<long long>(blockIdx.x) * nb * nb;
  for (int j = 0; j < jb; ++j) {
    if (t < jb) {
      const T v = blk[t + j * lda];
      s[t][j] = v;
      saved[t + j * nb] = v;
    }
  }
  __syncthreads();
  for (int step = 0; step < jb; ++step) {
    const int j = upper ? step : jb - 1 - step;
    T ajj = T(-1), dinv = T(0);
    if (!unit) {
      dinv = T(1) / s[j][j];
      ajj = -dinv;
    }
    T y = T(0);
    bool mine = false;
    if (upper && t < j) {
      mine = true;
      const int send = min((t & ~3) + 4, j);
      for (int jj = t; jj < send; ++jj) {
        const T v = (jj == t && unit) ? T(1) : s[t][jj];
        y = AddRn(y, MulRn(v, s[jj][j]));
      }
      for (int c = send; c < j; ++c) y = Fma(s[t][c], s[c][j], y);
      y = MulRn(y, ajj);
    } else if (!upper && t > j && t < jb) {
      mine = true;
      const int r0 = j + 1, li = t - r0, s0 = li & ~3;
      for (int lc = 0; lc < s0; ++lc) y = Fma(s[t][r0 + lc], s[r0 + lc][j], y);
      for (int lc = s0; lc <= li; ++lc) {
        const T v = (lc == li && unit) ? T(1) : s[t][r0 + lc];
        y = AddRn(y, MulRn(v, s[r0 + lc][j]));
      }
      y = MulRn(y, ajj);
    }
    __syncthreads();
    if (mine) s[t][j] = y;
    if (t == j && !unit) s[j][j] = dinv;
    __syncthreads();
  }
  if (t < jb) {
    for (int j = 0; j < jb; ++j) {
      const bool tri = upper ? t <= j : t >= j;
      if (tri) blk[t + j * lda] = s[t][j];
    }
  }
}

// dense(i, j) := the triangle value of A(i, j) (zero outside it, one on a
// unit diagonal) for i in [r0, r1), j in [c0, c1).
template <typename T>
__global__ void DenseTriangleKernel(int r0, int r1, int c0, int c1, const T* a, long long lda,
                                    int upper, int unit, T* dense, long long ldd) {
  const int rows = r1 - r0;
  const long long total = static_cast<long long>(rows) * (c1 - c0);
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = r0 + static_cast<int>(e % rows), j = c0 + static_cast<int>(e / rows);
    T v = T(0);
    if (i == j) v = unit ? T(1) : a[i + j * lda];
    else if (upper ? i < j : i > j) v = a[i + j * lda];
    dense[i + j * ldd] = v;
  }
}

// *out = 1 + the first i with A(i, i) == 0, or 0.
template <typename T>
__global__ void FirstZeroDiagKernel(int n, const T* a, long long lda, int* out) {
  __shared__ int best;
  if (threadIdx.x == 0) best = INT_MAX;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (a[i + i * lda] == T(0)) {
      atomicMin(&best, i);
      break;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *out = (best == INT_MAX) ? 0 : best + 1;
}

// work(i, jj - j) := A(i, jj) and A(i, jj) := 0 below the diagonal of the
// block column [j, j + jb).
template <typename T>
__global__ void GetriCopyKernel(int n, int j, T* a, long long lda, T* work, long long ldw) {
  const int jj = j + blockIdx.y;
  for (int i = jj + 1 + blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    work[i + static_cast<long long>(blockIdx.y) * ldw] = a[i + jj * lda];
    a[i + jj * lda] = T(0);
  }
}

// Column j of inv(A) without blocks: A(:, j) += A(:, j+1:n) * (-work(j+1:n)),
// the GEMV chain (t = -1 * work, one fma per column in order).
template <typename T>
__global__ void GetriGemvKernel(int n, int j, T* a, long long lda, const T* work) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T y = a[i + j * lda];
  for (int c = j + 1; c < n; ++c) y = Fma(a[i + c * lda], -work[c], y);
  a[i + j * lda] = y;
}

// The same for all columns in one CTA (n small).
template <typename T>
__global__ void __launch_bounds__(1024)
    GetriUnblockedKernel(int n, T* a, long long lda, T* work, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  for (int j = n - 1; j >= 0; --j) {
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      work[i] = a[i + j * lda];
      a[i + j * lda] = T(0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      T y = a[i + j * lda];
      for (int c = j + 1; c < n; ++c) y = Fma(a[i + c * lda], -work[c], y);
      a[i + j * lda] = y;
    }
    __syncthreads();
  }
}

// Column interchanges j <-> ipiv(j) for j = n-2 down to 0; each row's swaps
// are independent of the other rows'.
template <typename T>
__global__ void ColumnSwapKernel(int n, T* a, long long lda, const int* ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = n - 2; j >= 0; --j) {
    const int jp = ipiv[j] - 1;
    if (jp != j) {
      const T t = a[i + j * lda];
      a[i + j * lda] = a[i + jp * lda];
      a[i + jp * lda] = t;
    }
  }
}

template <typename T>
bool Trti2(bool upper, bool unit, int n, T* a, int lda) {
  if (n <= 0) return true;
  T* tmp = static_cast<T*>(Workspace(kWsTrti2, sizeof(T) * static_cast<size_t>(n)));
  if (tmp == nullptr) return false;
  Trti2Kernel<T><<<1, kTrti2Threads, 0, Ctx().stream>>>(n, a, lda, upper ? 1 : 0, unit ? 1 : 0,
                                                         tmp, Ctx().guard);
  CountLaunch();
  return !LaunchFailed("trti2");
}

}  // namespace

template <typename T>
int Trti2Full(bool upper, bool unit, int n, T* a, int lda) {
  Trti2<T>(upper, unit, n, a, lda);
  return 0;
}
template int Trti2Full<double>(bool, bool, int, double*, int);
template int Trti2Full<float>(bool, bool, int, float*, int);

// xTRTRI after argument checks: INFO > 0 (A untouched) for an exactly zero
// diagonal element when not unit.
template <typename T>
int TrtriFull(bool upper, bool unit, int n, T* a, int lda) {
  if (n == 0) return 0;
  if (!unit) {
    int* out = Ctx().dev_status + 5;
    FirstZeroDiagKernel<T><<<1, 1024, 0, Ctx().stream>>>(n, a, lda, out);
    CountLaunch();
    if (LaunchFailed("trtri diagonal")) return 0;
    int h = 0;
    if (Failed(cudaMemcpyAsync(&h, out, sizeof(int), cudaMemcpyDeviceToHost, Ctx().stream),
               "trtri info") ||
        Failed(cudaStreamSynchronize(Ctx().stream), "trtri sync"))
      return 0;
    if (h > 0) return h;
  }
  constexpr int nb = 64;  // ILAENV(1, xTRTRI) (src/lapack/environment.cc:134-137)
  if (nb >= n) {
    Trti2<T>(upper, unit, n, a, lda);
    return 0;
  }
  // Every diagonal block's TRTI2 reads only that block, and the reference
  // inverts block j right after the TRMM and TRSM of its block column, which
  // write other entries and divide by the block as it was. So all blocks are
  // inverted at once up front (one CTA each), their original values kept for
  // those TRSMs; every value is the same as in the reference's order.
  const int nblk = (n + nb - 1) / nb;
  T* orig = static_cast<T*>(
      Workspace(kWsTrti2, sizeof(T) * static_cast<size_t>(nblk) * nb * nb));
  if (orig == nullptr) return 0;
  Trti2BlocksKernel<T><<<nblk, 64, 0, Ctx().stream>>>(n, nb, a, lda, upper ? 1 : 0,
                                                       unit ? 1 : 0, orig, Ctx().guard);
  CountLaunch();
  if (LaunchFailed("trti2 blocks")) return 0;
  const auto A = [&](int i, int j) { return a + i + static_cast<long long>(j) * lda; };
  const auto D = [&](int j) { return orig + static_cast<long long>(j / nb) * nb * nb; };
  // The finished part of the inverse, kept dense for the TRMMs (each TRMM
  // multiplies by it with the zeros and ones written out): one block column
  // is added per step instead of rewriting the whole triangle. Workspaces
  // are sized once, so that no step reallocates.
  const long long ldd = (n + 1) / 2 * 2;
  T* dense = static_cast<T*>(Workspace(kWsLevel3, sizeof(T) * static_cast<size_t>(ldd) * n));
  if (dense == nullptr ||
      Workspace(kWsLevel3Copy, sizeof(T) * static_cast<size_t>(n) * nb) == nullptr)
    return 0;
  Failed(cudaMemsetAsync(dense, 0, sizeof(T) * static_cast<size_t>(ldd) * n, Ctx().stream),
         "trtri dense");
  const auto add_columns = [&](int r0, int r1, int c0, int c1) {
    const long long total = static_cast<long long>(r1 - r0) * (c1 - c0);
    if (total <= 0) return;
    const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
    DenseTriangleKernel<T><<<blocks, 256, 0, Ctx().stream>>>(r0, r1, c0, c1, a, lda,
                                                              upper ? 1 : 0, unit ? 1 : 0,
                                                              dense, ldd);
    CountLaunch();
  };
  if (upper) {
    add_columns(0, std::min(nb, n), 0, std::min(nb, n));
    for (int j = nb; j < n; j += nb) {
      const int jb = std::min(nb, n - j);
      TrmmDense<T>(true, false, false, j, jb, T(1), dense, static_cast<int>(ldd), A(0, j), lda);
      TrsmFull<T>(false, false, false, unit, j, jb, T(-1), D(j), nb, A(0, j), lda);
      add_columns(0, j + jb, j, j + jb);
    }
  } else {
    const int nn = ((n - 1) / nb) * nb;
    add_columns(nn, n, nn, n);
    for (int j = nn - nb; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      const int m = n - j - jb;
      const T* tri = dense + (j + jb) + (j + jb) * ldd;
      TrmmDense<T>(true, true, false, m, jb, T(1), tri, static_cast<int>(ldd), A(j + jb, j),
                   lda);
      TrsmFull<T>(false, true, false, unit, m, jb, T(-1), D(j), nb, A(j + jb, j), lda);
      add_columns(j, n, j, j + jb);
    }
  }
  return 0;
}
template int TrtriFull<double>(bool, bool, int, double*, int);
template int TrtriFull<float>(bool, bool, int, float*, int);

// xGETRI after argument checks (n > 0, lwork >= n). *iws: the workspace size
// the reference reports in WORK(1) on success.
template <typename T>
int GetriFull(int n, T* a, int lda, const int* ipiv, int lwork, int* iws_out) {
  const int info = TrtriFull<T>(true, false, n, a, lda);
  if (info > 0) return info;

  int nb = 64;  // ILAENV(1, xGETRI) (src/lapack/environment.cc:105-106)
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
  *iws_out = iws;
  cudaStream_t st = Ctx().stream;
  const auto A = [&](int i, int j) { return a + i + static_cast<long long>(j) * lda; };
  if (nb < nbmin || nb >= n) {
    T* w = static_cast<T*>(Workspace(kWsGetri, sizeof(T) * static_cast<size_t>(n)));
    if (w == nullptr) return 0;
    if (n <= 1024) {
      GetriUnblockedKernel<T><<<1, 1024, 0, st>>>(n, a, lda, w, Ctx().guard);
      CountLaunch();
      LaunchFailed("getri unblocked");
    } else {
      for (int j = n - 1; j >= 0; --j) {
        GetriCopyKernel<T><<<dim3((n + 255) / 256, 1), 256, 0, st>>>(n, j, a, lda, w, n);
        CountLaunch();
        if (j < n - 1) {
          GetriGemvKernel<T><<<(n + 255) / 256, 256, 0, st>>>(n, j, a, lda, w);
          CountLaunch();
        }
        if (LaunchFailed("getri column")) return 0;
      }
    }
  } else {
    // The block columns of L, leading dimension rounded up to even so that
    // the GEMM reads them in place.
    const int ldw = (ldwork + 1) / 2 * 2;
    const size_t welems = static_cast<size_t>(ldw) * nb;
    T* w = static_cast<T*>(Workspace(kWsGetri, sizeof(T) * welems));
    if (w == nullptr) return 0;
    // Entries on and above the diagonal of a block are never read; zeroed
    // so that the buffer holds no stale values at all.
    Failed(cudaMemsetAsync(w, 0, sizeof(T) * welems, st), "getri work");
    const int nn = ((n - 1) / nb) * nb;
    for (int j = nn; j >= 0; j -= nb) {
      const int jb = std::min(nb, n - j);
      GetriCopyKernel<T><<<dim3((n + 255) / 256, jb), 256, 0, st>>>(n, j, a, lda, w, ldw);
      CountLaunch();
      if (LaunchFailed("getri copy")) return 0;
      if (j + jb < n) {
        GemmFull<T>(false, false, n, jb, n - j - jb, T(-1), A(0, j + jb), lda, w + j + jb, ldw,
                    T(1), A(0, j), lda);
      }
      TrsmFull<T>(false, true, false, true, n, jb, T(1), w + j, ldw, A(0, j), lda);
    }
  }
  if (n > 1) {
    ColumnSwapKernel<T><<<(n + 255) / 256, 256, 0, st>>>(n, a, lda, ipiv);
    CountLaunch();
    LaunchFailed("getri column swaps");
  }
  return 0;
}
template int GetriFull<double>(int, double*, int, const int*, int, int*);
template int GetriFull<float>(int, float*, int, const int*, int, int*);

}  // namespace hb
