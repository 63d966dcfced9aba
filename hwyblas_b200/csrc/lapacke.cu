// LAPACKE C interface of the LU and Cholesky drivers (the reference's
// src/lapack/lapacke.cc:37-137, lapacke_linear.cc:22-73,
// lapacke_symmetric.cc:22-72, on the CallWork scheme of
// lapacke_util.h:418-500):
//
//   LAPACKE_xyyzzz       layout check (LAPACKE_xerbla(name, -1)), then,
//                        unless switched off, a NaN check of the inputs
//                        (returns -i for the i-th argument, no message),
//                        then the _work function;
//   LAPACKE_xyyzzz_work  column-major: the LAPACK routine on the caller's
//                        arrays, INFO < 0 shifted by one (the layout
//                        argument); row-major: each leading dimension must
//                        cover the columns (else LAPACKE_xerbla and -i), the
//                        matrices are transposed into column-major
//                        temporaries, the routine runs on them, and the
//                        outputs are transposed back.
//
// The LAPACK routines are this library's dgetrf_ etc., so the results are
// the column-major ones on the transposed data, bit for bit. Temporaries
// live where the caller's matrix lives: host vectors for host arrays (as the
// reference's malloc), device workspace and a tiled transpose kernel for
// device arrays. A failed temporary allocation gives
// LAPACK_TRANSPOSE_MEMORY_ERROR, as in the reference.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <string>
#include <vector>

#include "../../include/hwyblas_b200.h"
#include "internal.h"

namespace hb {
namespace {

// -1: not yet determined (LAPACKE_get_nancheck reads LAPACKE_NANCHECK once).
std::atomic<int> g_nancheck{-1};

bool IsDevice(const void* p) {
  if (p == nullptr) return false;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

template <typename T>
std::string Name(const char* rest) {
  return std::string("LAPACKE_") + (sizeof(T) == 8 ? "d" : "s") + rest;
}

// out(r, c) = in(c, r): both column-major, out rows x cols. 32 x 32 tiles
// through shared memory, so that both sides are read and written along
// their contiguous dimension.
template <typename T>
__global__ void TransposeKernel(int rows, int cols, const T* in, long long ld_in, T* out,
                                long long ld_out) {
  __shared__ T tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[c + r * ld_in];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[r + c * ld_out] = tile[threadIdx.x][k];
  }
}

template <typename T>
void Transpose(int rows, int cols, const T* in, long long ld_in, T* out, long long ld_out) {
  if (rows <= 0 || cols <= 0) return;
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
  TransposeKernel<T><<<grid, dim3(32, 8), 0, Ctx().stream>>>(rows, cols, in, ld_in, out,
                                                               ld_out);
  CountLaunch();
  LaunchFailed("lapacke transpose");
}

// Whether the logical rows x cols matrix (row-major: a[i*ld + j]) has a NaN
// in part 'G' (all), 'U' (i <= j), 'L' (i >= j), 'u' (i < j) or 'l' (i > j).
template <typename T>
__global__ void NanKernel(int rows, int cols, const T* a, long long ld, int rowmajor, char part,
                          int* flag) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = rowmajor ? static_cast<int>(e / cols) : static_cast<int>(e % rows);
    const int j = rowmajor ? static_cast<int>(e % cols) : static_cast<int>(e / rows);
    if ((part == 'U' && i > j) || (part == 'L' && i < j)) continue;
    if ((part == 'u' && i >= j) || (part == 'l' && i <= j)) continue;
    const T x = rowmajor ? a[static_cast<long long>(i) * ld + j] : a[i + j * ld];
    if (x != x) atomicExch(flag, 1);
  }
}

// LAPACKE_xge_nancheck / xtr_nancheck (lapacke_util.h:60-180): like the
// reference, at most ld rows (columns for row-major) are looked at.
template <typename T>
bool HasNan(int layout, char part, int m, int n, const T* a, int lda) {
  if (a == nullptr || m <= 0 || n <= 0) return false;
  const bool rowmajor = layout == LAPACK_ROW_MAJOR;
  if (rowmajor) n = std::min(n, lda);
  else m = std::min(m, lda);
  if (m <= 0 || n <= 0) return false;
  if (!IsDevice(a)) {
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < m; ++i) {
        if ((part == 'U' && i > j) || (part == 'L' && i < j)) continue;
        if ((part == 'u' && i >= j) || (part == 'l' && i <= j)) continue;
        const T x = rowmajor ? a[static_cast<size_t>(i) * lda + j]
                             : a[i + static_cast<size_t>(j) * lda];
        if (std::isnan(x)) return true;
      }
    }
    return false;
  }
  int* flag = static_cast<int*>(Workspace(kWsLapacke1, 256));
  if (flag == nullptr) return false;
  cudaStream_t st = Ctx().stream;
  cudaMemsetAsync(flag, 0, sizeof(int), st);
  const long long total = static_cast<long long>(m) * n;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
  NanKernel<T><<<blocks, 256, 0, st>>>(m, n, a, lda, rowmajor ? 1 : 0, part, flag);
  CountLaunch();
  int h = 0;
  cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (Failed(cudaStreamSynchronize(st), "lapacke nancheck")) return false;
  return h != 0;
}

// NaN-check part of a triangle argument; invalid uplo checks nothing.
char TrPart(char uplo) {
  const char u = (uplo >= 'a' && uplo <= 'z') ? static_cast<char>(uplo - 32) : uplo;
  return (u == 'U' || u == 'L') ? u : 0;
}

// LAPACKE_xtr_nancheck (lapacke_util.h:89-119): the triangle, without the
// diagonal when unit; invalid uplo or diag checks nothing.
template <typename T>
bool HasNanTr(int layout, char uplo, char diag, int n, const T* a, int lda) {
  const char part = TrPart(uplo);
  const char d = (diag >= 'a' && diag <= 'z') ? static_cast<char>(diag - 32) : diag;
  if (part == 0 || (d != 'U' && d != 'N')) return false;
  return HasNan(layout, d == 'U' ? static_cast<char>(part + 32) : part, n, n, a, lda);
}

template <typename T>
bool HasNanPo(int layout, char uplo, int n, const T* a, int lda) {
  const char part = TrPart(uplo);
  return part != 0 && HasNan(layout, part, n, n, a, lda);
}

// One matrix argument of a _work function: rows x cols with leading
// dimension ld; ld_info is -i for the ld argument's position.
template <typename T>
struct Arg {
  T* data;
  int rows, cols, ld, ld_info;
  bool in, out;
};

// A column-major temporary of a row-major argument.
template <typename T>
struct Temp {
  std::vector<T> host;
  T* ptr = nullptr;
  int ld = 1;
  bool dev = false;
  bool Make(const Arg<T>& a, int slot) {
    ld = std::max(1, a.rows);
    const size_t elems = static_cast<size_t>(ld) * std::max(1, a.cols);
    dev = IsDevice(a.data);
    if (dev) {
      ptr = static_cast<T*>(Workspace(slot, sizeof(T) * elems));
      return ptr != nullptr;
    }
    try {
      host.resize(elems);
    } catch (const std::bad_alloc&) {
      return false;
    }
    ptr = host.data();
    return true;
  }
  // temp(i, j) = a[i * a.ld + j]
  void In(const Arg<T>& a) {
    if (a.rows <= 0 || a.cols <= 0) return;
    if (dev) {
      Transpose<T>(a.rows, a.cols, a.data, a.ld, ptr, ld);
      return;
    }
    for (int i = 0; i < a.rows; ++i)
      for (int j = 0; j < a.cols; ++j)
        ptr[i + static_cast<size_t>(j) * ld] = a.data[static_cast<size_t>(i) * a.ld + j];
  }
  void Out(const Arg<T>& a) {
    if (a.rows <= 0 || a.cols <= 0) return;
    if (dev) {
      Transpose<T>(a.cols, a.rows, ptr, ld, a.data, a.ld);
      Failed(cudaStreamSynchronize(Ctx().stream), "lapacke transpose");
      return;
    }
    for (int i = 0; i < a.rows; ++i)
      for (int j = 0; j < a.cols; ++j)
        a.data[static_cast<size_t>(i) * a.ld + j] = ptr[i + static_cast<size_t>(j) * ld];
  }
};

// CallWork (lapacke_util.h:418-480): call(p, ld) runs the LAPACK routine on
// column-major arrays p[i] with leading dimensions ld[i].
template <typename T, int N, typename F>
lapack_int CallWork(int layout, const std::string& name, const Arg<T> (&args)[N], F call) {
  T* p[N];
  int ld[N];
  if (layout == LAPACK_COL_MAJOR) {
    for (int i = 0; i < N; ++i) {
      p[i] = args[i].data;
      ld[i] = args[i].ld;
    }
    const int info = call(p, ld);
    return info < 0 ? info - 1 : info;
  }
  if (layout != LAPACK_ROW_MAJOR) {
    LAPACKE_xerbla(name.c_str(), -1);
    return -1;
  }
  for (int i = 0; i < N; ++i) {
    if (args[i].ld < args[i].cols) {
      LAPACKE_xerbla(name.c_str(), args[i].ld_info);
      return args[i].ld_info;
    }
  }
  Temp<T> tmp[N];
  for (int i = 0; i < N; ++i) {
    if (!tmp[i].Make(args[i], i == 0 ? kWsLapacke0 : kWsLapacke1)) {
      LAPACKE_xerbla(name.c_str(), LAPACK_TRANSPOSE_MEMORY_ERROR);
      return LAPACK_TRANSPOSE_MEMORY_ERROR;
    }
    p[i] = tmp[i].ptr;
    ld[i] = tmp[i].ld;
  }
  for (int i = 0; i < N; ++i)
    if (args[i].in) tmp[i].In(args[i]);
  int info = call(p, ld);
  if (info < 0) info -= 1;
  for (int i = 0; i < N; ++i)
    if (args[i].out) tmp[i].Out(args[i]);
  return info;
}

// The LAPACK routines by type.
void Getrf(bool rec, int* m, int* n, double* a, int* lda, int* ipiv, int* info) {
  (rec ? dgetrf2_ : dgetrf_)(m, n, a, lda, ipiv, info);
}
void Getrf(bool rec, int* m, int* n, float* a, int* lda, int* ipiv, int* info) {
  (rec ? sgetrf2_ : sgetrf_)(m, n, a, lda, ipiv, info);
}
void Getrs(const char* t, int* n, int* r, const double* a, int* lda, const int* ipiv, double* b,
           int* ldb, int* info) {
  dgetrs_(t, n, r, a, lda, ipiv, b, ldb, info);
}
void Getrs(const char* t, int* n, int* r, const float* a, int* lda, const int* ipiv, float* b,
           int* ldb, int* info) {
  sgetrs_(t, n, r, a, lda, ipiv, b, ldb, info);
}
void Gesv(int* n, int* r, double* a, int* lda, int* ipiv, double* b, int* ldb, int* info) {
  dgesv_(n, r, a, lda, ipiv, b, ldb, info);
}
void Gesv(int* n, int* r, float* a, int* lda, int* ipiv, float* b, int* ldb, int* info) {
  sgesv_(n, r, a, lda, ipiv, b, ldb, info);
}
void Potrf(bool rec, const char* u, int* n, double* a, int* lda, int* info) {
  (rec ? dpotrf2_ : dpotrf_)(u, n, a, lda, info);
}
void Potrf(bool rec, const char* u, int* n, float* a, int* lda, int* info) {
  (rec ? spotrf2_ : spotrf_)(u, n, a, lda, info);
}
void Potrs(const char* u, int* n, int* r, const double* a, int* lda, double* b, int* ldb,
           int* info) {
  dpotrs_(u, n, r, a, lda, b, ldb, info);
}
void Potrs(const char* u, int* n, int* r, const float* a, int* lda, float* b, int* ldb,
           int* info) {
  spotrs_(u, n, r, a, lda, b, ldb, info);
}
void Getri(int* n, double* a, int* lda, const int* ipiv, double* w, int* lw, int* info) {
  dgetri_(n, a, lda, ipiv, w, lw, info);
}
void Getri(int* n, float* a, int* lda, const int* ipiv, float* w, int* lw, int* info) {
  sgetri_(n, a, lda, ipiv, w, lw, info);
}
void Trtri(const char* u, const char* d, int* n, double* a, int* lda, int* info) {
  dtrtri_(u, d, n, a, lda, info);
}
void Trtri(const char* u, const char* d, int* n, float* a, int* lda, int* info) {
  strtri_(u, d, n, a, lda, info);
}
void Posv(const char* u, int* n, int* r, double* a, int* lda, double* b, int* ldb, int* info) {
  dposv_(u, n, r, a, lda, b, ldb, info);
}
void Posv(const char* u, int* n, int* r, float* a, int* lda, float* b, int* ldb, int* info) {
  sposv_(u, n, r, a, lda, b, ldb, info);
}

}  // namespace
}  // namespace hb

namespace hb {
namespace {

bool NanCheck() { return LAPACKE_get_nancheck() != 0; }

template <typename T>
lapack_int GetrfWork(int layout, int m, int n, T* a, int lda, int* ipiv, bool rec) {
  const Arg<T> args[1] = {{a, m, n, lda, -5, true, true}};
  return CallWork(layout, Name<T>(rec ? "getrf2_work" : "getrf_work"), args,
                  [&](T** p, int* ld) {
                    int info = 0;
                    Getrf(rec, &m, &n, p[0], &ld[0], ipiv, &info);
                    return info;
                  });
}

template <typename T>
lapack_int GetrfMain(int layout, int m, int n, T* a, int lda, int* ipiv, bool rec) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>(rec ? "getrf2" : "getrf").c_str(), -1);
    return -1;
  }
  if (NanCheck() && HasNan(layout, 'G', m, n, a, lda)) return -4;
  return GetrfWork(layout, m, n, a, lda, ipiv, rec);
}

template <typename T>
lapack_int GetrsWork(int layout, char trans, int n, int nrhs, const T* a, int lda,
                     const int* ipiv, T* b, int ldb) {
  const Arg<T> args[2] = {{const_cast<T*>(a), n, n, lda, -6, true, false},
                          {b, n, nrhs, ldb, -9, true, true}};
  return CallWork(layout, Name<T>("getrs_work"), args, [&](T** p, int* ld) {
    int info = 0;
    Getrs(&trans, &n, &nrhs, p[0], &ld[0], ipiv, p[1], &ld[1], &info);
    return info;
  });
}

template <typename T>
lapack_int GetrsMain(int layout, char trans, int n, int nrhs, const T* a, int lda,
                     const int* ipiv, T* b, int ldb) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>("getrs").c_str(), -1);
    return -1;
  }
  if (NanCheck()) {
    if (HasNan(layout, 'G', n, n, a, lda)) return -5;
    if (HasNan(layout, 'G', n, nrhs, b, ldb)) return -8;
  }
  return GetrsWork(layout, trans, n, nrhs, a, lda, ipiv, b, ldb);
}

template <typename T>
lapack_int GesvWork(int layout, int n, int nrhs, T* a, int lda, int* ipiv, T* b, int ldb) {
  const Arg<T> args[2] = {{a, n, n, lda, -5, true, true}, {b, n, nrhs, ldb, -8, true, true}};
  return CallWork(layout, Name<T>("gesv_work"), args, [&](T** p, int* ld) {
    int info = 0;
    Gesv(&n, &nrhs, p[0], &ld[0], ipiv, p[1], &ld[1], &info);
    return info;
  });
}

template <typename T>
lapack_int GesvMain(int layout, int n, int nrhs, T* a, int lda, int* ipiv, T* b, int ldb) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>("gesv").c_str(), -1);
    return -1;
  }
  if (NanCheck()) {
    if (HasNan(layout, 'G', n, n, a, lda)) return -4;
    if (HasNan(layout, 'G', n, nrhs, b, ldb)) return -7;
  }
  return GesvWork(layout, n, nrhs, a, lda, ipiv, b, ldb);
}

template <typename T>
lapack_int PotrfWork(int layout, char uplo, int n, T* a, int lda, bool rec) {
  const Arg<T> args[1] = {{a, n, n, lda, -5, true, true}};
  return CallWork(layout, Name<T>(rec ? "potrf2_work" : "potrf_work"), args,
                  [&](T** p, int* ld) {
                    int info = 0;
                    Potrf(rec, &uplo, &n, p[0], &ld[0], &info);
                    return info;
                  });
}

template <typename T>
lapack_int PotrfMain(int layout, char uplo, int n, T* a, int lda, bool rec) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>(rec ? "potrf2" : "potrf").c_str(), -1);
    return -1;
  }
  if (NanCheck() && HasNanPo(layout, uplo, n, a, lda)) return -4;
  return PotrfWork(layout, uplo, n, a, lda, rec);
}

// xPOTRS reads A (a triangle) and updates B; xPOSV updates both.
template <typename T>
lapack_int PosWork(int layout, char uplo, int n, int nrhs, T* a, int lda, T* b, int ldb,
                   bool solve_only) {
  const Arg<T> args[2] = {{a, n, n, lda, -6, true, !solve_only},
                          {b, n, nrhs, ldb, -8, true, true}};
  return CallWork(layout, Name<T>(solve_only ? "potrs_work" : "posv_work"), args,
                  [&](T** p, int* ld) {
                    int info = 0;
                    if (solve_only)
                      Potrs(&uplo, &n, &nrhs, p[0], &ld[0], p[1], &ld[1], &info);
                    else
                      Posv(&uplo, &n, &nrhs, p[0], &ld[0], p[1], &ld[1], &info);
                    return info;
                  });
}

template <typename T>
lapack_int PosMain(int layout, char uplo, int n, int nrhs, T* a, int lda, T* b, int ldb,
                   bool solve_only) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>(solve_only ? "potrs" : "posv").c_str(), -1);
    return -1;
  }
  if (NanCheck()) {
    if (HasNanPo(layout, uplo, n, a, lda)) return -5;
    if (HasNan(layout, 'G', n, nrhs, b, ldb)) return -7;
  }
  return PosWork(layout, uplo, n, nrhs, a, lda, b, ldb, solve_only);
}

// xGETRI (lapacke_linear.cc:75-96): a workspace query (lwork = -1) runs on
// the caller's array after the leading-dimension check, as CallWork's query
// branch (lapacke_util.h:437-452).
template <typename T>
lapack_int GetriWork(int layout, int n, T* a, int lda, const int* ipiv, T* work, int lwork) {
  const std::string name = Name<T>("getri_work");
  const auto call = [&](T** p, int* ld) {
    int info = 0;
    Getri(&n, p[0], &ld[0], ipiv, work, &lwork, &info);
    return info;
  };
  if (lwork == -1 && layout == LAPACK_ROW_MAJOR) {
    if (lda < n) {
      LAPACKE_xerbla(name.c_str(), -4);
      return -4;
    }
    T* p[1] = {a};
    int ld[1] = {std::max(1, n)};
    const int info = call(p, ld);
    return info < 0 ? info - 1 : info;
  }
  const Arg<T> args[1] = {{a, n, n, lda, -4, true, true}};
  return CallWork(layout, name, args, call);
}

// WithWorkspace (lapacke_util.h:494-512): query, allocate, call.
template <typename T>
lapack_int GetriMain(int layout, int n, T* a, int lda, const int* ipiv) {
  const std::string name = Name<T>("getri");
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(name.c_str(), -1);
    return -1;
  }
  if (NanCheck() && HasNan(layout, 'G', n, n, a, lda)) return -3;
  T query = T(0);
  lapack_int info = GetriWork(layout, n, a, lda, ipiv, &query, -1);
  if (info != 0) return info;
  const int lwork = static_cast<int>(query);
  std::vector<T> buffer;
  try {
    buffer.resize(static_cast<size_t>(std::max(lwork, 1)));
  } catch (const std::bad_alloc&) {
    LAPACKE_xerbla(name.c_str(), LAPACK_WORK_MEMORY_ERROR);
    return LAPACK_WORK_MEMORY_ERROR;
  }
  return GetriWork(layout, n, a, lda, ipiv, buffer.data(), lwork);
}

// xTRTRI (lapacke_linear.cc:276-298).
template <typename T>
lapack_int TrtriWork(int layout, char uplo, char diag, int n, T* a, int lda) {
  const Arg<T> args[1] = {{a, n, n, lda, -6, true, true}};
  return CallWork(layout, Name<T>("trtri_work"), args, [&](T** p, int* ld) {
    int info = 0;
    Trtri(&uplo, &diag, &n, p[0], &ld[0], &info);
    return info;
  });
}

template <typename T>
lapack_int TrtriMain(int layout, char uplo, char diag, int n, T* a, int lda) {
  if (layout != LAPACK_ROW_MAJOR && layout != LAPACK_COL_MAJOR) {
    LAPACKE_xerbla(Name<T>("trtri").c_str(), -1);
    return -1;
  }
  if (NanCheck() && HasNanTr(layout, uplo, diag, n, a, lda)) return -5;
  return TrtriWork(layout, uplo, diag, n, a, lda);
}

}  // namespace
}  // namespace hb

extern "C" {

HWYBLAS_API void LAPACKE_xerbla(const char* name, lapack_int info) {
  if (info == LAPACK_WORK_MEMORY_ERROR) {
    printf("Not enough memory to allocate work array in %s\n", name);
  } else if (info == LAPACK_TRANSPOSE_MEMORY_ERROR) {
    printf("Not enough memory to transpose matrix in %s\n", name);
  } else if (info < 0) {
    printf("Wrong parameter %d in %s\n", -static_cast<int>(info), name);
  }
  fflush(stdout);
}

HWYBLAS_API void LAPACKE_set_nancheck(int flag) { hb::g_nancheck.store(flag ? 1 : 0); }

HWYBLAS_API int LAPACKE_get_nancheck(void) {
  const int flag = hb::g_nancheck.load();
  if (flag != -1) return flag;
  // The environment variable, read once; NaN checks are on by default.
  const char* env = getenv("LAPACKE_NANCHECK");
  const int value = (env == nullptr || atoi(env) != 0) ? 1 : 0;
  int expected = -1;
  hb::g_nancheck.compare_exchange_strong(expected, value);
  return hb::g_nancheck.load();
}

#define HB_LAPACKE_LU(p, T)                                                           \
  HWYBLAS_API lapack_int LAPACKE_##p##getrf(int layout, lapack_int m, lapack_int n,   \
                                            T* a, lapack_int lda, lapack_int* ipiv) { \
    return hb::GetrfMain<T>(layout, m, n, a, lda, ipiv, false);                       \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##getrf_work(int layout, lapack_int m,            \
                                                 lapack_int n, T* a, lapack_int lda,  \
                                                 lapack_int* ipiv) {                  \
    return hb::GetrfWork<T>(layout, m, n, a, lda, ipiv, false);                       \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##getrf2(int layout, lapack_int m, lapack_int n,  \
                                             T* a, lapack_int lda, lapack_int* ipiv) { \
    return hb::GetrfMain<T>(layout, m, n, a, lda, ipiv, true);                        \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##getrf2_work(int layout, lapack_int m,           \
                                                  lapack_int n, T* a, lapack_int lda, \
                                                  lapack_int* ipiv) {                 \
    return hb::GetrfWork<T>(layout, m, n, a, lda, ipiv, true);                        \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##getrs(int layout, char trans, lapack_int n,     \
                                            lapack_int nrhs, const T* a,              \
                                            lapack_int lda, const lapack_int* ipiv,   \
                                            T* b, lapack_int ldb) {                   \
    return hb::GetrsMain<T>(layout, trans, n, nrhs, a, lda, ipiv, b, ldb);            \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##getrs_work(                                     \
      int layout, char trans, lapack_int n, lapack_int nrhs, const T* a,              \
      lapack_int lda, const lapack_int* ipiv, T* b, lapack_int ldb) {                 \
    return hb::GetrsWork<T>(layout, trans, n, nrhs, a, lda, ipiv, b, ldb);            \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##gesv(int layout, lapack_int n, lapack_int nrhs, \
                                           T* a, lapack_int lda, lapack_int* ipiv,    \
                                           T* b, lapack_int ldb) {                    \
    return hb::GesvMain<T>(layout, n, nrhs, a, lda, ipiv, b, ldb);                    \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##gesv_work(int layout, lapack_int n,             \
                                                lapack_int nrhs, T* a, lapack_int lda, \
                                                lapack_int* ipiv, T* b,               \
                                                lapack_int ldb) {                     \
    return hb::GesvWork<T>(layout, n, nrhs, a, lda, ipiv, b, ldb);                    \
  }

#define HB_LAPACKE_INV(p, T)                                                              \
  HWYBLAS_API lapack_int LAPACKE_##p##getri(int layout, lapack_int n, T* a, lapack_int lda,  \
                                            const lapack_int* ipiv) {                       \
    return hb::GetriMain<T>(layout, n, a, lda, ipiv);                                       \
  }                                                                                         \
  HWYBLAS_API lapack_int LAPACKE_##p##getri_work(int layout, lapack_int n, T* a,            \
                                                 lapack_int lda, const lapack_int* ipiv,    \
                                                 T* work, lapack_int lwork) {               \
    return hb::GetriWork<T>(layout, n, a, lda, ipiv, work, lwork);                          \
  }                                                                                         \
  HWYBLAS_API lapack_int LAPACKE_##p##trtri(int layout, char uplo, char diag, lapack_int n, \
                                            T* a, lapack_int lda) {                         \
    return hb::TrtriMain<T>(layout, uplo, diag, n, a, lda);                                 \
  }                                                                                         \
  HWYBLAS_API lapack_int LAPACKE_##p##trtri_work(int layout, char uplo, char diag,          \
                                                 lapack_int n, T* a, lapack_int lda) {      \
    return hb::TrtriWork<T>(layout, uplo, diag, n, a, lda);                                 \
  }
HB_LAPACKE_INV(d, double)
HB_LAPACKE_INV(s, float)
#undef HB_LAPACKE_INV

HB_LAPACKE_LU(d, double)
HB_LAPACKE_LU(s, float)
#undef HB_LAPACKE_LU

#define HB_LAPACKE_PO(p, T)                                                           \
  HWYBLAS_API lapack_int LAPACKE_##p##potrf(int layout, char uplo, lapack_int n, T* a, \
                                            lapack_int lda) {                         \
    return hb::PotrfMain<T>(layout, uplo, n, a, lda, false);                          \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##potrf_work(int layout, char uplo, lapack_int n, \
                                                 T* a, lapack_int lda) {              \
    return hb::PotrfWork<T>(layout, uplo, n, a, lda, false);                          \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##potrf2(int layout, char uplo, lapack_int n,     \
                                             T* a, lapack_int lda) {                  \
    return hb::PotrfMain<T>(layout, uplo, n, a, lda, true);                           \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##potrf2_work(int layout, char uplo, lapack_int n, \
                                                  T* a, lapack_int lda) {             \
    return hb::PotrfWork<T>(layout, uplo, n, a, lda, true);                           \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##potrs(int layout, char uplo, lapack_int n,      \
                                            lapack_int nrhs, const T* a,              \
                                            lapack_int lda, T* b, lapack_int ldb) {   \
    return hb::PosMain<T>(layout, uplo, n, nrhs, const_cast<T*>(a), lda, b, ldb, true); \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##potrs_work(int layout, char uplo, lapack_int n, \
                                                 lapack_int nrhs, const T* a,         \
                                                 lapack_int lda, T* b, lapack_int ldb) { \
    return hb::PosWork<T>(layout, uplo, n, nrhs, const_cast<T*>(a), lda, b, ldb, true); \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##posv(int layout, char uplo, lapack_int n,       \
                                           lapack_int nrhs, T* a, lapack_int lda,     \
                                           T* b, lapack_int ldb) {                    \
    return hb::PosMain<T>(layout, uplo, n, nrhs, a, lda, b, ldb, false);              \
  }                                                                                   \
  HWYBLAS_API lapack_int LAPACKE_##p##posv_work(int layout, char uplo, lapack_int n,  \
                                                lapack_int nrhs, T* a, lapack_int lda, \
                                                T* b, lapack_int ldb) {               \
    return hb::PosWork<T>(layout, uplo, n, nrhs, a, lda, b, ldb, false);              \
  }

HB_LAPACKE_PO(d, double)
HB_LAPACKE_PO(s, float)
#undef HB_LAPACKE_PO

}  // extern "C"
