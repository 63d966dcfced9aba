// Glue for building the reference's own LU/Cholesky drivers (TEST
// INFRASTRUCTURE ONLY). The reference's src/lapack/getrf.cc, potrf.cc,
// triangular.cc and environment.cc compile without Highway; they reach BLAS through the exported
// Fortran symbols (src/lapack/blas.h:48-79, 338-352) and their leaves through
// hwyblas::lapack::GetrfLeaf/PotrfLeaf (src/lapack/factor_kernels.h:34-40).
// The Highway-based BLAS itself cannot be built here (Highway is absent), so
// this file supplies those symbols from the oracle's restatement. Linking the
// reference drivers to them lets the tests check the oracle's own LAPACK
// restatement against the reference's driver code, bit for bit.
//
// The complex LU and Cholesky leaves and the complex GEMM, TRSM and HERK come
// from the oracle as well (zgetrf_, zpotrf_ and their c forms are checked).
// Routines the checked path never reaches (norms and condition estimates)
// abort; the Fortran ones are in ref_stubs.c. triangular.cc is
// built too, for xTRTRI and xTRTI2 under xGETRI, and gesvx.cc and trsen.cc
// for xGERFS and its xLACN2.
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <utility>

#include "src/common.h"
#include "src/lapack/factor_kernels.h"
#include "oracle_internal.h"

namespace {
[[noreturn]] void Unreached(const char* name) {
  fprintf(stderr, "oracle/_ref: %s is not part of the checked path\n", name);
  abort();
}
int g_last_error_pos = 0;
char g_last_error_name[16] = {0};
}  // namespace

namespace hwyblas {
void ReportError(const char* routine, blasint info) {
  g_last_error_pos = info;
  snprintf(g_last_error_name, sizeof(g_last_error_name), "%s", routine);
}

namespace lapack {
template <typename T>
blasint GetrfLeaf(blasint m, blasint n, T* a, blasint lda, blasint* ipiv) {
  return orc::GetrfLeaf<T>(m, n, a, lda, ipiv);
}
template <typename T>
blasint PotrfLeaf(bool upper, blasint n, T* a, blasint lda) {
  return orc::PotrfLeaf<T>(upper, n, a, lda);
}
template <typename T>
void Lacgv(blasint, T*, blasint) {
  Unreached("Lacgv");
}
// Norms and safe scaling: only xTRCON, xTRRFS, xLATRS, xGECON and xGESVX use
// them, and the checked paths (xTRTRI, xTRTI2, xGERFS) do not.
template <typename T>
void Rscl(blasint, RealT<T>, T*, blasint) {
  Unreached("Rscl");
}
template <typename T>
RealT<T> Lange(char, blasint, blasint, const T*, blasint, RealT<T>*) {
  Unreached("Lange");
}
template <typename T>
RealT<T> Lantr(char, char, char, blasint, blasint, const T*, blasint, RealT<T>*) {
  Unreached("Lantr");
}
template <typename T>
T Ladiv(T, T) {
  Unreached("Ladiv");
}
template std::complex<float> Ladiv<std::complex<float>>(std::complex<float>,
                                                        std::complex<float>);
template std::complex<double> Ladiv<std::complex<double>>(std::complex<double>,
                                                          std::complex<double>);
// Householder, rotation and eigenvalue helpers of trsen.cc (built only for
// its xLACN2) and the complex helpers of gesvx.cc: never reached.
template <typename R>
void Ladiv(R, R, R, R, R*, R*) {
  Unreached("Ladiv");
}
template <typename T>
void Lacpy(char, blasint, blasint, const T*, blasint, T*, blasint) {
  Unreached("Lacpy");
}
template <typename T>
void Larfg(blasint, T*, T*, blasint, T*) {
  Unreached("Larfg");
}
template <typename T>
void Larf(char, blasint, blasint, const T*, blasint, T, T*, blasint, T*) {
  Unreached("Larf");
}
template <typename R>
void Lartg(R, R, R*, R*, R*) {
  Unreached("Lartg");
}
template <typename R>
void Lanv2(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*) {
  Unreached("Lanv2");
}
template <typename T>
std::enable_if_t<IsComplex<T>::value> Lartg(T, T, RealT<T>*, T*, T*) {
  Unreached("Lartg");
}
template <typename T>
std::enable_if_t<IsComplex<T>::value> Rot(blasint, T*, blasint, T*, blasint, RealT<T>, T) {
  Unreached("Rot");
}
template <typename T>
blasint Imax1(blasint, const T*, blasint) {
  Unreached("Imax1");
}
template <typename T>
RealT<T> Sum1(blasint, const T*, blasint) {
  Unreached("Sum1");
}
#define ORC_REAL_INST(R)                                                   \
  template void Ladiv<R>(R, R, R, R, R*, R*);                              \
  template void Lartg<R>(R, R, R*, R*, R*);                                \
  template void Lanv2<R>(R*, R*, R*, R*, R*, R*, R*, R*, R*, R*);
ORC_REAL_INST(float)
ORC_REAL_INST(double)
#undef ORC_REAL_INST
#define ORC_CPLX_INST(T)                                                   \
  template std::enable_if_t<IsComplex<T>::value> Lartg<T>(T, T, RealT<T>*, T*, T*); \
  template std::enable_if_t<IsComplex<T>::value> Rot<T>(blasint, T*, blasint, T*, blasint, \
                                                        RealT<T>, T);     \
  template blasint Imax1<T>(blasint, const T*, blasint);                   \
  template RealT<T> Sum1<T>(blasint, const T*, blasint);
ORC_CPLX_INST(std::complex<float>)
ORC_CPLX_INST(std::complex<double>)
#undef ORC_CPLX_INST
#define ORC_INST(T)                                                   \
  template blasint GetrfLeaf<T>(blasint, blasint, T*, blasint, blasint*); \
  template blasint PotrfLeaf<T>(bool, blasint, T*, blasint);          \
  template void Lacgv<T>(blasint, T*, blasint);                       \
  template void Rscl<T>(blasint, RealT<T>, T*, blasint);              \
  template void Lacpy<T>(char, blasint, blasint, const T*, blasint, T*, blasint); \
  template void Larfg<T>(blasint, T*, T*, blasint, T*);               \
  template void Larf<T>(char, blasint, blasint, const T*, blasint, T, T*, blasint, T*); \
  template RealT<T> Lange<T>(char, blasint, blasint, const T*, blasint, RealT<T>*); \
  template RealT<T> Lantr<T>(char, char, char, blasint, blasint, const T*, blasint, RealT<T>*);
ORC_INST(float)
ORC_INST(double)
ORC_INST(std::complex<float>)
ORC_INST(std::complex<double>)
#undef ORC_INST
}  // namespace lapack
}  // namespace hwyblas

using hwyblas::blasint;

extern "C" {
int orc_ref_last_error(char* name, int len) {
  if (name && len > 0) snprintf(name, len, "%s", g_last_error_name);
  const int p = g_last_error_pos;
  g_last_error_pos = 0;
  return p;
}

void dgemm_(const char* ta, const char* tb, const blasint* m, const blasint* n,
            const blasint* k, const double* alpha, const double* a,
            const blasint* lda, const double* b, const blasint* ldb,
            const double* beta, double* c, const blasint* ldc) {
  const int info = orc::GemmF<double>(*ta, *tb, *m, *n, *k, *alpha, a, *lda, b,
                                      *ldb, *beta, c, *ldc);
  if (info) hwyblas::ReportError("DGEMM", info);
}
void sgemm_(const char* ta, const char* tb, const blasint* m, const blasint* n,
            const blasint* k, const float* alpha, const float* a,
            const blasint* lda, const float* b, const blasint* ldb,
            const float* beta, float* c, const blasint* ldc) {
  const int info = orc::GemmF<float>(*ta, *tb, *m, *n, *k, *alpha, a, *lda, b,
                                     *ldb, *beta, c, *ldc);
  if (info) hwyblas::ReportError("SGEMM", info);
}
void dtrsm_(const char* s, const char* u, const char* t, const char* d,
            const blasint* m, const blasint* n, const double* alpha,
            const double* a, const blasint* lda, double* b,
            const blasint* ldb) {
  const int info =
      orc::TrsmF<double>(*s, *u, *t, *d, *m, *n, *alpha, a, *lda, b, *ldb);
  if (info) hwyblas::ReportError("DTRSM", info);
}
void strsm_(const char* s, const char* u, const char* t, const char* d,
            const blasint* m, const blasint* n, const float* alpha,
            const float* a, const blasint* lda, float* b, const blasint* ldb) {
  const int info =
      orc::TrsmF<float>(*s, *u, *t, *d, *m, *n, *alpha, a, *lda, b, *ldb);
  if (info) hwyblas::ReportError("STRSM", info);
}
void dsyrk_(const char* u, const char* t, const blasint* n, const blasint* k,
            const double* alpha, const double* a, const blasint* lda,
            const double* beta, double* c, const blasint* ldc) {
  const int info = orc::SyrkD(*u, *t, *n, *k, *alpha, a, *lda, *beta, c, *ldc);
  if (info) hwyblas::ReportError("DSYRK", info);
}
void ssyrk_(const char* u, const char* t, const blasint* n, const blasint* k,
            const float* alpha, const float* a, const blasint* lda, const float* beta,
            float* c, const blasint* ldc) {
  const int info = orc::Syrk<float>(*u, *t, *n, *k, *alpha, a, *lda, *beta, c, *ldc);
  if (info) hwyblas::ReportError("SSYRK", info);
}
#define ORC_ZL3(P, U, R)                                                                  \
  void P##gemm_(const char* ta, const char* tb, const blasint* m, const blasint* n,        \
                const blasint* k, const R* alpha, const R* a, const blasint* lda,          \
                const R* b, const blasint* ldb, const R* beta, R* c, const blasint* ldc) { \
    const int info =                                                                       \
        orc::ZgemmF<R>(*ta, *tb, *m, *n, *k, alpha, a, *lda, b, *ldb, beta, c, *ldc);      \
    if (info) hwyblas::ReportError(U "GEMM", info);                                        \
  }                                                                                        \
  void P##trsm_(const char* s, const char* u, const char* t, const char* d,                \
                const blasint* m, const blasint* n, const R* alpha, const R* a,            \
                const blasint* lda, R* b, const blasint* ldb) {                            \
    const int info = orc::ZtrsmF<R>(*s, *u, *t, *d, *m, *n, alpha, a, *lda, b, *ldb);     \
    if (info) hwyblas::ReportError(U "TRSM", info);                                        \
  }
#define ORC_ZHERK(P, U, R)                                                                \
  void P##herk_(const char* u, const char* t, const blasint* n, const blasint* k,           \
                const R* alpha, const R* a, const blasint* lda, const R* beta, R* c,        \
                const blasint* ldc) {                                                      \
    const int info = orc::ZherkF<R>(*u, *t, *n, *k, *alpha, a, *lda, *beta, c, *ldc);      \
    if (info) hwyblas::ReportError(U "HERK", info);                                        \
  }
ORC_ZHERK(z, "Z", double)
ORC_ZHERK(c, "C", float)
#undef ORC_ZHERK
ORC_ZL3(z, "Z", double)
ORC_ZL3(c, "C", float)
#undef ORC_ZL3
blasint idamax_(const blasint* n, const double* x, const blasint* incx) {
  return orc::Iamax<double>(*n, x, *incx);
}
blasint isamax_(const blasint* n, const float* x, const blasint* incx) {
  return orc::Iamax<float>(*n, x, *incx);
}
// TRMV, GEMV, SWAP, ASUM, COPY and AXPY for xTRTI2, xGETRI, xGERFS and xLACN2:
// unit strides, the only form those drivers use (src/lapack/triangular.cc:
// 46-75; src/lapack/getrf.cc:436-476; src/lapack/gesvx.cc:407-440;
// src/lapack/trsen.cc:2284-2360).
#define ORC_L2(P, T)                                                                      \
  void P##trmv_(const char* u, const char* t, const char* d, const blasint* n, const T* a, \
                const blasint* lda, T* x, const blasint* incx) {                          \
    if ((*t != 'N' && *t != 'n') || *incx != 1) Unreached(#P "trmv_ form");                \
    orc::TrmvN<T>(*u == 'L' || *u == 'l', *d == 'U' || *d == 'u', *n, a, *lda, x);       \
  }                                                                                        \
  void P##gemv_(const char* t, const blasint* m, const blasint* n, const T* alpha,         \
                const T* a, const blasint* lda, const T* x, const blasint* incx,           \
                const T* beta, T* y, const blasint* incy) {                                \
    if (*incx != 1 || *incy != 1) Unreached(#P "gemv_ form");                             \
    if (*t == 'N' || *t == 'n') orc::GemvN<T>(*m, *n, *alpha, a, *lda, x, *beta, y);       \
    else orc::GemvT<T>(*m, *n, *alpha, a, *lda, x, *beta, y);                              \
  }                                                                                        \
  T P##asum_(const blasint* n, const T* x, const blasint* incx) {                          \
    if (*incx != 1) Unreached(#P "asum_ form");                                            \
    return orc::AbsSum<T>(*n, x);                                                          \
  }                                                                                        \
  void P##copy_(const blasint* n, const T* x, const blasint* incx, T* y,                   \
                const blasint* incy) {                                                     \
    for (blasint i = 0; i < *n; ++i) y[i * *incy] = x[i * *incx];                         \
  }                                                                                        \
  void P##axpy_(const blasint* n, const T* alpha, const T* x, const blasint* incx, T* y,   \
                const blasint* incy) {                                                     \
    if (*incx != 1 || *incy != 1) Unreached(#P "axpy_ form");                             \
    orc::AxpyRef<T>(*n, *alpha, x, y);                                                     \
  }                                                                                        \
  void P##swap_(const blasint* n, T* x, const blasint* incx, T* y, const blasint* incy) {  \
    for (blasint i = 0; i < *n; ++i) std::swap(x[i * *incx], y[i * *incy]);               \
  }                                                                                        \
  void P##trmm_(const char* s, const char* u, const char* t, const char* d,                \
                const blasint* m, const blasint* n, const T* alpha, const T* a,            \
                const blasint* lda, T* b, const blasint* ldb) {                            \
    const int info = orc::Trmm<T>(*s, *u, *t, *d, *m, *n, *alpha, a, *lda, b, *ldb);      \
    if (info) hwyblas::ReportError(#P "TRMM", info);                                       \
  }
ORC_L2(d, double)
ORC_L2(s, float)
#undef ORC_L2

void dscal_(const blasint* n, const double* a, double* x, const blasint* incx) {
  if (*n <= 0 || *incx <= 0) return;
  for (blasint i = 0; i < *n; ++i) x[i * *incx] *= *a;
}
void sscal_(const blasint* n, const float* a, float* x, const blasint* incx) {
  if (*n <= 0 || *incx <= 0) return;
  for (blasint i = 0; i < *n; ++i) x[i * *incx] *= *a;
}

}  // extern "C"
