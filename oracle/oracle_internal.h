// Shared declarations of the oracle (TEST INFRASTRUCTURE ONLY).
#ifndef HWYBLAS_ORACLE_INTERNAL_H_
#define HWYBLAS_ORACLE_INTERNAL_H_

#include <cstddef>

namespace orc {

extern int g_lanes;    // doubles per vector of the reference's SIMD target
extern int g_threads;  // OpenMP threads of the GEMM restatement

// Element (i, p) of op(X) is data[i * rs + p * cs] (src/gemm.h:28-36).
template <typename T>
struct Opnd {
  const T* data = nullptr;
  ptrdiff_t rs = 1, cs = 1;
  T at(size_t i, size_t p) const {
    return data[static_cast<ptrdiff_t>(i) * rs + static_cast<ptrdiff_t>(p) * cs];
  }
  Opnd sub(size_t i0, size_t j0) const {
    Opnd o = *this;
    o.data += static_cast<ptrdiff_t>(i0) * rs + static_cast<ptrdiff_t>(j0) * cs;
    return o;
  }
};

enum Part { kAll = 0, kLower = 1, kUpper = 2 };

template <typename T>
void Gemm(size_t m, size_t n, size_t k, T alpha, Opnd<T> a, Opnd<T> b, T beta,
          T* c, size_t ldc, Part part);
template <typename T>
int GemmF(char transa, char transb, int m, int n, int k, T alpha, const T* a,
          int lda, const T* b, int ldb, T beta, T* c, int ldc);
template <typename T>
int TrsmF(char side, char uplo, char transa, char diag, int m, int n, T alpha,
          const T* a, int lda, T* b, int ldb);
int SyrkD(char uplo, char trans, int n, int k, double alpha, const double* a,
          int lda, double beta, double* c, int ldc);
template <typename T>
int Syrk(char uplo, char trans, int n, int k, T alpha, const T* a, int lda, T beta, T* c,
         int ldc);
template <typename T>
int Iamax(int n, const T* x, int incx);
// Complex GEMM and TRSM on interleaved (re, im) arrays, alpha and beta as
// (re, im) pairs (oracle_blas.cc).
template <typename R>
int ZgemmF(char transa, char transb, int m, int n, int k, const R* alpha, const R* a, int lda,
           const R* b, int ldb, const R* beta, R* c, int ldc);
template <typename R>
int ZtrsmF(char side, char uplo, char transa, char diag, int m, int n, const R* alpha,
           const R* a, int lda, R* b, int ldb);
template <typename R>
int ZherkF(char uplo, char trans, int n, int k, R alpha, const R* a, int lda, R beta, R* c,
           int ldc);
template <typename T>
int Trmm(char side, char uplo, char transa, char diag, int m, int n, T alpha, const T* a,
         int lda, T* b, int ldb);
// TRMV with op N and GEMV with op N on contiguous vectors, in the
// reference's kernel order (src/trmv-inl.h, src/gemv-inl.h).
template <typename T>
void TrmvN(bool lower, bool unit, int n, const T* a, int lda, T* x);
template <typename T>
void GemvN(int m, int n, T alpha, const T* a, int lda, const T* x, T beta, T* y);
template <typename T>
void GemvT(int m, int n, T alpha, const T* a, int lda, const T* x, T beta, T* y);
// ASUM and AXPY on contiguous vectors in the reference's lane order
// (src/level1-inl.h:37-76, 186-217).
template <typename T>
T AbsSum(int n, const T* x);
template <typename T>
void AxpyRef(int n, T alpha, const T* x, T* y);

template <typename T>
int GetrfLeaf(int m, int n, T* a, int lda, int* ipiv);
template <typename T>
int PotrfLeaf(bool upper, int n, T* a, int lda);

}  // namespace orc

#endif  // HWYBLAS_ORACLE_INTERNAL_H_
