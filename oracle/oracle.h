/* Oracle for the parity tests: a CPU restatement of hwyBLAS's level-3 hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: tests/, the smoke
 * check in __graft_entry__.py and the CPU-baseline legs of bench.py may load
 * it; the product library (hwyblas_b200/) never links, loads or calls it.
 *
 * Every routine follows the reference's per-element operation order exactly
 * (sequential FMA over k in chunks of KC, alpha/beta merge order, recursion
 * split points, pivot choice), so results are bit-identical to the reference
 * built for a target with `lanes` doubles per vector (8 = AVX-512, 4 = AVX2;
 * the lane count only changes the rounding of short AXPY columns in the LU and
 * Cholesky leaves and the micro-tile geometry of triangular-C SYRK).
 *
 * Argument errors are returned as the 1-based Fortran position (BLAS) or
 * -position (LAPACK INFO), and nothing is printed.
 */
#ifndef HWYBLAS_ORACLE_H_
#define HWYBLAS_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

void orc_set_lanes(int lanes);
int orc_get_lanes(void);
void orc_set_threads(int threads);

/* BLAS. Return 0 or the Fortran position of the first invalid argument. */
int orc_dgemm(char transa, char transb, int m, int n, int k, double alpha,
              const double* a, int lda, const double* b, int ldb, double beta,
              double* c, int ldc);
int orc_sgemm(char transa, char transb, int m, int n, int k, float alpha,
              const float* a, int lda, const float* b, int ldb, float beta,
              float* c, int ldc);
int orc_dtrsm(char side, char uplo, char transa, char diag, int m, int n,
              double alpha, const double* a, int lda, double* b, int ldb);
int orc_strsm(char side, char uplo, char transa, char diag, int m, int n,
              float alpha, const float* a, int lda, float* b, int ldb);
int orc_ssyrk(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
              float beta, float* c, int ldc);
int orc_dsyrk(char uplo, char trans, int n, int k, double alpha,
              const double* a, int lda, double beta, double* c, int ldc);
int orc_idamax(int n, const double* x, int incx);
int orc_isamax(int n, const float* x, int incx);

/* LAPACK. Return INFO as the reference does. */
void orc_dlaswp(int n, double* a, int lda, int k1, int k2, const int* ipiv,
                int incx);
int orc_dgetrf(int m, int n, double* a, int lda, int* ipiv);
int orc_dgetrf2(int m, int n, double* a, int lda, int* ipiv);
int orc_sgetrf(int m, int n, float* a, int lda, int* ipiv);
int orc_sgetrf2(int m, int n, float* a, int lda, int* ipiv);
void orc_slaswp(int n, float* a, int lda, int k1, int k2, const int* ipiv, int incx);
int orc_sgesv(int n, int nrhs, float* a, int lda, int* ipiv, float* b, int ldb);
int orc_dgetrs(char trans, int n, int nrhs, const double* a, int lda,
               const int* ipiv, double* b, int ldb);
int orc_sgetrs(char trans, int n, int nrhs, const float* a, int lda,
               const int* ipiv, float* b, int ldb);
int orc_dgesv(int n, int nrhs, double* a, int lda, int* ipiv, double* b,
              int ldb);
int orc_dpotrf(char uplo, int n, double* a, int lda);
int orc_dpotrf2(char uplo, int n, double* a, int lda);
int orc_dpotrs(char uplo, int n, int nrhs, const double* a, int lda, double* b,
               int ldb);
int orc_spotrf(char uplo, int n, float* a, int lda);
int orc_spotrf2(char uplo, int n, float* a, int lda);
int orc_spotrs(char uplo, int n, int nrhs, const float* a, int lda, float* b, int ldb);
int orc_sposv(char uplo, int n, int nrhs, float* a, int lda, float* b, int ldb);
int orc_dposv(char uplo, int n, int nrhs, double* a, int lda, double* b,
              int ldb);

/* Complex GEMM, interleaved (re, im) (src/gemm.cc:67-123,
 * src/gemm_kernel-inl.h:226-428). */
int orc_zgemm(char ta, char tb, int m, int n, int k, const double* alpha, const double* a,
              int lda, const double* b, int ldb, const double* beta, double* c, int ldc);
int orc_cgemm(char ta, char tb, int m, int n, int k, const float* alpha, const float* a,
              int lda, const float* b, int ldb, const float* beta, float* c, int ldc);
/* Complex TRSM (src/trsm.cc:87-180, src/trsm-inl.h:175-214) and the complex
 * reciprocal of the C++ runtime (pins the device's restatement). */
int orc_ztrsm(char side, char uplo, char ta, char diag, int m, int n, const double* alpha,
              const double* a, int lda, double* b, int ldb);
int orc_ctrsm(char side, char uplo, char ta, char diag, int m, int n, const float* alpha,
              const float* a, int lda, float* b, int ldb);
void orc_zrecip(int n, const double* c, double* out);
void orc_crecip(int n, const float* c, float* out);
/* Complex HERK (src/level3.cc:85-140, 439-452), alpha and beta real. */
int orc_zherk(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
              double beta, double* c, int ldc);
int orc_cherk(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
              float beta, float* c, int ldc);
/* Complex Cholesky family (src/lapack/potrf.cc, posv.cc at std::complex). */
int orc_zpotrf(char uplo, int n, double* a, int lda);
int orc_zpotrf2(char uplo, int n, double* a, int lda);
int orc_zpotrs(char uplo, int n, int nrhs, const double* a, int lda, double* b, int ldb);
int orc_zposv(char uplo, int n, int nrhs, double* a, int lda, double* b, int ldb);
int orc_cpotrf(char uplo, int n, float* a, int lda);
int orc_cpotrf2(char uplo, int n, float* a, int lda);
int orc_cpotrs(char uplo, int n, int nrhs, const float* a, int lda, float* b, int ldb);
int orc_cposv(char uplo, int n, int nrhs, float* a, int lda, float* b, int ldb);
/* Complex LU family (src/lapack/getrf.cc:28-374 at std::complex). */
int orc_zgetrf(int m, int n, double* a, int lda, int* ipiv);
int orc_zgetrf2(int m, int n, double* a, int lda, int* ipiv);
void orc_zlaswp(int n, double* a, int lda, int k1, int k2, const int* ipiv, int incx);
int orc_zgetrs(char trans, int n, int nrhs, const double* a, int lda, const int* ipiv,
               double* b, int ldb);
int orc_zgesv(int n, int nrhs, double* a, int lda, int* ipiv, double* b, int ldb);
int orc_cgetrf(int m, int n, float* a, int lda, int* ipiv);
int orc_cgetrf2(int m, int n, float* a, int lda, int* ipiv);
void orc_claswp(int n, float* a, int lda, int k1, int k2, const int* ipiv, int incx);
int orc_cgetrs(char trans, int n, int nrhs, const float* a, int lda, const int* ipiv,
               float* b, int ldb);
int orc_cgesv(int n, int nrhs, float* a, int lda, int* ipiv, float* b, int ldb);
/* Level 3 through the GEMM problem model (src/level3.cc:26-342). */
int orc_dsymm(char side, char uplo, int m, int n, double alpha, const double* a, int lda,
              const double* b, int ldb, double beta, double* c, int ldc);
int orc_ssymm(char side, char uplo, int m, int n, float alpha, const float* a, int lda,
              const float* b, int ldb, float beta, float* c, int ldc);
int orc_dsyr2k(char uplo, char trans, int n, int k, double alpha, const double* a, int lda,
               const double* b, int ldb, double beta, double* c, int ldc);
int orc_ssyr2k(char uplo, char trans, int n, int k, float alpha, const float* a, int lda,
               const float* b, int ldb, float beta, float* c, int ldc);
int orc_dgemmtr(char uplo, char ta, char tb, int n, int k, double alpha, const double* a,
                int lda, const double* b, int ldb, double beta, double* c, int ldc);
int orc_sgemmtr(char uplo, char ta, char tb, int n, int k, float alpha, const float* a,
                int lda, const float* b, int ldb, float beta, float* c, int ldc);
int orc_dtrmm(char side, char uplo, char transa, char diag, int m, int n, double alpha,
              const double* a, int lda, double* b, int ldb);
int orc_strmm(char side, char uplo, char transa, char diag, int m, int n, float alpha,
              const float* a, int lda, float* b, int ldb);

/* Triangular inverse and GETRI (src/lapack/triangular.cc:18-166,
 * src/lapack/getrf.cc:369-483). */
int orc_dtrti2(char uplo, char diag, int n, double* a, int lda);
int orc_strti2(char uplo, char diag, int n, float* a, int lda);
int orc_dtrtri(char uplo, char diag, int n, double* a, int lda);
int orc_strtri(char uplo, char diag, int n, float* a, int lda);
int orc_dgetri(int n, double* a, int lda, const int* ipiv, double* work, int lwork);
int orc_sgetri(int n, float* a, int lda, const int* ipiv, float* work, int lwork);

/* Iterative refinement with error bounds (src/lapack/gesvx.cc:319-456);
 * work holds 3 n, iwork n. */
int orc_dgerfs(char trans, int n, int nrhs, const double* a, int lda, const double* af,
               int ldaf, const int* ipiv, const double* b, int ldb, double* x, int ldx,
               double* ferr, double* berr, double* work, int* iwork);
int orc_sgerfs(char trans, int n, int nrhs, const float* a, int lda, const float* af,
               int ldaf, const int* ipiv, const float* b, int ldb, float* x, int ldx,
               float* ferr, float* berr, float* work, int* iwork);

/* Leaves, exposed for the known-answer tests. */
int orc_dgetrf_leaf(int m, int n, double* a, int lda, int* ipiv);
int orc_dpotrf_leaf(int upper, int n, double* a, int lda);

#ifdef __cplusplus
}
#endif
#endif /* HWYBLAS_ORACLE_H_ */
