/*
 * hwyBLAS-B200: the level-3 hot path of hwyBLAS (GEMM, TRSM, SYRK, I?AMAX and
 * the LU / Cholesky drivers built on them) as hand-written CUDA kernels for
 * NVIDIA B200 (sm_100a), behind the reference's own C ABI.
 *
 * Calling convention (as the reference, include/hwyblas/hwyblas.h:1-16):
 * Fortran-77 style, every argument by pointer, column-major, 32-bit integers,
 * only the first character of CHARACTER arguments is read (case-insensitive)
 * and the hidden length arguments are neither declared nor read.
 *
 * Memory: every matrix or vector pointer may be host memory (pageable or
 * pinned; the library copies it to the GPU and back) or device / managed
 * memory of the current CUDA device (used in place). All calls are
 * synchronous on return, as BLAS requires. Work is issued on the library's
 * per-thread stream, or on the stream set with hwyblas_set_stream.
 *
 * Errors: an invalid argument calls xerbla_ (or the handler installed with
 * hwyblas_set_error_handler) with the reference's Fortran argument position
 * and returns without side effects; LAPACK routines return INFO < 0 / > 0 as
 * the reference does. A CUDA failure is reported through
 * hwyblas_last_cuda_error() and a message on stderr; there is no CPU fallback.
 */
#ifndef HWYBLAS_B200_H_
#define HWYBLAS_B200_H_

#include <stddef.h>
#include <stdint.h>

#define HWYBLAS_API __attribute__((visibility("default")))

#ifdef __cplusplus
extern "C" {
#endif

typedef int hwyblas_int;

/* ------------------------------------------------------------------------ */
/* Fortran BLAS                                                             */

/* C := alpha*op(A)*op(B) + beta*C. Replaces dgemm_
 * (include/hwyblas/hwyblas.h:570, src/gemm.cc:151-158). Per element the
 * result is bit-identical to the reference: sequential FMA over k in chunks
 * of 256, merged as alpha*acc (+ C, or fma(C, beta, .)). */
HWYBLAS_API void dgemm_(const char* transa, const char* transb,
                        const hwyblas_int* m, const hwyblas_int* n,
                        const hwyblas_int* k, const double* alpha,
                        const double* a, const hwyblas_int* lda,
                        const double* b, const hwyblas_int* ldb,
                        const double* beta, double* c, const hwyblas_int* ldc);
/* Replaces sgemm_ (include/hwyblas/hwyblas.h:564, src/gemm.cc:142-149);
 * chunks of 384. */
HWYBLAS_API void sgemm_(const char* transa, const char* transb,
                        const hwyblas_int* m, const hwyblas_int* n,
                        const hwyblas_int* k, const float* alpha,
                        const float* a, const hwyblas_int* lda, const float* b,
                        const hwyblas_int* ldb, const float* beta, float* c,
                        const hwyblas_int* ldc);
/* Solves op(A)*X = alpha*B or X*op(A) = alpha*B in place. Replaces dtrsm_
 * (include/hwyblas/hwyblas.h:792, src/trsm.cc:196-201). */
HWYBLAS_API void dtrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m,
                        const hwyblas_int* n, const double* alpha,
                        const double* a, const hwyblas_int* lda, double* b,
                        const hwyblas_int* ldb);
/* Single precision (include/hwyblas/hwyblas.h:787, src/trsm.cc:190-195):
 * the same algorithm at float. */
HWYBLAS_API void strsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m,
                        const hwyblas_int* n, const float* alpha,
                        const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb);
/* C := alpha*A*A**T + beta*C (trans N) or alpha*A**T*A + beta*C on one
 * triangle. Replaces dsyrk_ (include/hwyblas/hwyblas.h:637,
 * src/level3.cc:416-421). */
HWYBLAS_API void dsyrk_(const char* uplo, const char* trans,
                        const hwyblas_int* n, const hwyblas_int* k,
                        const double* alpha, const double* a,
                        const hwyblas_int* lda, const double* beta, double* c,
                        const hwyblas_int* ldc);
/* Single precision (include/hwyblas/hwyblas.h:632, src/level3.cc:410-415). */
HWYBLAS_API void ssyrk_(const char* uplo, const char* trans,
                        const hwyblas_int* n, const hwyblas_int* k,
                        const float* alpha, const float* a,
                        const hwyblas_int* lda, const float* beta, float* c,
                        const hwyblas_int* ldc);
/* Complex GEMM, interleaved (re, im) arrays, leading dimensions in complex
 * elements, transa/transb N, T or C (conjugate transpose); bit-identical to
 * the reference's complex micro-kernel. Replace zgemm_ / cgemm_
 * (include/hwyblas/hwyblas.h:582, 576; src/gemm.cc:67-123). */
HWYBLAS_API void zgemm_(const char* transa, const char* transb, const hwyblas_int* m,
                        const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                        const double* a, const hwyblas_int* lda, const double* b,
                        const hwyblas_int* ldb, const double* beta, double* c,
                        const hwyblas_int* ldc);
HWYBLAS_API void cgemm_(const char* transa, const char* transb, const hwyblas_int* m,
                        const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                        const float* a, const hwyblas_int* lda, const float* b,
                        const hwyblas_int* ldb, const float* beta, float* c,
                        const hwyblas_int* ldc);
/* Complex TRSM in place, transa N, T or C; interleaved arrays. Replace
 * ztrsm_ / ctrsm_ (include/hwyblas/hwyblas.h:802, 797; src/trsm.cc:137-180,
 * 202-215). */
HWYBLAS_API void ztrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const double* alpha, const double* a, const hwyblas_int* lda,
                        double* b, const hwyblas_int* ldb);
HWYBLAS_API void ctrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const float* alpha, const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb);
/* C := alpha*A*B + beta*C (side L) or alpha*B*A + beta*C (side R), A
 * symmetric with only the uplo triangle read. Replace dsymm_ / ssymm_
 * (include/hwyblas/hwyblas.h:597, 591; src/level3.cc:369-375, 362-368). */
HWYBLAS_API void dsymm_(const char* side, const char* uplo, const hwyblas_int* m,
                        const hwyblas_int* n, const double* alpha, const double* a,
                        const hwyblas_int* lda, const double* b, const hwyblas_int* ldb,
                        const double* beta, double* c, const hwyblas_int* ldc);
HWYBLAS_API void ssymm_(const char* side, const char* uplo, const hwyblas_int* m,
                        const hwyblas_int* n, const float* alpha, const float* a,
                        const hwyblas_int* lda, const float* b, const hwyblas_int* ldb,
                        const float* beta, float* c, const hwyblas_int* ldc);
/* C := alpha*A*B**T + alpha*B*A**T + beta*C (trans N) or with A**T*B and
 * B**T*A, on the uplo triangle. Replace dsyr2k_ / ssyr2k_
 * (include/hwyblas/hwyblas.h:674, 668; src/level3.cc:463-469, 456-462). */
HWYBLAS_API void dsyr2k_(const char* uplo, const char* trans, const hwyblas_int* n,
                         const hwyblas_int* k, const double* alpha, const double* a,
                         const hwyblas_int* lda, const double* b, const hwyblas_int* ldb,
                         const double* beta, double* c, const hwyblas_int* ldc);
HWYBLAS_API void ssyr2k_(const char* uplo, const char* trans, const hwyblas_int* n,
                         const hwyblas_int* k, const float* alpha, const float* a,
                         const hwyblas_int* lda, const float* b, const hwyblas_int* ldb,
                         const float* beta, float* c, const hwyblas_int* ldc);
/* C := alpha*op(A)*op(B) + beta*C on the uplo triangle of the n x n C.
 * Replace dgemmtr_ / sgemmtr_ and the alias names dgemmt_ / sgemmt_
 * (include/hwyblas/hwyblas.h:717, 711, 743, 737; src/level3.cc:508-560). */
HWYBLAS_API void dgemmtr_(const char* uplo, const char* transa, const char* transb,
                          const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                          const double* a, const hwyblas_int* lda, const double* b,
                          const hwyblas_int* ldb, const double* beta, double* c,
                          const hwyblas_int* ldc);
HWYBLAS_API void sgemmtr_(const char* uplo, const char* transa, const char* transb,
                          const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                          const float* a, const hwyblas_int* lda, const float* b,
                          const hwyblas_int* ldb, const float* beta, float* c,
                          const hwyblas_int* ldc);
HWYBLAS_API void dgemmt_(const char* uplo, const char* transa, const char* transb,
                         const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                         const double* a, const hwyblas_int* lda, const double* b,
                         const hwyblas_int* ldb, const double* beta, double* c,
                         const hwyblas_int* ldc);
HWYBLAS_API void sgemmt_(const char* uplo, const char* transa, const char* transb,
                         const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                         const float* a, const hwyblas_int* lda, const float* b,
                         const hwyblas_int* ldb, const float* beta, float* c,
                         const hwyblas_int* ldc);
/* B := alpha*op(A)*B (side L) or alpha*B*op(A), A triangular (unit diagonal
 * not read when diag U). Replace dtrmm_ / strmm_ (include/hwyblas/hwyblas.h:769,
 * 764; src/level3.cc:587-592, 581-586). */
HWYBLAS_API void dtrmm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const double* alpha, const double* a, const hwyblas_int* lda,
                        double* b, const hwyblas_int* ldb);
HWYBLAS_API void strmm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const float* alpha, const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb);
/* 1-based index of the first element of largest |x| (0 if n < 1 or
 * incx <= 0). Replaces idamax_ (include/hwyblas/hwyblas.h:169,
 * src/level1.cc:895-897). */
HWYBLAS_API hwyblas_int idamax_(const hwyblas_int* n, const double* x,
                                const hwyblas_int* incx);

/* Prints " ** On entry to NAME parameter number I had an illegal value" and
 * returns (does not stop the program). Replaces xerbla_
 * (include/hwyblas/hwyblas.h:888, src/common.cc:68-79). */
HWYBLAS_API void xerbla_(const char* srname, const hwyblas_int* info,
                         size_t srname_len);

/* Error handler called instead of xerbla_/cblas_xerbla; returns the previous
 * one, NULL restores the default. Replaces hwyblas_set_error_handler
 * (include/hwyblas/hwyblas.h:895-903, src/common.cc:81-84). */
typedef void (*hwyblas_error_handler)(const char* name, hwyblas_int position);
HWYBLAS_API hwyblas_error_handler
hwyblas_set_error_handler(hwyblas_error_handler handler);

/* ------------------------------------------------------------------------ */
/* LAPACK                                                                   */

/* A = P*L*U, blocked right-looking with nb = 64 (include/hwyblas/lapack.h:93,
 * src/lapack/getrf.cc:216-280, 508-512). ipiv is 1-based and global; INFO is
 * the first exactly-zero pivot. Same pivots as the reference. */
HWYBLAS_API void dgetrf_(const hwyblas_int* m, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv,
                         hwyblas_int* info);
/* Recursive LU (include/hwyblas/lapack.h:105, src/lapack/getrf.cc:112-207). */
HWYBLAS_API void dgetrf2_(const hwyblas_int* m, const hwyblas_int* n,
                          double* a, const hwyblas_int* lda, hwyblas_int* ipiv,
                          hwyblas_int* info);
/* Row interchanges (include/hwyblas/lapack.h:120, src/lapack/getrf.cc:28-81). */
HWYBLAS_API void dlaswp_(const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, const hwyblas_int* k1,
                         const hwyblas_int* k2, const hwyblas_int* ipiv,
                         const hwyblas_int* incx);
/* Solve with the LU factors (include/hwyblas/lapack.h:139,
 * src/lapack/getrf.cc:287-339). */
HWYBLAS_API void dgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const double* a,
                         const hwyblas_int* lda, const hwyblas_int* ipiv,
                         double* b, const hwyblas_int* ldb, hwyblas_int* info);
/* LU and solve (include/hwyblas/lapack.h:158, src/lapack/getrf.cc:348-374). */
HWYBLAS_API void dgesv_(const hwyblas_int* n, const hwyblas_int* nrhs,
                        double* a, const hwyblas_int* lda, hwyblas_int* ipiv,
                        double* b, const hwyblas_int* ldb, hwyblas_int* info);
/* Single-precision LU family: the reference instantiates one template for
 * s and d (src/lapack/getrf.cc:507-546); same algorithms at float, chunks of
 * 384 in the GEMM chains (include/hwyblas/lapack.h:90, 102, 117, 135, 155). */
HWYBLAS_API void sgetrf_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv,
                         hwyblas_int* info);
HWYBLAS_API void sgetrf2_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* ipiv,
                          hwyblas_int* info);
HWYBLAS_API void slaswp_(const hwyblas_int* n, float* a, const hwyblas_int* lda,
                         const hwyblas_int* k1, const hwyblas_int* k2,
                         const hwyblas_int* ipiv, const hwyblas_int* incx);
HWYBLAS_API void sgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const float* a,
                         const hwyblas_int* lda, const hwyblas_int* ipiv,
                         float* b, const hwyblas_int* ldb, hwyblas_int* info);
HWYBLAS_API void sgesv_(const hwyblas_int* n, const hwyblas_int* nrhs, float* a,
                        const hwyblas_int* lda, hwyblas_int* ipiv, float* b,
                        const hwyblas_int* ldb, hwyblas_int* info);
/* Complex LU family (src/lapack/getrf.cc:548-549, the same templates at
 * c64 and c32): interleaved (re, im) arrays, leading dimensions in complex
 * elements. Pivots are the first largest |re| + |im|; 1/pivot and the tiny-
 * pivot quotient are the C++ runtime's complex division. */
HWYBLAS_API void zgetrf_(const hwyblas_int* m, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info);
HWYBLAS_API void zgetrf2_(const hwyblas_int* m, const hwyblas_int* n, double* a,
                          const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info);
HWYBLAS_API void zlaswp_(const hwyblas_int* n, double* a, const hwyblas_int* lda,
                         const hwyblas_int* k1, const hwyblas_int* k2,
                         const hwyblas_int* ipiv, const hwyblas_int* incx);
HWYBLAS_API void zgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const double* a, const hwyblas_int* lda,
                         const hwyblas_int* ipiv, double* b, const hwyblas_int* ldb,
                         hwyblas_int* info);
HWYBLAS_API void zgesv_(const hwyblas_int* n, const hwyblas_int* nrhs, double* a,
                        const hwyblas_int* lda, hwyblas_int* ipiv, double* b,
                        const hwyblas_int* ldb, hwyblas_int* info);
HWYBLAS_API void cgetrf_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info);
HWYBLAS_API void cgetrf2_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info);
HWYBLAS_API void claswp_(const hwyblas_int* n, float* a, const hwyblas_int* lda,
                         const hwyblas_int* k1, const hwyblas_int* k2,
                         const hwyblas_int* ipiv, const hwyblas_int* incx);
HWYBLAS_API void cgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const float* a, const hwyblas_int* lda,
                         const hwyblas_int* ipiv, float* b, const hwyblas_int* ldb,
                         hwyblas_int* info);
HWYBLAS_API void cgesv_(const hwyblas_int* n, const hwyblas_int* nrhs, float* a,
                        const hwyblas_int* lda, hwyblas_int* ipiv, float* b,
                        const hwyblas_int* ldb, hwyblas_int* info);
/* Complex Cholesky family (src/lapack/potrf.cc:48-199, posv.cc:31-114 at
 * c64 and c32) and the complex HERK it updates with (src/level3.cc:85-140,
 * 439-452; alpha and beta real, the diagonal of C kept real). */
HWYBLAS_API void zpotrf_(const char* uplo, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void zpotrf2_(const char* uplo, const hwyblas_int* n, double* a,
                          const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void zpotrs_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const double* a, const hwyblas_int* lda, double* b,
                         const hwyblas_int* ldb, hwyblas_int* info);
HWYBLAS_API void zposv_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                        double* a, const hwyblas_int* lda, double* b, const hwyblas_int* ldb,
                        hwyblas_int* info);
HWYBLAS_API void zherk_(const char* uplo, const char* trans, const hwyblas_int* n,
                        const hwyblas_int* k, const double* alpha, const double* a,
                        const hwyblas_int* lda, const double* beta, double* c,
                        const hwyblas_int* ldc);
HWYBLAS_API void cpotrf_(const char* uplo, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void cpotrf2_(const char* uplo, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void cpotrs_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const float* a, const hwyblas_int* lda, float* b,
                         const hwyblas_int* ldb, hwyblas_int* info);
HWYBLAS_API void cposv_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                        float* a, const hwyblas_int* lda, float* b, const hwyblas_int* ldb,
                        hwyblas_int* info);
HWYBLAS_API void cherk_(const char* uplo, const char* trans, const hwyblas_int* n,
                        const hwyblas_int* k, const float* alpha, const float* a,
                        const hwyblas_int* lda, const float* beta, float* c,
                        const hwyblas_int* ldc);
/* Inverse from the LU factorization: inv(U) by ?trtri, then inv(A) L =
 * inv(U) in block columns of 64 (lwork >= 64 n; narrower blocks for a
 * smaller lwork, column by column below 2 n), then the column interchanges.
 * WORK(1) returns 64 n (query, lwork = -1) or the size used. info > 0:
 * U(info, info) is exactly zero. Replace dgetri_ / sgetri_
 * (include/hwyblas/lapack.h:174, 171; src/lapack/getrf.cc:369-483, 538-544). */
HWYBLAS_API void dgetri_(const hwyblas_int* n, double* a, const hwyblas_int* lda,
                         const hwyblas_int* ipiv, double* work, const hwyblas_int* lwork,
                         hwyblas_int* info);
HWYBLAS_API void sgetri_(const hwyblas_int* n, float* a, const hwyblas_int* lda,
                         const hwyblas_int* ipiv, float* work, const hwyblas_int* lwork,
                         hwyblas_int* info);
/* Iterative refinement of X for op(A) X = B with the LU factors AF, IPIV
 * (at most 5 steps while the componentwise backward error BERR halves and
 * exceeds eps), then forward error bounds FERR by the LACN2 estimate;
 * WORK holds 3 n, IWORK n. Replace dgerfs_ / sgerfs_
 * (include/hwyblas/lapack.h:465, 458; src/lapack/gesvx.cc:319-456, 796-806). */
HWYBLAS_API void dgerfs_(const char* trans, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const double* a, const hwyblas_int* lda, const double* af,
                         const hwyblas_int* ldaf, const hwyblas_int* ipiv, const double* b,
                         const hwyblas_int* ldb, double* x, const hwyblas_int* ldx,
                         double* ferr, double* berr, double* work, hwyblas_int* iwork,
                         hwyblas_int* info);
HWYBLAS_API void sgerfs_(const char* trans, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const float* a, const hwyblas_int* lda, const float* af,
                         const hwyblas_int* ldaf, const hwyblas_int* ipiv, const float* b,
                         const hwyblas_int* ldb, float* x, const hwyblas_int* ldx,
                         float* ferr, float* berr, float* work, hwyblas_int* iwork,
                         hwyblas_int* info);
/* Inverse of a triangular matrix in place (unit diagonal not read when
 * diag = 'U'): ?trtri blocked (64), ?trti2 unblocked. ?trtri: info > 0 when
 * A(info, info) is exactly zero (A unchanged). Replace dtrtri_ / strtri_ /
 * dtrti2_ / strti2_ (include/hwyblas/lapack.h:288, 285, 276, 273;
 * src/lapack/triangular.cc:18-166, 1645-1659). */
HWYBLAS_API void dtrtri_(const char* uplo, const char* diag, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void strtri_(const char* uplo, const char* diag, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void dtrti2_(const char* uplo, const char* diag, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void strti2_(const char* uplo, const char* diag, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* info);
/* Cholesky, blocked with nb = 64 (include/hwyblas/lapack.h:663,
 * src/lapack/potrf.cc:128-199, 747-751). */
HWYBLAS_API void dpotrf_(const char* uplo, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* info);
/* Recursive Cholesky (include/hwyblas/lapack.h:671,
 * src/lapack/potrf.cc:48-119). */
HWYBLAS_API void dpotrf2_(const char* uplo, const hwyblas_int* n, double* a,
                          const hwyblas_int* lda, hwyblas_int* info);
/* Solve with the Cholesky factor (include/hwyblas/lapack.h:726,
 * src/lapack/posv.cc:31-76). */
HWYBLAS_API void dpotrs_(const char* uplo, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const double* a,
                         const hwyblas_int* lda, double* b,
                         const hwyblas_int* ldb, hwyblas_int* info);
/* Cholesky and solve (include/hwyblas/lapack.h:746, src/lapack/posv.cc:78-114). */
HWYBLAS_API void dposv_(const char* uplo, const hwyblas_int* n,
                        const hwyblas_int* nrhs, double* a,
                        const hwyblas_int* lda, double* b,
                        const hwyblas_int* ldb, hwyblas_int* info);

/* Single-precision Cholesky family: one template for s and d in the
 * reference (src/lapack/potrf.cc:747-773, posv.cc; include/hwyblas/lapack.h:
 * 661, 669, 722, 742); same algorithms at float. */
HWYBLAS_API void spotrf_(const char* uplo, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void spotrf2_(const char* uplo, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* info);
HWYBLAS_API void spotrs_(const char* uplo, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const float* a,
                         const hwyblas_int* lda, float* b,
                         const hwyblas_int* ldb, hwyblas_int* info);
HWYBLAS_API void sposv_(const char* uplo, const hwyblas_int* n,
                        const hwyblas_int* nrhs, float* a,
                        const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb, hwyblas_int* info);

/* ------------------------------------------------------------------------ */
/* LAPACKE (include/hwyblas/lapacke.h:35-106, 114-149, 206-260, 624-720;
 * src/lapack/lapacke.cc:37-137, lapacke_linear.cc:22-73,
 * lapacke_symmetric.cc:22-72, lapacke_util.h:418-480). LAPACKE_xyyzzz checks
 * the layout (LAPACKE_xerbla(name, -1)), then, unless switched off
 * (LAPACKE_set_nancheck or LAPACKE_NANCHECK=0), returns -i if input argument
 * i holds a NaN, then calls LAPACKE_xyyzzz_work. The _work function calls
 * the LAPACK routine directly for column-major arrays (INFO < 0 shifted by
 * one for the layout argument); for row-major arrays it checks that each
 * leading dimension covers the columns (else LAPACKE_xerbla and -i),
 * transposes into column-major temporaries (host or device, where the
 * caller's array lives), calls the routine and transposes the outputs
 * back. Results are bit-identical to the column-major routine on the
 * transposed data. */
#define lapack_int hwyblas_int
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#define LAPACK_WORK_MEMORY_ERROR -1010
#define LAPACK_TRANSPOSE_MEMORY_ERROR -1011

/* Prints "Wrong parameter i in NAME" (or the out-of-memory message). */
HWYBLAS_API void LAPACKE_xerbla(const char* name, lapack_int info);
HWYBLAS_API void LAPACKE_set_nancheck(int flag);
HWYBLAS_API int LAPACKE_get_nancheck(void);

HWYBLAS_API lapack_int LAPACKE_dgetrf(int matrix_layout, lapack_int m, lapack_int n,
                                      double* a, lapack_int lda, lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_dgetrf_work(int matrix_layout, lapack_int m,
                                           lapack_int n, double* a, lapack_int lda,
                                           lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_dgetrf2(int matrix_layout, lapack_int m, lapack_int n,
                                       double* a, lapack_int lda, lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_dgetrf2_work(int matrix_layout, lapack_int m,
                                            lapack_int n, double* a, lapack_int lda,
                                            lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_dgetrs(int matrix_layout, char trans, lapack_int n,
                                      lapack_int nrhs, const double* a, lapack_int lda,
                                      const lapack_int* ipiv, double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dgetrs_work(int matrix_layout, char trans, lapack_int n,
                                           lapack_int nrhs, const double* a,
                                           lapack_int lda, const lapack_int* ipiv,
                                           double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dgesv(int matrix_layout, lapack_int n, lapack_int nrhs,
                                     double* a, lapack_int lda, lapack_int* ipiv,
                                     double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dgesv_work(int matrix_layout, lapack_int n,
                                          lapack_int nrhs, double* a, lapack_int lda,
                                          lapack_int* ipiv, double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sgetrf(int matrix_layout, lapack_int m, lapack_int n,
                                      float* a, lapack_int lda, lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_sgetrf_work(int matrix_layout, lapack_int m,
                                           lapack_int n, float* a, lapack_int lda,
                                           lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_sgetrf2(int matrix_layout, lapack_int m, lapack_int n,
                                       float* a, lapack_int lda, lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_sgetrf2_work(int matrix_layout, lapack_int m,
                                            lapack_int n, float* a, lapack_int lda,
                                            lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_sgetrs(int matrix_layout, char trans, lapack_int n,
                                      lapack_int nrhs, const float* a, lapack_int lda,
                                      const lapack_int* ipiv, float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sgetrs_work(int matrix_layout, char trans, lapack_int n,
                                           lapack_int nrhs, const float* a,
                                           lapack_int lda, const lapack_int* ipiv,
                                           float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sgesv(int matrix_layout, lapack_int n, lapack_int nrhs,
                                     float* a, lapack_int lda, lapack_int* ipiv,
                                     float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sgesv_work(int matrix_layout, lapack_int n,
                                          lapack_int nrhs, float* a, lapack_int lda,
                                          lapack_int* ipiv, float* b, lapack_int ldb);
/* LAPACKE forms of ?getri and ?trtri (include/hwyblas/lapacke.h:269-287,
 * 478-500; src/lapack/lapacke_linear.cc:75-96, 276-298, 500-548): row-major
 * through a transposed temporary; LAPACKE_?getri allocates the workspace
 * after a query. */
HWYBLAS_API lapack_int LAPACKE_dgetri(int matrix_layout, lapack_int n, double* a,
                                      lapack_int lda, const lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_sgetri(int matrix_layout, lapack_int n, float* a,
                                      lapack_int lda, const lapack_int* ipiv);
HWYBLAS_API lapack_int LAPACKE_dgetri_work(int matrix_layout, lapack_int n, double* a,
                                           lapack_int lda, const lapack_int* ipiv,
                                           double* work, lapack_int lwork);
HWYBLAS_API lapack_int LAPACKE_sgetri_work(int matrix_layout, lapack_int n, float* a,
                                           lapack_int lda, const lapack_int* ipiv,
                                           float* work, lapack_int lwork);
HWYBLAS_API lapack_int LAPACKE_dtrtri(int matrix_layout, char uplo, char diag, lapack_int n,
                                      double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_strtri(int matrix_layout, char uplo, char diag, lapack_int n,
                                      float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dtrtri_work(int matrix_layout, char uplo, char diag,
                                           lapack_int n, double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_strtri_work(int matrix_layout, char uplo, char diag,
                                           lapack_int n, float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dpotrf(int matrix_layout, char uplo, lapack_int n,
                                      double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dpotrf_work(int matrix_layout, char uplo, lapack_int n,
                                           double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dpotrf2(int matrix_layout, char uplo, lapack_int n,
                                       double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dpotrf2_work(int matrix_layout, char uplo, lapack_int n,
                                            double* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_dpotrs(int matrix_layout, char uplo, lapack_int n,
                                      lapack_int nrhs, const double* a, lapack_int lda,
                                      double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dpotrs_work(int matrix_layout, char uplo, lapack_int n,
                                           lapack_int nrhs, const double* a,
                                           lapack_int lda, double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dposv(int matrix_layout, char uplo, lapack_int n,
                                     lapack_int nrhs, double* a, lapack_int lda,
                                     double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_dposv_work(int matrix_layout, char uplo, lapack_int n,
                                          lapack_int nrhs, double* a, lapack_int lda,
                                          double* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_spotrf(int matrix_layout, char uplo, lapack_int n,
                                      float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_spotrf_work(int matrix_layout, char uplo, lapack_int n,
                                           float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_spotrf2(int matrix_layout, char uplo, lapack_int n,
                                       float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_spotrf2_work(int matrix_layout, char uplo, lapack_int n,
                                            float* a, lapack_int lda);
HWYBLAS_API lapack_int LAPACKE_spotrs(int matrix_layout, char uplo, lapack_int n,
                                      lapack_int nrhs, const float* a, lapack_int lda,
                                      float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_spotrs_work(int matrix_layout, char uplo, lapack_int n,
                                           lapack_int nrhs, const float* a,
                                           lapack_int lda, float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sposv(int matrix_layout, char uplo, lapack_int n,
                                     lapack_int nrhs, float* a, lapack_int lda,
                                     float* b, lapack_int ldb);
HWYBLAS_API lapack_int LAPACKE_sposv_work(int matrix_layout, char uplo, lapack_int n,
                                          lapack_int nrhs, float* a, lapack_int lda,
                                          float* b, lapack_int ldb);

/* ------------------------------------------------------------------------ */
/* CBLAS (include/hwyblas/cblas.h:20-45)                                    */

#define CBLAS_INDEX size_t
typedef enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum CBLAS_TRANSPOSE {
  CblasNoTrans = 111,
  CblasTrans = 112,
  CblasConjTrans = 113,
  CblasConjNoTrans = 114
} CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

/* Replaces cblas_xerbla (include/hwyblas/cblas.h:45). */
HWYBLAS_API void cblas_xerbla(hwyblas_int p, const char* rout, const char* form,
                              ...);
/* Row-major as the column-major product with A and B swapped
 * (include/hwyblas/cblas.h:615, src/cblas.cc:517-537, 1596). */
HWYBLAS_API void cblas_dgemm(const CBLAS_LAYOUT layout,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k,
                             const double alpha, const double* a,
                             const hwyblas_int lda, const double* b,
                             const hwyblas_int ldb, const double beta,
                             double* c, const hwyblas_int ldc);
/* include/hwyblas/cblas.h:607, src/cblas.cc:1585. */
HWYBLAS_API void cblas_sgemm(const CBLAS_LAYOUT layout,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k,
                             const float alpha, const float* a,
                             const hwyblas_int lda, const float* b,
                             const hwyblas_int ldb, const float beta, float* c,
                             const hwyblas_int ldc);
/* Row-major: other side and triangle (include/hwyblas/cblas.h:865,
 * src/cblas.cc:661-691, 1960). */
HWYBLAS_API void cblas_dtrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m,
                             const hwyblas_int n, const double alpha,
                             const double* a, const hwyblas_int lda, double* b,
                             const hwyblas_int ldb);
/* Single precision (include/hwyblas/cblas.h:858, src/cblas.cc:1950). */
HWYBLAS_API void cblas_strsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m,
                             const hwyblas_int n, const float alpha,
                             const float* a, const hwyblas_int lda, float* b,
                             const hwyblas_int ldb);
/* CBLAS forms of the level-3 routines above, both layouts, CBLAS argument
 * positions in error reports (include/hwyblas/cblas.h:835, 828 trmm; 714, 708
 * symm; 791, 784 syr2k; 649, 641 gemmtr; 683, 675 gemmt; src/cblas.cc:
 * 1631-1700, 1727-1746, 1842-1861, 1908-1927). */
/* CBLAS complex GEMM, alpha and beta by address (include/hwyblas/cblas.h:631,
 * 623; src/cblas.cc:520-537). */
/* CBLAS complex TRSM, alpha by address (include/hwyblas/cblas.h:879, 872;
 * src/cblas.cc:666-700, 1970-1990). */
HWYBLAS_API void cblas_ztrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const void* alpha, const void* a, const hwyblas_int lda, void* b,
                             const hwyblas_int ldb);
HWYBLAS_API void cblas_ctrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const void* alpha, const void* a, const hwyblas_int lda, void* b,
                             const hwyblas_int ldb);
/* CBLAS complex HERK (src/cblas.cc:1825-1841): row-major flips the triangle
 * and swaps N and C. */
HWYBLAS_API void cblas_zherk(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                             hwyblas_int n, hwyblas_int k, double alpha, const void* a,
                             hwyblas_int lda, double beta, void* c, hwyblas_int ldc);
HWYBLAS_API void cblas_cherk(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                             hwyblas_int n, hwyblas_int k, float alpha, const void* a,
                             hwyblas_int lda, float beta, void* c, hwyblas_int ldc);
HWYBLAS_API void cblas_zgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k, const void* alpha,
                             const void* a, const hwyblas_int lda, const void* b,
                             const hwyblas_int ldb, const void* beta, void* c,
                             const hwyblas_int ldc);
HWYBLAS_API void cblas_cgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k, const void* alpha,
                             const void* a, const hwyblas_int lda, const void* b,
                             const hwyblas_int ldb, const void* beta, void* c,
                             const hwyblas_int ldc);
HWYBLAS_API void cblas_dtrmm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const double alpha, const double* a, const hwyblas_int lda,
                             double* b, const hwyblas_int ldb);
HWYBLAS_API void cblas_strmm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const float alpha, const float* a, const hwyblas_int lda,
                             float* b, const hwyblas_int ldb);
HWYBLAS_API void cblas_dsymm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const hwyblas_int m, const hwyblas_int n,
                             const double alpha, const double* a, const hwyblas_int lda,
                             const double* b, const hwyblas_int ldb, const double beta,
                             double* c, const hwyblas_int ldc);
HWYBLAS_API void cblas_ssymm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const hwyblas_int m, const hwyblas_int n,
                             const float alpha, const float* a, const hwyblas_int lda,
                             const float* b, const hwyblas_int ldb, const float beta,
                             float* c, const hwyblas_int ldc);
HWYBLAS_API void cblas_dsyr2k(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                              const CBLAS_TRANSPOSE trans, const hwyblas_int n,
                              const hwyblas_int k, const double alpha, const double* a,
                              const hwyblas_int lda, const double* b, const hwyblas_int ldb,
                              const double beta, double* c, const hwyblas_int ldc);
HWYBLAS_API void cblas_ssyr2k(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                              const CBLAS_TRANSPOSE trans, const hwyblas_int n,
                              const hwyblas_int k, const float alpha, const float* a,
                              const hwyblas_int lda, const float* b, const hwyblas_int ldb,
                              const float beta, float* c, const hwyblas_int ldc);
HWYBLAS_API void cblas_dgemmtr(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                               const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                               const hwyblas_int n, const hwyblas_int k, const double alpha,
                               const double* a, const hwyblas_int lda, const double* b,
                               const hwyblas_int ldb, const double beta, double* c,
                               const hwyblas_int ldc);
HWYBLAS_API void cblas_sgemmtr(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                               const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                               const hwyblas_int n, const hwyblas_int k, const float alpha,
                               const float* a, const hwyblas_int lda, const float* b,
                               const hwyblas_int ldb, const float beta, float* c,
                               const hwyblas_int ldc);
HWYBLAS_API void cblas_dgemmt(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                              const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                              const hwyblas_int n, const hwyblas_int k, const double alpha,
                              const double* a, const hwyblas_int lda, const double* b,
                              const hwyblas_int ldb, const double beta, double* c,
                              const hwyblas_int ldc);
HWYBLAS_API void cblas_sgemmt(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo,
                              const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                              const hwyblas_int n, const hwyblas_int k, const float alpha,
                              const float* a, const hwyblas_int lda, const float* b,
                              const hwyblas_int ldb, const float beta, float* c,
                              const hwyblas_int ldc);
/* 0-based (include/hwyblas/cblas.h:128, src/cblas.cc:845). */
HWYBLAS_API CBLAS_INDEX cblas_idamax(const hwyblas_int n, const double* x,
                                     const hwyblas_int incx);

/* ------------------------------------------------------------------------ */
/* Extensions (hwyblas_ prefix, as the reference's own additions)           */

/* FP64-accurate GEMM on the INT8 tensor cores (Ozaki scheme): each row of
 * op(A) and column of op(B) is scaled by a power of two and cut into `slices`
 * 8-bit integer slices (1..8), the slice products with index sum below
 * `slices` run as exact INT32 tensor-core GEMMs, and the levels are
 * recombined in FP64 with compensated summation. slices = 0 chooses the
 * count from the inputs: the smallest whose estimated normwise error, given
 * the exponent spread of the rows of op(A) and columns of op(B) and K, is at
 * most half the plain FP64 path's (7 for uniform data, 8 for spreads of
 * several binades), or the plain path when no count up to 8 is. Arguments
 * and errors as dgemm_ (position 14: slices). Returns the slice count used
 * (0: the plain FP64 path ran: non-finite inputs, or slices = 0 and a spread
 * too wide for 8 slices; -1: error). No counterpart in the reference. */
HWYBLAS_API hwyblas_int hwyblas_dgemm_emulated(
    const char* transa, const char* transb, const hwyblas_int* m,
    const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
    const double* a, const hwyblas_int* lda, const double* b,
    const hwyblas_int* ldb, const double* beta, double* c,
    const hwyblas_int* ldc, const hwyblas_int* slices);
/* out(:, jj) = op(A) * op(B)(:, cols[jj] - 0) for jj < ncols (0-based column
 * indices into the n columns of op(B)), accumulated in double-double and
 * rounded once: the higher-precision reference against which the error of
 * every FP64 path is stated. No counterpart in the reference. */
HWYBLAS_API void hwyblas_dgemm_ddref(const char* transa, const char* transb,
                                     const hwyblas_int* m,
                                     const hwyblas_int* ncols,
                                     const hwyblas_int* k, const double* a,
                                     const hwyblas_int* lda, const double* b,
                                     const hwyblas_int* ldb,
                                     const hwyblas_int* n,
                                     const hwyblas_int* cols, double* out,
                                     const hwyblas_int* ldo);
/* R = B - A X (A n x n; X, B, R n x nrhs; column-major) with extra
 * precision: every product is split exactly into its rounded value and
 * error, the products are summed in double-double and each entry is rounded
 * once, so its error is about n eps^2 |A| |X| rather than n eps |A| |X|. The
 * residual of the mixed solvers' refinement, and the yardstick against which
 * the solvers' forward errors are stated. Invalid arguments are reported
 * with their positions (1, 2, 4, 6, 8, 10). No counterpart in the
 * reference. */
HWYBLAS_API void hwyblas_dresidual_dd(const hwyblas_int* n, const hwyblas_int* nrhs,
                                      const double* a, const hwyblas_int* lda,
                                      const double* x, const hwyblas_int* ldx,
                                      const double* b, const hwyblas_int* ldb, double* r,
                                      const hwyblas_int* ldr);

/* Mixed-precision solve of A X = B (LAPACK DSGESV semantics; the reference
 * has no mixed-precision solver, README.md:81). The LU's trailing updates run
 * as INT8-slice GEMMs on the tensor cores (hwyblas_set_mixed_slices slices,
 * default 4), the panels (pivot search, diagonal block) in FP64; X is then
 * refined in FP64 until every column meets ||r||_inf <= ||x||_inf ||A||_inf
 * eps sqrt(n) and its last correction is below 2^-52 ||x||_inf or stopped
 * halving. ITER >= 0: refinement steps taken, A unchanged, IPIV from
 * the mixed factorization. ITER < 0: the FP64 path ran (-2 non-finite A, -3
 * breakdown, -31 no convergence in 30 steps), A holds its LU factors and
 * IPIV its pivots (src/lapack/getrf.cc:217-280 order). INFO as dgesv_. */
HWYBLAS_API void hwyblas_dgesv_mixed(const hwyblas_int* n, const hwyblas_int* nrhs,
                                     double* a, const hwyblas_int* lda,
                                     hwyblas_int* ipiv, const double* b,
                                     const hwyblas_int* ldb, double* x,
                                     const hwyblas_int* ldx, hwyblas_int* iter,
                                     hwyblas_int* info);
/* Mixed-precision Cholesky solve (LAPACK DSPOSV semantics), as
 * hwyblas_dgesv_mixed with a Cholesky factorization; on ITER < 0, A holds
 * the FP64 factor of src/lapack/potrf.cc:121-199. */
HWYBLAS_API void hwyblas_dposv_mixed(const char* uplo, const hwyblas_int* n,
                                     const hwyblas_int* nrhs, double* a,
                                     const hwyblas_int* lda, const double* b,
                                     const hwyblas_int* ldb, double* x,
                                     const hwyblas_int* ldx, hwyblas_int* iter,
                                     hwyblas_int* info);
/* Slice count (1..8) of the mixed solvers' trailing updates for the calling
 * thread; returns the previous value (other values only query). Like the
 * reference's hwyblas_set_ilaenv (lapack.h:74-80), a tuning knob. */
HWYBLAS_API int hwyblas_set_mixed_slices(int slices);

/* Test hook of the batched routines: forces the launch configuration that
 * the autotuner would otherwise choose per routine, type and size bucket
 * (64, 128 or 256 threads per CTA of the register-tiled FMA kernels; 1128,
 * 128 threads with six CTAs an SM, for the LU, solve and TRSM; in FP64 also
 * 1001 and 1002, whose products run on the tensor pipe in 32 x 32 and
 * 64 x 64 tiles).
 * A configuration that the routine does not have is ignored; 0 restores the
 * autotuner. Results do not depend on the configuration. Returns the
 * previous setting. No counterpart in the reference. */
HWYBLAS_API int hwyblas_batched_set_config(int config);

/* Batched LU, LU solve and GEMM over `count` independent problems of
 * uneven sizes (no counterpart in the reference, which solves one problem a
 * call). Arrays of sizes, leading dimensions and INFO are host memory; the
 * matrices and pivot vectors are device memory (each array entry a device
 * pointer, checked to lie inside one device allocation). One persistent
 * launch per call: CTAs take problems largest first; threads per CTA come
 * from an autotuner (per routine, type and size bucket, measured once per
 * process). Every problem's result is bit-identical to the single-problem
 * routine (dgetrf_, dgetrs_, dtrsm_, dgemm_ and their single-precision forms).
 * Errors
 * are reported through the error handler with the position of the offending
 * argument (any problem). Synchronous on return. */
HWYBLAS_API void hwyblas_dgetrf_batched(const hwyblas_int* n, double* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        hwyblas_int* info, hwyblas_int count);
HWYBLAS_API void hwyblas_sgetrf_batched(const hwyblas_int* n, float* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        hwyblas_int* info, hwyblas_int count);
HWYBLAS_API void hwyblas_dgetrs_batched(char trans, const hwyblas_int* n,
                                        const hwyblas_int* nrhs, double* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        double* const* b, const hwyblas_int* ldb,
                                        hwyblas_int count, hwyblas_int* info);
HWYBLAS_API void hwyblas_sgetrs_batched(char trans, const hwyblas_int* n,
                                        const hwyblas_int* nrhs, float* const* a,
                                        const hwyblas_int* lda, hwyblas_int* const* ipiv,
                                        float* const* b, const hwyblas_int* ldb,
                                        hwyblas_int count, hwyblas_int* info);
HWYBLAS_API void hwyblas_dtrsm_batched(char side, char uplo, char transa, char diag,
                                       const hwyblas_int* m, const hwyblas_int* n,
                                       double alpha, double* const* a,
                                       const hwyblas_int* lda, double* const* b,
                                       const hwyblas_int* ldb, hwyblas_int count);
HWYBLAS_API void hwyblas_strsm_batched(char side, char uplo, char transa, char diag,
                                       const hwyblas_int* m, const hwyblas_int* n,
                                       float alpha, float* const* a,
                                       const hwyblas_int* lda, float* const* b,
                                       const hwyblas_int* ldb, hwyblas_int count);
HWYBLAS_API void hwyblas_dgemm_batched(char transa, char transb, const hwyblas_int* m,
                                       const hwyblas_int* n, const hwyblas_int* k,
                                       double alpha, double* const* a,
                                       const hwyblas_int* lda, double* const* b,
                                       const hwyblas_int* ldb, double beta,
                                       double* const* c, const hwyblas_int* ldc,
                                       hwyblas_int count);
HWYBLAS_API void hwyblas_sgemm_batched(char transa, char transb, const hwyblas_int* m,
                                       const hwyblas_int* n, const hwyblas_int* k,
                                       float alpha, float* const* a,
                                       const hwyblas_int* lda, float* const* b,
                                       const hwyblas_int* ldb, float beta,
                                       float* const* c, const hwyblas_int* ldc,
                                       hwyblas_int count);

/* Stream for subsequent calls of the calling thread (a cudaStream_t; NULL
 * restores the library's per-thread stream). No counterpart in the
 * reference, which has no device. */
HWYBLAS_API void hwyblas_set_stream(void* stream);
/* Last CUDA error seen by the library on the calling thread (cudaError_t as
 * int; 0 if none), cleared by the read. No counterpart in the reference. */
HWYBLAS_API int hwyblas_last_cuda_error(void);
/* Number of kernels the library has launched (all threads). No counterpart
 * in the reference; used to count launches inside timed regions. */
HWYBLAS_API uint64_t hwyblas_launch_count(void);
/* Kernel timer (instrumentation, no counterpart in the reference): while
 * family f is selected (1 FP64 DMMA GEMM kernel, 2 emulated-GEMM slice-product
 * kernel, 3 LU leaf kernel; 0 none), each launch of that kernel is bracketed
 * by CUDA events on its stream. hwyblas_kernel_timer_read waits for them and
 * returns the summed milliseconds (and the launch count), then forgets them. */
HWYBLAS_API void hwyblas_kernel_timer(int family);
HWYBLAS_API double hwyblas_kernel_timer_read(int* launches);
/* Measured FP64 tensor-pipe throughput of the current device (TFLOP/s), from
 * a DMMA issue-rate loop; the FP64 roofline denominator. No counterpart in
 * the reference. */
HWYBLAS_API double hwyblas_fp64_peak_tflops(void);
/* Measured INT8 throughput of the current device's 5th-generation tensor
 * cores (TOPS), from a tcgen05.mma kind::i8 issue loop on every SM; the
 * roofline denominator of the emulated GEMM's slice products. No counterpart
 * in the reference. */
HWYBLAS_API double hwyblas_int8_peak_tops(void);
/* Test hook for the bounded waits: sets how many times each CTA of the LU
 * panel's cooperative pivot exchange (panels of more than 16 x 1024 rows)
 * polls for its peers before it gives up, sets the timeout status (reported
 * as cudaErrorLaunchTimeout by hwyblas_last_cuda_error) and returns; 0
 * restores the default of 2^26. Applies to the current device; returns the
 * previous limit. No counterpart in the reference. */
HWYBLAS_API unsigned int hwyblas_set_leaf_wait_limit(unsigned int polls);

/* IDAMAX that allocates no memory: for callers that must not allocate
 * device memory during a call (a cudaMalloc/cudaFree synchronizes the whole
 * device and stalls the caller's other streams; a caller that has given all
 * free device memory to its own pool has none to spare). No counterpart in
 * the reference; the index is the one idamax_ returns (src/level1.cc:383-402).
 *   x       device-accessible vector of n elements with stride incx
 *   result  device-accessible int that receives the 1-based index (0 when
 *           n < 1 or incx <= 0), stream-ordered: read it after `stream`
 *   stream  a cudaStream_t (NULL: the legacy default stream)
 * Returns 0 once the work is enqueued, -1 if n > 16,777,216 (the partial
 * results of the fixed 16 KB scratch array), -2 / -4 if x / result is not
 * accessible from the current device (each also reported through the error
 * handler as IDAMAX_NOALLOC), or a positive cudaError_t.
 * The scratch is a static array in the library's device code, one per
 * device. Every call looks its address up (this allocates nothing); the
 * first call that sees an address on a device (the first on that device,
 * or the first after its context was created again, as after
 * cudaDeviceReset) zeroes the array on `stream`: make that call before
 * capturing a stream. All calls on a device share the array: calls that
 * overlap in time (unordered streams, or several host threads at once) race
 * on it. */
HWYBLAS_API int hwyblas_idamax_noalloc(int n, const double* x, int incx,
                                       int* result, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HWYBLAS_B200_H_ */
