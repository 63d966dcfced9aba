// Internal interfaces of libhwyblas_b200: per-thread context (stream, device
// workspace, error state) and the device-level routines. Device-level
// routines take device pointers, column-major with leading dimensions, and
// only enqueue work on the context's stream; the C ABI (api.cc) validates
// arguments, stages host memory and synchronises.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <functional>
#include <cstdint>

namespace hb {

// Which part of C a product updates (the reference's Part, src/gemm.h:39).
enum Part : int { kAll = 0, kLower = 1, kUpper = 2 };
// A triangular GEMM operand (TRMM): op(A) or op(B) lower or upper. Products
// are restricted to the k range the reference multiplies for each of its
// micro-tiles (src/gemm-inl.h:62-85).
enum Tri : int { kTriNone = 0, kTriALower = 1, kTriAUpper = 2, kTriBLower = 3, kTriBUpper = 4 };

// A strided view of op(X): element (i, p) is data[i * rs + p * cs], with one
// of rs, cs equal to 1 (column-major storage, possibly transposed). This is
// the reference's Operand (src/gemm.h:28-36) for general matrices.
template <typename T>
struct View {
  const T* data = nullptr;
  long long rs = 1, cs = 1;
  View sub(long long i0, long long j0) const {
    View v = *this;
    v.data += i0 * rs + j0 * cs;
    return v;
  }
  bool trans() const { return rs != 1; }
  long long ld() const { return rs != 1 ? rs : cs; }
};
template <typename T>
inline View<T> ColMajor(const T* p, long long ld, bool trans = false) {
  View<T> v;
  v.data = p;
  v.rs = trans ? ld : 1;
  v.cs = trans ? 1 : ld;
  return v;
}

struct Context {
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  int device = -1;
  int num_sms = 148;
  // Device status words: [0] wait-timeout flag written by kernels whose
  // bounded waits gave up; [1] LAPACK INFO of the running driver; the rest
  // are grid-barrier counters and scratch ints.
  int* dev_status = nullptr;
  // If non-null, kernels return at once while *guard != 0 (used by drivers
  // that must stop after a failure, e.g. Cholesky's non-positive minor).
  const int* guard = nullptr;
  int last_error = 0;
  // Workspace bank of the work being enqueued: 0 on the context's stream, 1
  // on the side stream (see OnSide), so that the two streams never share a
  // scratch buffer.
  int ws_bank = 0;
  // If nonzero, the persistent FP64 GEMM launches at most this many CTAs,
  // leaving the other SMs to the side stream's work (look-ahead).
  int sm_cap = 0;
  // Set while the side stream factors panels beside a capped GEMM: the LU
  // leaf then takes its cooperative variant, whose CTAs can run on any free
  // SMs (a 16-CTA cluster needs 16 free SMs of one GPC).
  bool side_leaf = false;
};

// The calling thread's second stream (highest priority) with two events, for
// look-ahead: work that a later step needs first runs there while the
// context's stream does the bulk of the current step. ok is false if the
// stream could not be created (callers then stay on one stream).
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t to_side = nullptr, to_main = nullptr;
  bool ok = false;
};
SideStream& Side();

// The calling thread's context on the current device (created on first use).
Context& Ctx();
// Grows and returns slot `slot` of the thread's device workspace (at least
// `bytes`, 256-byte aligned). Valid until the next call with the same slot.
void* Workspace(int slot, size_t bytes);
enum WorkspaceSlot : int {
  kWsStageA = 0,   // host-pointer staging
  kWsStageB = 1,
  kWsStageC = 2,
  kWsPackA = 3,    // canonical (transposed / realigned) GEMM operands
  kWsPackB = 4,
  kWsLeaf = 5,     // LU panel exchange buffers
  kWsEmul = 6,     // emulated-GEMM slices
  kWsEmulAcc = 7,
  kWsMixed = 8,    // mixed-precision solver buffers
  kWsMixed2 = 9,
  kWsMixed3 = 10,
  kWsBatch = 11,
  kWsEmulW = 12,   // emulated-GEMM FP64 partial sums between passes
  kWsStageX = 13,  // host-pointer staging of a solver's solution
  kWsEmul2 = 14,   // emulated-GEMM buffers of a second, concurrent stream
  kWsEmulAcc2 = 15,
  kWsEmulW2 = 16,
  kWsTourney = 17, // tournament-pivoting leaf: candidates and results
  kWsLapacke0 = 18, // LAPACKE row-major temporaries (device callers)
  kWsLapacke1 = 19,
  kWsLevel3 = 20,      // SYMM's symmetrized operand, TRMM's triangle
  kWsLevel3Copy = 21,  // TRMM's copy of B
  kWsGetri = 22,       // GETRI's block column of L
  kWsTrti2 = 23,       // TRTI2's column between read and write
  kWsStageAF = 24,     // host-pointer staging of GERFS's factors
  kWsRefine = 25,      // GERFS vectors
  kWsRefineInt = 26,
  kWsGerfsWork = 27,   // host-pointer staging of GERFS's WORK and IWORK
  kWsGerfsIwork = 28,
  kWsSplitK = 29,      // per-chunk accumulators of a split DMMA GEMM
  kWsZFactor = 30,     // aligned copy of a complex matrix being factored
  kWsZFactorB = 31,    // aligned copy of the right-hand sides of its solve
  kWsResidual = 32,    // hwyblas_dresidual_dd partial sums
  kWsMixedInv = 33,    // mixed Cholesky: the inverse of a diagonal block
  kWsTrsmBarrier = 34, // cooperative TRSM: its grid barrier counter
  kNumWorkspaceSlots = 35
};

// Makes `to` wait for the work enqueued on `from` so far.
inline void StreamAfter(cudaEvent_t ev, cudaStream_t from, cudaStream_t to) {
  if (from == to) return;
  cudaEventRecord(ev, from);
  cudaStreamWaitEvent(to, ev, 0);
}

// Enqueues f's work on the side stream with the second workspace bank.
template <typename F>
void OnSide(F f) {
  Context& ctx = Ctx();
  SideStream& side = Side();
  const cudaStream_t saved = ctx.stream;
  const int bank = ctx.ws_bank;
  if (side.ok) {
    ctx.stream = side.stream;
    ctx.ws_bank = 1;
  }
  f();
  ctx.stream = saved;
  ctx.ws_bank = bank;
}

// Records a CUDA error on the context and prints it; returns true if `e` is
// an error.
bool Failed(cudaError_t e, const char* what);
// Checks the last launch.
bool LaunchFailed(const char* what);

extern std::atomic<uint64_t> g_launches;
inline void CountLaunch(uint64_t n = 1) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
}

// Kernel timer (instrumentation): when the timed family is enabled, the
// launch sites of that kernel family bracket each launch with CUDA events on
// their stream. KernelTimerStart returns the start event (nullptr when
// disabled); KernelTimerStop records the stop event and keeps the pair.
enum KernelFamily : int {
  kFamilyNone = 0,
  kFamilyDmmaGemm = 1,   // DgemmDmmaKernel
  kFamilyOzakiGemm = 2,  // OzakiGemmKernel (all passes)
  kFamilyLuLeaf = 3,     // GetrfLeafPanelKernel
};
cudaEvent_t KernelTimerStart(int family, cudaStream_t stream);
void KernelTimerStop(cudaEvent_t start, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Device-level routines (device pointers; stream-ordered on Ctx().stream).

// C := alpha*op(A)*op(B) + beta*C on `part` of C; requires m, n, k > 0 and
// alpha != 0. Bit-identical to the reference's GEMM (double: chunks of 256).
// `tri` names a triangular operand whose zero triangle (and unit diagonal) is
// stored explicitly; only the reference's per-micro-tile k ranges are
// multiplied, so every chain is the reference's.
void Dgemm(int m, int n, int k, double alpha, View<double> a, View<double> b,
           double beta, double* c, int ldc, Part part = kAll, Tri tri = kTriNone);
// Bytes of the partial sums Dgemm takes from kWsSplitK when it splits an
// m x n x k product over its KC chunks (0 when it does not split).
size_t DgemmSplitBytes(int m, int n, int k);
// FP32 (chunks of 384), FFMA on the CUDA cores.
void Sgemm(int m, int n, int k, float alpha, View<float> a, View<float> b,
           float beta, float* c, int ldc, Part part = kAll, Tri tri = kTriNone);
// C := beta*C on `part` (beta == 0 writes zeros without reading C).
template <typename T>
void ScaleMatrix(int m, int n, T beta, T* c, int ldc, Part part = kAll);
// Solves X*T = B (right) or T*X = B (left) for an r x r triangular op(A)
// `tri` (lower/unit as given for op(A)); B is r x other (left) or other x r.
template <typename T>
void TrsmSolve(bool left, View<T> tri, bool lower, bool unit, int r,
               int other, T* b, int ldb);
// Device IAMAX: writes the 1-based index to *out (device int).
template <typename T>
void Iamax(int n, const T* x, int incx, int* out);
// A complex element as its two parts, aligned as one part: row interchanges
// move it whole (Laswp<ZPair<R>>).
template <typename R>
struct ZPair {
  R re, im;
};
// Lanes of the reference's SIMD vectors of doubles (8 for AVX-512).
int RefLanesDouble();
// LASWP on device data; ipiv is a device array (1-based, Fortran k1/k2/incx).
template <typename T>
void Laswp(int n, T* a, int lda, int k1, int k2, const int* ipiv, int incx);
// ipiv[i] += delta for i in [begin, end) (device).
void AdjustPivots(int* ipiv, int begin, int end, int delta);
// GetrfLeaf on device: m x n, min(m, n) <= 16; ipiv (device, leaf-relative,
// 1-based); *info (device) set to info_base + j + 1 at the first zero pivot
// if it is still 0.
template <typename T>
void GetrfLeaf(int m, int n, T* a, int lda, int* ipiv, int* info, int info_base,
               int leaf_w = 16);
// Sets the poll limit of the cooperative leaf's exchange on the current
// device (0: the default); returns the previous one.
unsigned int SetLeafWaitLimit(unsigned int polls);
// PotrfLeaf on device: n <= 64; sets *info to info_base + j + 1 and stops at
// the first non-positive (or NaN) diagonal, if *info is still 0.
template <typename T>
void PotrfLeaf(bool upper, int n, T* a, int lda, int* info, int info_base);

// LAPACK drivers on device data (ipiv, info: device pointers).
template <typename T>
void Getrf(int m, int n, T* a, int lda, int* ipiv, int* info);
template <typename T>
void Getrf2(int m, int n, T* a, int lda, int* ipiv, int* info);
template <typename T>
void Getrs(bool trans, int n, int nrhs, const T* a, int lda, const int* ipiv,
           T* b, int ldb);
template <typename T>
void Potrf(bool upper, int n, T* a, int lda, int* info);
// Potrf2 of a block whose first column is global column col0 (for INFO);
// later kernels become no-ops after a failure.
void PotrfPanel(bool upper, int n, double* a, int lda, int* info, int col0);
// Pivoted LU of an m x nc panel (m >= nc) for the mixed solver (mixed_panel.cu):
// right-looking over leaf-wide sub-panels, not the reference's recursion;
// pivots relative to the panel's first row; *info set at the first zero pivot.
void MixedPanel(int m, int nc, double* a, int lda, int* ipiv, int* info, int col0);
// Lower Cholesky of an n x n diagonal block for the mixed solver
// (mixed_panel.cu): right-looking over 32-column sub-panels; the upper
// triangle is scratch; *info as PotrfPanel sets it; `arrivals` is one device
// word of scratch for this stream.
void CholBlock(int n, double* a, int lda, int* info, int col0, unsigned int* arrivals);
template <typename T>
void Potrf2(bool upper, int n, T* a, int lda, int* info);
template <typename T>
void Potrs(bool upper, int n, int nrhs, const T* a, int lda, T* b, int ldb);

// Level-3 with reference semantics (quick returns, alpha scaling).
template <typename T>
void TrsmFull(bool left, bool lower, bool trans, bool unit, int m, int n,
              T alpha, const T* a, int lda, T* b, int ldb);
template <typename T>
void SyrkFull(bool lower, bool trans, int n, int k, T alpha, const T* a, int lda, T beta,
              T* c, int ldc);
// SYMM, SYR2K, GEMMTR and TRMM (src/level3.cc:26-76, 153-342) after argument
// checks.
template <typename T>
void SymmFull(bool left, bool lower, int m, int n, T alpha, const T* a, int lda, const T* b,
              int ldb, T beta, T* c, int ldc);
template <typename T>
void Syr2kFull(bool lower, bool trans, int n, int k, T alpha, const T* a, int lda,
               const T* b, int ldb, T beta, T* c, int ldc);
// TRTI2, TRTRI and GETRI (src/lapack/triangular.cc:18-166,
// src/lapack/getrf.cc:369-483) after argument checks. TRTRI returns i > 0 for
// A(i, i) == 0 (non-unit; A untouched); GETRI returns its INFO and the WORK(1)
// value of a successful call in *iws.
template <typename T>
int Trti2Full(bool upper, bool unit, int n, T* a, int lda);
template <typename T>
int TrtriFull(bool upper, bool unit, int n, T* a, int lda);
template <typename T>
int GetriFull(int n, T* a, int lda, const int* ipiv, int lwork, int* iws);
// GERFS (src/lapack/gesvx.cc:319-456) after argument checks, n, nrhs > 0:
// device a, af, ipiv, b, x (refined in place), work (3n) and iwork (n) or
// null; host ferr and berr.
template <typename T>
void GerfsFull(bool trans, int n, int nrhs, const T* a, int lda, const T* af, int ldaf,
               const int* ipiv, const T* b, int ldb, T* x, int ldx, T* ferr, T* berr,
               T* work, int* iwork);
// Complex GEMM (src/gemm.cc:67-123) after argument checks: interleaved
// (re, im) arrays, leading dimensions in complex elements, op 0 N / 1 T / 2 C.
template <typename R>
void ZgemmFull(int ta, int tb, int m, int n, int k, const R* alpha, const R* a, int lda,
               const R* b, int ldb, const R* beta, R* c, int ldc);
// Complex TRSM (src/trsm.cc:137-180) after argument checks, op 0 N / 1 T / 2 C.
template <typename R>
void ZtrsmFull(bool left, bool lower, int op, bool unit, int m, int n, const R* alpha,
               const R* a, int lda, R* b, int ldb);
// Complex LU (src/lapack/getrf.cc:112-280) on device data with leading
// dimension lda in complex elements; ipiv and *info on the device (INFO as
// for Getrf). recursive: xGETRF2 instead of the blocked xGETRF.
template <typename R>
void ZGetrf(bool recursive, int m, int n, R* a, int lda, int* ipiv, int* info);
// Complex LU solve (src/lapack/getrf.cc:287-339), op 0 N / 1 T / 2 C.
template <typename R>
void ZGetrs(int op, int n, int nrhs, const R* a, int lda, const int* ipiv, R* b, int ldb);
// Complex HERK (src/level3.cc:85-140) on the triangle of C, op 0 N / 2 C,
// alpha and beta real.
template <typename R>
void ZherkFull(bool lower, int op, int n, int k, R alpha, const R* a, int lda, R beta, R* c,
               int ldc);
// Complex Cholesky (src/lapack/potrf.cc:48-199) on device data; *info on the
// device. recursive: xPOTRF2 instead of the blocked xPOTRF.
template <typename R>
void ZPotrf(bool recursive, bool upper, int n, R* a, int lda, int* info);
// Complex Cholesky solve (src/lapack/posv.cc:31-76).
template <typename R>
void ZPotrs(bool upper, int n, int nrhs, const R* a, int lda, R* b, int ldb);
// Complex LASWP on device data (src/lapack/getrf.cc:28-81).
template <typename R>
void ZLaswp(int n, R* a, int lda, int k1, int k2, const int* ipiv, int incx);
template <typename T>
void GemmtrFull(bool lower, bool ta, bool tb, int n, int k, T alpha, const T* a, int lda,
                const T* b, int ldb, T beta, T* c, int ldc);
template <typename T>
void TrmmFull(bool left, bool lower, bool trans, bool unit, int m, int n, T alpha,
              const T* a, int lda, T* b, int ldb);
// TRMM with the triangle already dense in tri (zeros outside it, ones on a
// unit diagonal), leading dimension ldt.
template <typename T>
void TrmmDense(bool left, bool lower, bool trans, int m, int n, T alpha, const T* tri, int ldt,
               T* b, int ldb);
template <typename T>
void GemmFull(bool ta, bool tb, int m, int n, int k, T alpha, const T* a,
              int lda, const T* b, int ldb, T beta, T* c, int ldc);

// FP64-accurate GEMM on INT8 tensor cores with `slices` slices (1..8);
// returns the slice count used, 0 if non-finite inputs sent it to Dgemm, -1
// on a CUDA error. check_finite = false skips that test and its host
// synchronization (callers whose inputs are known finite, or that detect a
// non-finite result themselves). ws_set 1 takes a second set of workspace
// slots, for a call that runs concurrently with another one on a second
// stream. lower_only: only C's lower triangle is wanted (tiles of C strictly
// above its diagonal are skipped; the diagonal tiles are computed whole).
// col_blocks > 1 with block_done (a full C and k within one chunk): the
// products run in that many column blocks of C and block_done(first column,
// columns) is called on the host as each block's launches are queued on the
// stream, e.g. to queue that block's copy to the host.
int DgemmEmulated(int m, int n, int k, double alpha, View<double> a,
                  View<double> b, double beta, double* c, int ldc, int slices,
                  bool check_finite = true, int ws_set = 0, bool lower_only = false,
                  int col_blocks = 1,
                  const std::function<void(int, int)>* block_done = nullptr);
int OzakiMaxK(int S);
// out(:, jj) = op(A) op(B)(:, cols[jj]) in double-double (error reference).
void DgemmDoubleDouble(int m, int ncols, int k, View<double> a, View<double> b,
                       const int* cols, double* out, int ldo);

// Host-side wait-timeout check: returns true (and reports) if any kernel on
// the context set the timeout flag since the last check. Synchronises.
bool CheckDeviceStatus(const char* what);

// r := b - A x (A n x n, x, b, r n x nrhs, device) with extra precision:
// double-double accumulation of exactly split products, rounded once. part:
// ResidualDdPartBytes(n, nrhs) bytes of device scratch.
void ResidualDd(int n, int nrhs, const double* a, long long lda, const double* b,
                long long ldb, const double* x, long long ldx, double* r, long long ldr,
                double* part);
size_t ResidualDdPartBytes(int n, int nrhs);

// Mixed-precision solvers (LAPACK DSGESV / DSPOSV semantics) on device data;
// the trailing updates of the factorization use `slices` INT8 slices. Return
// INFO (0; > 0 from the FP64 fallback's factorization; -1 on a CUDA error)
// and set *iter to DSGESV's ITER.
int DgesvMixed(int n, int nrhs, double* a, int lda, int* ipiv, const double* b,
               int ldb, double* x, int ldx, int slices, int* iter);
int DposvMixed(bool upper, int n, int nrhs, double* a, int lda, const double* b,
               int ldb, double* x, int ldx, int slices, int* iter);

// Reports an invalid argument through the error handler (default: xerbla_).
void ReportError(const char* routine, int info);

}  // namespace hb
