// The C ABI: the reference's Fortran BLAS/LAPACK and CBLAS entry points
// (argument checks with the reference's xerbla positions, quick returns),
// the per-thread CUDA context and device workspace, and the staging of host
// pointers. Every entry point is synchronous on return.
//
// Argument checks follow src/gemm.cc:73-110 (GEMM), src/trsm.cc:137-169
// (TRSM), src/level3.cc:84-124 (SYRK), src/level1.cc:383-402 (IAMAX),
// src/lapack/getrf.cc:112-131, 216-234, 287-309, 348-365 (GETRF2, GETRF,
// GETRS, GESV), src/lapack/potrf.cc:48-67, 128-147 and src/lapack/posv.cc:31-54
// (POTRF2, POTRF, POTRS, POSV); error reporting follows src/common.cc:25-84
// and the CBLAS position maps of src/cblas.cc:121-149, 517-537, 661-691.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/hwyblas_b200.h"
#include "internal.h"

namespace hb {

std::atomic<uint64_t> g_launches{0};

namespace {
std::mutex g_timer_mu;
int g_timer_family = kFamilyNone;
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_timer_events;
}  // namespace

cudaEvent_t KernelTimerStart(int family, cudaStream_t stream) {
  std::lock_guard<std::mutex> lock(g_timer_mu);
  if (family != g_timer_family || family == kFamilyNone) return nullptr;
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  cudaEventRecord(e, stream);
  return e;
}

void KernelTimerStop(cudaEvent_t start, cudaStream_t stream) {
  if (start == nullptr) return;
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, stream);
  std::lock_guard<std::mutex> lock(g_timer_mu);
  g_timer_events.emplace_back(start, e);
}

namespace {

struct WorkspaceBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

struct ThreadState {
  Context ctx;
  WorkspaceBuf ws[2][kNumWorkspaceSlots];  // [bank][slot]
  SideStream side;
  bool initialized = false;
  ~ThreadState() {
    // Device memory is released with the process; freeing here could run
    // after the CUDA runtime has shut down.
  }
};

thread_local ThreadState t_state;

std::atomic<hwyblas_error_handler> g_handler{nullptr};

struct CblasCtx {
  const char* name;
  const int* positions;
};
thread_local const CblasCtx* t_cblas = nullptr;

void Init(ThreadState& st) {
  if (st.initialized) return;
  Context& c = st.ctx;
  cudaGetDevice(&c.device);
  cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device);
  // A blocking stream: it is ordered after work on the legacy default stream,
  // so inputs produced there (e.g. by PyTorch) are complete when we start.
  if (Failed(cudaStreamCreate(&c.own_stream), "stream create")) return;
  c.stream = c.own_stream;
  if (Failed(cudaMalloc(&c.dev_status, 4096), "status alloc")) return;
  cudaMemset(c.dev_status, 0, 4096);
  st.initialized = true;
}

}  // namespace

Context& Ctx() {
  Init(t_state);
  return t_state.ctx;
}

SideStream& Side() {
  ThreadState& st = t_state;
  Init(st);
  SideStream& s = st.side;
  if (!s.ok && s.stream == nullptr) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    s.ok = cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking, greatest) ==
               cudaSuccess &&
           cudaEventCreateWithFlags(&s.to_side, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&s.to_main, cudaEventDisableTiming) == cudaSuccess;
    if (!s.ok) cudaGetLastError();
  }
  return s;
}

void* Workspace(int slot, size_t bytes) {
  ThreadState& st = t_state;
  Init(st);
  WorkspaceBuf& w = st.ws[st.ctx.ws_bank][slot];
  if (bytes == 0) bytes = 256;
  if (w.bytes < bytes) {
    if (w.ptr != nullptr) {
      // Work in flight may still use the old buffer.
      cudaStreamSynchronize(st.ctx.stream);
      cudaFree(w.ptr);
      w.ptr = nullptr;
      w.bytes = 0;
    }
    const size_t want = bytes + bytes / 4;
    if (Failed(cudaMalloc(&w.ptr, want), "workspace alloc")) return nullptr;
    w.bytes = want;
  }
  return w.ptr;
}

bool Failed(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return false;
  t_state.ctx.last_error = static_cast<int>(e);
  fprintf(stderr, "hwyblas_b200: CUDA error in %s: %s\n", what,
          cudaGetErrorString(e));
  return true;
}

bool LaunchFailed(const char* what) { return Failed(cudaGetLastError(), what); }

bool CheckDeviceStatus(const char* what) {
  Context& c = Ctx();
  int flag = 0;
  if (Failed(cudaMemcpyAsync(&flag, c.dev_status, sizeof(int),
                             cudaMemcpyDeviceToHost, c.stream),
             what) ||
      Failed(cudaStreamSynchronize(c.stream), what)) {
    return true;
  }
  if (flag != 0) {
    fprintf(stderr, "hwyblas_b200: a device wait timed out in %s\n", what);
    cudaMemsetAsync(c.dev_status, 0, sizeof(int), c.stream);
    t_state.ctx.last_error = static_cast<int>(cudaErrorLaunchTimeout);
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Error reporting.

void ReportError(const char* routine, int info) {
  const hwyblas_error_handler h = g_handler.load(std::memory_order_acquire);
  if (const CblasCtx* c = t_cblas) {
    const int position = c->positions[info - 1];
    if (h != nullptr) {
      h(c->name, position);
    } else {
      cblas_xerbla(position, c->name, "");
    }
    return;
  }
  if (h != nullptr) {
    h(routine, info);
  } else {
    xerbla_(routine, &info, strlen(routine));
  }
}

namespace {

class CblasScope {
 public:
  CblasScope(const char* name, std::initializer_list<int> positions) {
    int i = 0;
    for (int p : positions) pos_[i++] = p;
    ctx_.name = name;
    ctx_.positions = pos_;
    t_cblas = &ctx_;
  }
  ~CblasScope() { t_cblas = nullptr; }

 private:
  CblasCtx ctx_;
  int pos_[16];
};

char Up(char c) { return (c >= 'a' && c <= 'z') ? static_cast<char>(c - 32) : c; }
bool DecodeOp(char c, bool* trans) {
  c = Up(c);
  *trans = (c == 'T' || c == 'C');
  return c == 'N' || c == 'T' || c == 'C';
}

// ---------------------------------------------------------------------------
// Host/device staging.

bool IsDevicePointer(const void* p) {
  if (p == nullptr) return false;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// A rows x cols column-major matrix (leading dimension ld) made available on
// the device: in place if it is device memory, else copied (if `copy_in`) to
// a compact device buffer whose leading dimension keeps 16-byte alignment.
template <typename T>
struct Staged {
  T* dev = nullptr;
  int ld = 0;
  bool host = false;
  T* host_ptr = nullptr;
  int host_ld = 0, rows = 0, cols = 0;

  bool In(const T* p, int ld_in, int rows_in, int cols_in, int slot,
          bool copy_in) {
    rows = rows_in;
    cols = cols_in;
    host_ptr = const_cast<T*>(p);
    host_ld = ld_in;
    if (IsDevicePointer(p)) {
      dev = const_cast<T*>(p);
      ld = ld_in;
      host = false;
      return true;
    }
    host = true;
    ld = std::max(16, (rows + 15) / 16 * 16);
    dev = static_cast<T*>(
        Workspace(slot, sizeof(T) * static_cast<size_t>(ld) * std::max(cols, 1)));
    if (dev == nullptr) return false;
    if (copy_in && rows > 0 && cols > 0) {
      return !Failed(cudaMemcpy2DAsync(dev, sizeof(T) * ld, p, sizeof(T) * ld_in,
                                       sizeof(T) * rows, cols,
                                       cudaMemcpyHostToDevice, Ctx().stream),
                     "copy in");
    }
    return true;
  }
  void Out() {
    if (!host || rows <= 0 || cols <= 0) return;
    Failed(cudaMemcpy2DAsync(host_ptr, sizeof(T) * host_ld, dev, sizeof(T) * ld,
                             sizeof(T) * rows, cols, cudaMemcpyDeviceToHost,
                             Ctx().stream),
           "copy out");
  }
};

// A 1-D int array (pivots) on the device.
struct StagedInts {
  int* dev = nullptr;
  int* host_ptr = nullptr;
  int n = 0;
  bool host = false;
  bool In(const int* p, int count, int slot_offset_bytes, bool copy_in) {
    n = count;
    host_ptr = const_cast<int*>(p);
    if (IsDevicePointer(p)) {
      dev = const_cast<int*>(p);
      return true;
    }
    host = true;
    dev = Ctx().dev_status + 64 + slot_offset_bytes / 4;
    if (count > 0 && count * 4 + slot_offset_bytes > 4096 - 256) {
      dev = static_cast<int*>(Workspace(kWsStageC, sizeof(int) * count));
    }
    if (copy_in && count > 0) {
      return !Failed(cudaMemcpyAsync(dev, p, sizeof(int) * count,
                                     cudaMemcpyHostToDevice, Ctx().stream),
                     "pivots in");
    }
    return true;
  }
  void Out() {
    if (!host || n <= 0) return;
    Failed(cudaMemcpyAsync(host_ptr, dev, sizeof(int) * n,
                           cudaMemcpyDeviceToHost, Ctx().stream),
           "pivots out");
  }
};

void Finish(const char* what) {
  CheckDeviceStatus(what);
}

int* DeviceInfo() { return Ctx().dev_status + 1; }
void ResetInfo() {
  cudaMemsetAsync(Ctx().dev_status + 1, 0, sizeof(int), Ctx().stream);
}
int ReadInfo() {
  int v = 0;
  Failed(cudaMemcpyAsync(&v, Ctx().dev_status + 1, sizeof(int),
                         cudaMemcpyDeviceToHost, Ctx().stream),
         "info out");
  Failed(cudaStreamSynchronize(Ctx().stream), "sync");
  return v;
}

// ---------------------------------------------------------------------------
// BLAS bodies.

template <typename T>
void GemmEntry(const char* name, const char* transa, const char* transb,
               const int* m_p, const int* n_p, const int* k_p, const T* alpha_p,
               const T* a, const int* lda_p, const T* b, const int* ldb_p,
               const T* beta_p, T* c, const int* ldc_p) {
  const int m = *m_p, n = *n_p, k = *k_p, lda = *lda_p, ldb = *ldb_p,
            ldc = *ldc_p;
  bool ta, tb;
  const bool va = DecodeOp(*transa, &ta), vb = DecodeOp(*transb, &tb);
  const int rows_a = ta ? k : m, rows_b = tb ? n : k;
  int info = 0;
  if (!va) info = 1;
  else if (!vb) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, m)) info = 13;
  if (info != 0) {
    ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p, beta = *beta_p;
  if (m == 0 || n == 0) return;
  if ((k == 0 || alpha == T(0)) && beta == T(1)) return;
  const bool compute = !(k == 0 || alpha == T(0));
  Staged<T> sa, sb, sc;
  if (compute) {
    if (!sa.In(a, lda, rows_a, ta ? m : k, kWsStageA, true)) return;
    if (!sb.In(b, ldb, rows_b, tb ? k : n, kWsStageB, true)) return;
  }
  if (!sc.In(c, ldc, m, n, kWsStageC, beta != T(0))) return;
  GemmFull<T>(ta, tb, m, n, k, alpha, sa.dev, sa.ld, sb.dev, sb.ld, beta, sc.dev,
              sc.ld);
  sc.Out();
  Finish(name);
}

template <typename T>
void TrsmEntry(const char* name, const char* side, const char* uplo,
               const char* transa, const char* diag, const int* m_p,
               const int* n_p, const T* alpha_p, const T* a, const int* lda_p,
               T* b, const int* ldb_p) {
  const int m = *m_p, n = *n_p, lda = *lda_p, ldb = *ldb_p;
  const char s = Up(*side), u = Up(*uplo), d = Up(*diag);
  bool trans;
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const bool vt = DecodeOp(*transa, &trans), vd = (d == 'U' || d == 'N');
  const bool left = (s == 'L');
  const int rows_a = left ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (!vt) info = 3;
  else if (!vd) info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, rows_a)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info != 0) {
    ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p;
  if (m == 0 || n == 0) return;
  Staged<T> sa, sb;
  if (alpha != T(0) && !sa.In(a, lda, rows_a, rows_a, kWsStageA, true)) return;
  if (!sb.In(b, ldb, m, n, kWsStageB, alpha != T(0))) return;
  TrsmFull<T>(left, u == 'L', trans, d == 'U', m, n, alpha, sa.dev,
              std::max(sa.ld, 1), sb.dev, sb.ld);
  sb.Out();
  Finish(name);
}

bool ValidLayout(const char* name, CBLAS_LAYOUT layout) {
  if (layout == CblasRowMajor || layout == CblasColMajor) return true;
  const hwyblas_error_handler h = g_handler.load(std::memory_order_acquire);
  if (h != nullptr) {
    h(name, 1);
  } else {
    cblas_xerbla(1, name, "Illegal layout setting, %d\n", static_cast<int>(layout));
  }
  return false;
}
char TransChar(CBLAS_TRANSPOSE t) {
  switch (t) {
    case CblasNoTrans: return 'N';
    case CblasTrans: return 'T';
    case CblasConjTrans: return 'C';
    default: return '?';
  }
}
char UploChar(CBLAS_UPLO u) {
  return u == CblasUpper ? 'U' : u == CblasLower ? 'L' : '?';
}
char DiagChar(CBLAS_DIAG d) {
  return d == CblasNonUnit ? 'N' : d == CblasUnit ? 'U' : '?';
}
char SideChar(CBLAS_SIDE s) {
  return s == CblasLeft ? 'L' : s == CblasRight ? 'R' : '?';
}
char FlipUplo(char c) { return c == 'U' ? 'L' : c == 'L' ? 'U' : c; }
char FlipSide(char c) { return c == 'L' ? 'R' : c == 'R' ? 'L' : c; }

template <typename T>
void CblasGemm(const char* name, CBLAS_LAYOUT layout,
                      CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb, int m,
                      int n, int k, T alpha, const T* a, int lda, const T* b,
                      int ldb, T beta, T* c, int ldc) {
  if (!ValidLayout(name, layout)) return;
  const char ta = TransChar(transa), tb = TransChar(transb);
  const char* fname = sizeof(T) == 8 ? "DGEMM" : "SGEMM";
  if (layout == CblasColMajor) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14});
    hb::GemmEntry<T>(fname, &ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb,
                     &beta, c, &ldc);
  } else {
    hb::CblasScope scope(name, {3, 2, 5, 4, 6, 7, 10, 11, 8, 9, 12, 13, 14});
    hb::GemmEntry<T>(fname, &tb, &ta, &n, &m, &k, &alpha, b, &ldb, a, &lda,
                     &beta, c, &ldc);
  }
}

}  // namespace
}  // namespace hb

using hb::Ctx;

extern "C" {

HWYBLAS_API void dgemm_(const char* transa, const char* transb,
                        const hwyblas_int* m, const hwyblas_int* n,
                        const hwyblas_int* k, const double* alpha,
                        const double* a, const hwyblas_int* lda,
                        const double* b, const hwyblas_int* ldb,
                        const double* beta, double* c, const hwyblas_int* ldc) {
  hb::GemmEntry<double>("DGEMM", transa, transb, m, n, k, alpha, a, lda, b, ldb,
                        beta, c, ldc);
}

HWYBLAS_API void sgemm_(const char* transa, const char* transb,
                        const hwyblas_int* m, const hwyblas_int* n,
                        const hwyblas_int* k, const float* alpha,
                        const float* a, const hwyblas_int* lda, const float* b,
                        const hwyblas_int* ldb, const float* beta, float* c,
                        const hwyblas_int* ldc) {
  hb::GemmEntry<float>("SGEMM", transa, transb, m, n, k, alpha, a, lda, b, ldb,
                       beta, c, ldc);
}

HWYBLAS_API void dtrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m,
                        const hwyblas_int* n, const double* alpha,
                        const double* a, const hwyblas_int* lda, double* b,
                        const hwyblas_int* ldb) {
  hb::TrsmEntry<double>("DTRSM", side, uplo, transa, diag, m, n, alpha, a, lda,
                        b, ldb);
}

HWYBLAS_API void strsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m,
                        const hwyblas_int* n, const float* alpha,
                        const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb) {
  hb::TrsmEntry<float>("STRSM", side, uplo, transa, diag, m, n, alpha, a, lda,
                       b, ldb);
}

extern "C++" {
// SYRK for T = double and float (src/level3.cc:410-421).
template <typename T>
static void SyrkEntry(const char* name, const char* uplo, const char* trans,
                      const hwyblas_int* n_p, const hwyblas_int* k_p, const T* alpha_p,
                      const T* a, const hwyblas_int* lda_p, const T* beta_p, T* c,
                      const hwyblas_int* ldc_p) {
  const int n = *n_p, k = *k_p, lda = *lda_p, ldc = *ldc_p;
  const char u = hb::Up(*uplo);
  bool t;
  const bool vu = (u == 'L' || u == 'U');
  const bool vt = hb::DecodeOp(*trans, &t);
  const int rows_a = t ? k : n;
  int info = 0;
  if (!vu) info = 1;
  else if (!vt) info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, rows_a)) info = 7;
  else if (ldc < std::max(1, n)) info = 10;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p, beta = *beta_p;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  const bool compute = !(alpha == T(0) || k == 0);
  hb::Staged<T> sa, sc;
  if (compute && !sa.In(a, lda, rows_a, t ? n : k, hb::kWsStageA, true)) return;
  // The whole square is copied so that the other triangle comes back as is.
  if (!sc.In(c, ldc, n, n, hb::kWsStageC, true)) return;
  hb::SyrkFull<T>(u == 'L', t, n, k, alpha, sa.dev, std::max(sa.ld, 1), beta,
               sc.dev, sc.ld);
  sc.Out();
  hb::Finish(name);
}

// SYMM (src/level3.cc:26-76).
// Complex GEMM (src/gemm.cc:67-123): R is the real type, arrays interleaved.
static int DecodeOp3(char c) {
  const char u = hb::Up(c);
  return u == 'N' ? 0 : u == 'T' ? 1 : u == 'C' ? 2 : -1;
}
template <typename R>
static void ZgemmEntry(const char* name, const char* transa, const char* transb,
                       const hwyblas_int* m_p, const hwyblas_int* n_p, const hwyblas_int* k_p,
                       const R* alpha, const R* a, const hwyblas_int* lda_p, const R* b,
                       const hwyblas_int* ldb_p, const R* beta, R* c, const hwyblas_int* ldc_p) {
  const int m = *m_p, n = *n_p, k = *k_p, lda = *lda_p, ldb = *ldb_p, ldc = *ldc_p;
  const int ta = DecodeOp3(*transa), tb = DecodeOp3(*transb);
  const int rows_a = ta == 0 ? m : k, rows_b = tb == 0 ? k : n;
  int info = 0;
  if (ta < 0) info = 1;
  else if (tb < 0) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, m)) info = 13;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  if (m == 0 || n == 0) return;
  const bool alpha_zero = alpha[0] == R(0) && alpha[1] == R(0);
  const bool beta_one = beta[0] == R(1) && beta[1] == R(0);
  const bool beta_zero = beta[0] == R(0) && beta[1] == R(0);
  if ((k == 0 || alpha_zero) && beta_one) return;
  const bool compute = !(k == 0 || alpha_zero);
  // Complex arrays staged as real ones with twice the rows.
  hb::Staged<R> sa, sb, sc;
  if (compute) {
    if (!sa.In(a, 2 * lda, 2 * rows_a, ta == 0 ? k : m, hb::kWsStageA, true)) return;
    if (!sb.In(b, 2 * ldb, 2 * rows_b, tb == 0 ? n : k, hb::kWsStageB, true)) return;
  }
  if (!sc.In(c, 2 * ldc, 2 * m, n, hb::kWsStageC, !beta_zero)) return;
  hb::ZgemmFull<R>(ta, tb, m, n, k, alpha, sa.dev, std::max(sa.ld / 2, 1), sb.dev,
                   std::max(sb.ld / 2, 1), beta, sc.dev, sc.ld / 2);
  sc.Out();
  hb::Finish(name);
}

// Complex TRSM (src/trsm.cc:137-180): R is the real type, arrays interleaved.
template <typename R>
static void ZtrsmEntry(const char* name, const char* side, const char* uplo,
                       const char* transa, const char* diag, const hwyblas_int* m_p,
                       const hwyblas_int* n_p, const R* alpha, const R* a,
                       const hwyblas_int* lda_p, R* b, const hwyblas_int* ldb_p) {
  const int m = *m_p, n = *n_p, lda = *lda_p, ldb = *ldb_p;
  const char s = hb::Up(*side), u = hb::Up(*uplo), d = hb::Up(*diag);
  const int op = DecodeOp3(*transa);
  const bool left = (s == 'L');
  const int ka = left ? m : n;
  int info = 0;
  if (s != 'L' && s != 'R') info = 1;
  else if (u != 'L' && u != 'U') info = 2;
  else if (op < 0) info = 3;
  else if (d != 'U' && d != 'N') info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, ka)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  if (m == 0 || n == 0) return;
  const bool alpha_zero = alpha[0] == R(0) && alpha[1] == R(0);
  hb::Staged<R> sa, sb;
  if (!alpha_zero && !sa.In(a, 2 * lda, 2 * ka, ka, hb::kWsStageA, true)) return;
  if (!sb.In(b, 2 * ldb, 2 * m, n, hb::kWsStageB, !alpha_zero)) return;
  hb::ZtrsmFull<R>(left, u == 'L', op, d == 'U', m, n, alpha, sa.dev, std::max(sa.ld / 2, 1),
                   sb.dev, sb.ld / 2);
  sb.Out();
  hb::Finish(name);
}

// CBLAS complex TRSM (src/cblas.cc:666-700): row-major as the other side and
// triangle, m and n swapped; alpha by address.
template <typename R>
static void CblasZtrsm(const char* name, const char* routine, CBLAS_LAYOUT layout,
                       CBLAS_SIDE side, CBLAS_UPLO uplo, CBLAS_TRANSPOSE transa,
                       CBLAS_DIAG diag, hwyblas_int m_in, hwyblas_int n_in, const void* alpha,
                       const void* a, hwyblas_int lda, void* b, hwyblas_int ldb) {
  if (!hb::ValidLayout(name, layout)) return;
  char sc = hb::SideChar(side), uc = hb::UploChar(uplo);
  const char tc = hb::TransChar(transa), dc = hb::DiagChar(diag);
  int m = m_in, n = n_in;
  const bool row = (layout == CblasRowMajor);
  if (row) {
    sc = hb::FlipSide(sc);
    uc = hb::FlipUplo(uc);
    std::swap(m, n);
  }
  const R* al = static_cast<const R*>(alpha);
  if (row) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 7, 6, 8, 9, 10, 11, 12});
    ZtrsmEntry<R>(routine, &sc, &uc, &tc, &dc, &m, &n, al, static_cast<const R*>(a), &lda,
                  static_cast<R*>(b), &ldb);
  } else {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12});
    ZtrsmEntry<R>(routine, &sc, &uc, &tc, &dc, &m, &n, al, static_cast<const R*>(a), &lda,
                  static_cast<R*>(b), &ldb);
  }
}

// CBLAS complex GEMM (src/cblas.cc:520-537): row-major as the column-major
// product of the swapped operands; alpha and beta by address.
template <typename R>
static void CblasZgemm(const char* name, const char* routine, CBLAS_LAYOUT layout,
                       CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb, hwyblas_int m,
                       hwyblas_int n, hwyblas_int k, const void* alpha, const void* a,
                       hwyblas_int lda, const void* b, hwyblas_int ldb, const void* beta,
                       void* c, hwyblas_int ldc) {
  if (!hb::ValidLayout(name, layout)) return;
  const char ta = hb::TransChar(transa), tb = hb::TransChar(transb);
  const R* al = static_cast<const R*>(alpha);
  const R* be = static_cast<const R*>(beta);
  if (layout == CblasColMajor) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14});
    ZgemmEntry<R>(routine, &ta, &tb, &m, &n, &k, al, static_cast<const R*>(a), &lda,
                  static_cast<const R*>(b), &ldb, be, static_cast<R*>(c), &ldc);
  } else {
    hb::CblasScope scope(name, {3, 2, 5, 4, 6, 7, 10, 11, 8, 9, 12, 13, 14});
    ZgemmEntry<R>(routine, &tb, &ta, &n, &m, &k, al, static_cast<const R*>(b), &ldb,
                  static_cast<const R*>(a), &lda, be, static_cast<R*>(c), &ldc);
  }
}

template <typename T>
static void SymmEntry(const char* name, const char* side, const char* uplo,
                      const hwyblas_int* m_p, const hwyblas_int* n_p, const T* alpha_p,
                      const T* a, const hwyblas_int* lda_p, const T* b,
                      const hwyblas_int* ldb_p, const T* beta_p, T* c,
                      const hwyblas_int* ldc_p) {
  const int m = *m_p, n = *n_p, lda = *lda_p, ldb = *ldb_p, ldc = *ldc_p;
  const char s = hb::Up(*side), u = hb::Up(*uplo);
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const int ka = (s == 'L') ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (lda < std::max(1, ka)) info = 7;
  else if (ldb < std::max(1, m)) info = 9;
  else if (ldc < std::max(1, m)) info = 12;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p, beta = *beta_p;
  if (m == 0 || n == 0 || (alpha == T(0) && beta == T(1))) return;
  const bool compute = (alpha != T(0));
  hb::Staged<T> sa, sb, sc;
  if (compute && !sa.In(a, lda, ka, ka, hb::kWsStageA, true)) return;
  if (compute && !sb.In(b, ldb, m, n, hb::kWsStageB, true)) return;
  if (!sc.In(c, ldc, m, n, hb::kWsStageC, beta != T(0))) return;
  hb::SymmFull<T>(s == 'L', u == 'L', m, n, alpha, sa.dev, std::max(sa.ld, 1), sb.dev,
                  std::max(sb.ld, 1), beta, sc.dev, sc.ld);
  sc.Out();
  hb::Finish(name);
}

// SYR2K (src/level3.cc:153-221).
template <typename T>
static void Syr2kEntry(const char* name, const char* uplo, const char* trans,
                       const hwyblas_int* n_p, const hwyblas_int* k_p, const T* alpha_p,
                       const T* a, const hwyblas_int* lda_p, const T* b,
                       const hwyblas_int* ldb_p, const T* beta_p, T* c,
                       const hwyblas_int* ldc_p) {
  const int n = *n_p, k = *k_p, lda = *lda_p, ldb = *ldb_p, ldc = *ldc_p;
  const char u = hb::Up(*uplo);
  bool t;
  const bool vu = (u == 'L' || u == 'U');
  const bool vt = hb::DecodeOp(*trans, &t);
  const int rows = t ? k : n;
  int info = 0;
  if (!vu) info = 1;
  else if (!vt) info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, rows)) info = 7;
  else if (ldb < std::max(1, rows)) info = 9;
  else if (ldc < std::max(1, n)) info = 12;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p, beta = *beta_p;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  const bool compute = !(alpha == T(0) || k == 0);
  hb::Staged<T> sa, sb, sc;
  if (compute && !sa.In(a, lda, rows, t ? n : k, hb::kWsStageA, true)) return;
  if (compute && !sb.In(b, ldb, rows, t ? n : k, hb::kWsStageB, true)) return;
  // The whole square is copied so that the other triangle comes back as is.
  if (!sc.In(c, ldc, n, n, hb::kWsStageC, true)) return;
  hb::Syr2kFull<T>(u == 'L', t, n, k, alpha, sa.dev, std::max(sa.ld, 1), sb.dev,
                   std::max(sb.ld, 1), beta, sc.dev, sc.ld);
  sc.Out();
  hb::Finish(name);
}

// GEMMTR and its alias GEMMT (src/level3.cc:226-280).
template <typename T>
static void GemmtrEntry(const char* name, const char* uplo, const char* transa,
                        const char* transb, const hwyblas_int* n_p, const hwyblas_int* k_p,
                        const T* alpha_p, const T* a, const hwyblas_int* lda_p, const T* b,
                        const hwyblas_int* ldb_p, const T* beta_p, T* c,
                        const hwyblas_int* ldc_p) {
  const int n = *n_p, k = *k_p, lda = *lda_p, ldb = *ldb_p, ldc = *ldc_p;
  const char u = hb::Up(*uplo);
  bool ta, tb;
  const bool vu = (u == 'L' || u == 'U');
  const bool va = hb::DecodeOp(*transa, &ta), vb = hb::DecodeOp(*transb, &tb);
  const int rows_a = ta ? k : n, rows_b = tb ? n : k;
  int info = 0;
  if (!vu) info = 1;
  else if (!va) info = 2;
  else if (!vb) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, n)) info = 13;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p, beta = *beta_p;
  if (n == 0 || ((alpha == T(0) || k == 0) && beta == T(1))) return;
  const bool compute = !(alpha == T(0) || k == 0);
  hb::Staged<T> sa, sb, sc;
  if (compute && !sa.In(a, lda, rows_a, ta ? n : k, hb::kWsStageA, true)) return;
  if (compute && !sb.In(b, ldb, rows_b, tb ? k : n, hb::kWsStageB, true)) return;
  if (!sc.In(c, ldc, n, n, hb::kWsStageC, true)) return;
  hb::GemmtrFull<T>(u == 'L', ta, tb, n, k, alpha, sa.dev, std::max(sa.ld, 1), sb.dev,
                    std::max(sb.ld, 1), beta, sc.dev, sc.ld);
  sc.Out();
  hb::Finish(name);
}

// TRMM (src/level3.cc:284-342).
template <typename T>
static void TrmmEntry(const char* name, const char* side, const char* uplo,
                      const char* transa, const char* diag, const hwyblas_int* m_p,
                      const hwyblas_int* n_p, const T* alpha_p, const T* a,
                      const hwyblas_int* lda_p, T* b, const hwyblas_int* ldb_p) {
  const int m = *m_p, n = *n_p, lda = *lda_p, ldb = *ldb_p;
  const char s = hb::Up(*side), u = hb::Up(*uplo), d = hb::Up(*diag);
  bool trans;
  const bool vs = (s == 'L' || s == 'R'), vu = (u == 'L' || u == 'U');
  const bool vt = hb::DecodeOp(*transa, &trans), vd = (d == 'U' || d == 'N');
  const int ka = (s == 'L') ? m : n;
  int info = 0;
  if (!vs) info = 1;
  else if (!vu) info = 2;
  else if (!vt) info = 3;
  else if (!vd) info = 4;
  else if (m < 0) info = 5;
  else if (n < 0) info = 6;
  else if (lda < std::max(1, ka)) info = 9;
  else if (ldb < std::max(1, m)) info = 11;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const T alpha = *alpha_p;
  if (m == 0 || n == 0) return;
  hb::Staged<T> sa, sb;
  if (alpha != T(0) && !sa.In(a, lda, ka, ka, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, m, n, hb::kWsStageB, alpha != T(0))) return;
  hb::TrmmFull<T>(s == 'L', u == 'L', trans, d == 'U', m, n, alpha, sa.dev,
                  std::max(sa.ld, 1), sb.dev, sb.ld);
  sb.Out();
  hb::Finish(name);
}
}  // extern "C++"

HWYBLAS_API void dsyrk_(const char* uplo, const char* trans, const hwyblas_int* n,
                        const hwyblas_int* k, const double* alpha, const double* a,
                        const hwyblas_int* lda, const double* beta, double* c,
                        const hwyblas_int* ldc) {
  SyrkEntry<double>("DSYRK", uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}

HWYBLAS_API void ssyrk_(const char* uplo, const char* trans, const hwyblas_int* n,
                        const hwyblas_int* k, const float* alpha, const float* a,
                        const hwyblas_int* lda, const float* beta, float* c,
                        const hwyblas_int* ldc) {
  SyrkEntry<float>("SSYRK", uplo, trans, n, k, alpha, a, lda, beta, c, ldc);
}

HWYBLAS_API void zgemm_(const char* transa, const char* transb, const hwyblas_int* m,
                        const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                        const double* a, const hwyblas_int* lda, const double* b,
                        const hwyblas_int* ldb, const double* beta, double* c,
                        const hwyblas_int* ldc) {
  ZgemmEntry<double>("ZGEMM", transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
HWYBLAS_API void cgemm_(const char* transa, const char* transb, const hwyblas_int* m,
                        const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                        const float* a, const hwyblas_int* lda, const float* b,
                        const hwyblas_int* ldb, const float* beta, float* c,
                        const hwyblas_int* ldc) {
  ZgemmEntry<float>("CGEMM", transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
HWYBLAS_API void ztrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const double* alpha, const double* a, const hwyblas_int* lda,
                        double* b, const hwyblas_int* ldb) {
  ZtrsmEntry<double>("ZTRSM", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb);
}
HWYBLAS_API void ctrsm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const float* alpha, const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb) {
  ZtrsmEntry<float>("CTRSM", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb);
}
HWYBLAS_API void cblas_ztrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const void* alpha, const void* a, const hwyblas_int lda, void* b,
                             const hwyblas_int ldb) {
  CblasZtrsm<double>("cblas_ztrsm", "ZTRSM", layout, side, uplo, transa, diag, m, n, alpha, a,
                     lda, b, ldb);
}
HWYBLAS_API void cblas_ctrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m, const hwyblas_int n,
                             const void* alpha, const void* a, const hwyblas_int lda, void* b,
                             const hwyblas_int ldb) {
  CblasZtrsm<float>("cblas_ctrsm", "CTRSM", layout, side, uplo, transa, diag, m, n, alpha, a,
                    lda, b, ldb);
}
HWYBLAS_API void cblas_zgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k, const void* alpha,
                             const void* a, const hwyblas_int lda, const void* b,
                             const hwyblas_int ldb, const void* beta, void* c,
                             const hwyblas_int ldc) {
  CblasZgemm<double>("cblas_zgemm", "ZGEMM", layout, transa, transb, m, n, k, alpha, a, lda, b,
                     ldb, beta, c, ldc);
}
HWYBLAS_API void cblas_cgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k, const void* alpha,
                             const void* a, const hwyblas_int lda, const void* b,
                             const hwyblas_int ldb, const void* beta, void* c,
                             const hwyblas_int ldc) {
  CblasZgemm<float>("cblas_cgemm", "CGEMM", layout, transa, transb, m, n, k, alpha, a, lda, b,
                    ldb, beta, c, ldc);
}

HWYBLAS_API void dsymm_(const char* side, const char* uplo, const hwyblas_int* m,
                        const hwyblas_int* n, const double* alpha, const double* a,
                        const hwyblas_int* lda, const double* b, const hwyblas_int* ldb,
                        const double* beta, double* c, const hwyblas_int* ldc) {
  SymmEntry<double>("DSYMM", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}
HWYBLAS_API void ssymm_(const char* side, const char* uplo, const hwyblas_int* m,
                        const hwyblas_int* n, const float* alpha, const float* a,
                        const hwyblas_int* lda, const float* b, const hwyblas_int* ldb,
                        const float* beta, float* c, const hwyblas_int* ldc) {
  SymmEntry<float>("SSYMM", side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc);
}

HWYBLAS_API void dsyr2k_(const char* uplo, const char* trans, const hwyblas_int* n,
                         const hwyblas_int* k, const double* alpha, const double* a,
                         const hwyblas_int* lda, const double* b, const hwyblas_int* ldb,
                         const double* beta, double* c, const hwyblas_int* ldc) {
  Syr2kEntry<double>("DSYR2K", uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
HWYBLAS_API void ssyr2k_(const char* uplo, const char* trans, const hwyblas_int* n,
                         const hwyblas_int* k, const float* alpha, const float* a,
                         const hwyblas_int* lda, const float* b, const hwyblas_int* ldb,
                         const float* beta, float* c, const hwyblas_int* ldc) {
  Syr2kEntry<float>("SSYR2K", uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

HWYBLAS_API void dgemmtr_(const char* uplo, const char* transa, const char* transb,
                          const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                          const double* a, const hwyblas_int* lda, const double* b,
                          const hwyblas_int* ldb, const double* beta, double* c,
                          const hwyblas_int* ldc) {
  GemmtrEntry<double>("DGEMMTR", uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c,
                      ldc);
}
HWYBLAS_API void sgemmtr_(const char* uplo, const char* transa, const char* transb,
                          const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                          const float* a, const hwyblas_int* lda, const float* b,
                          const hwyblas_int* ldb, const float* beta, float* c,
                          const hwyblas_int* ldc) {
  GemmtrEntry<float>("SGEMMTR", uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c,
                     ldc);
}
HWYBLAS_API void dgemmt_(const char* uplo, const char* transa, const char* transb,
                         const hwyblas_int* n, const hwyblas_int* k, const double* alpha,
                         const double* a, const hwyblas_int* lda, const double* b,
                         const hwyblas_int* ldb, const double* beta, double* c,
                         const hwyblas_int* ldc) {
  GemmtrEntry<double>("DGEMMT", uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c,
                      ldc);
}
HWYBLAS_API void sgemmt_(const char* uplo, const char* transa, const char* transb,
                         const hwyblas_int* n, const hwyblas_int* k, const float* alpha,
                         const float* a, const hwyblas_int* lda, const float* b,
                         const hwyblas_int* ldb, const float* beta, float* c,
                         const hwyblas_int* ldc) {
  GemmtrEntry<float>("SGEMMT", uplo, transa, transb, n, k, alpha, a, lda, b, ldb, beta, c,
                     ldc);
}

HWYBLAS_API void dtrmm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const double* alpha, const double* a, const hwyblas_int* lda,
                        double* b, const hwyblas_int* ldb) {
  TrmmEntry<double>("DTRMM", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb);
}
HWYBLAS_API void strmm_(const char* side, const char* uplo, const char* transa,
                        const char* diag, const hwyblas_int* m, const hwyblas_int* n,
                        const float* alpha, const float* a, const hwyblas_int* lda, float* b,
                        const hwyblas_int* ldb) {
  TrmmEntry<float>("STRMM", side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb);
}

HWYBLAS_API hwyblas_int idamax_(const hwyblas_int* n_p, const double* x,
                                const hwyblas_int* incx_p) {
  const int n = *n_p, incx = *incx_p;
  if (n < 1 || incx <= 0) return 0;
  if (n == 1) return 1;
  hb::Staged<double> sx;
  const long long span = static_cast<long long>(n - 1) * incx + 1;
  if (span > 0x7fffffff) return 0;
  if (!sx.In(x, static_cast<int>(span), static_cast<int>(span), 1,
             hb::kWsStageA, true))
    return 0;
  int* out = Ctx().dev_status + 2;
  hb::Iamax<double>(n, sx.dev, incx, out);
  int result = 0;
  hb::Failed(cudaMemcpyAsync(&result, out, sizeof(int), cudaMemcpyDeviceToHost,
                             Ctx().stream),
             "idamax out");
  hb::Finish("IDAMAX");
  return result;
}

HWYBLAS_API void xerbla_(const char* srname, const hwyblas_int* info,
                         size_t srname_len) {
  size_t len = 0;
  while (len < srname_len && srname[len] != '\0' && srname[len] != ' ') ++len;
  fprintf(stderr,
          " ** On entry to %.*s parameter number %d had an illegal value\n",
          static_cast<int>(len), srname, static_cast<int>(*info));
}

HWYBLAS_API hwyblas_error_handler
hwyblas_set_error_handler(hwyblas_error_handler handler) {
  return hb::g_handler.exchange(handler, std::memory_order_acq_rel);
}

// ---------------------------------------------------------------------------
// LAPACK.

static bool CheckGetrf(const char* name, int m, int n, int lda, int* info) {
  *info = 0;
  if (m < 0) *info = -1;
  else if (n < 0) *info = -2;
  else if (lda < std::max(1, m)) *info = -4;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return false;
  }
  return true;
}

extern "C++" {
// The LU family for T = double and float (the reference instantiates one
// template for both: getrf.cc:507-546).
template <typename T>
static void GetrfEntry(bool recursive, const char* name, const hwyblas_int* m_p,
                       const hwyblas_int* n_p, T* a, const hwyblas_int* lda_p,
                       hwyblas_int* ipiv, hwyblas_int* info) {
  const int m = *m_p, n = *n_p, lda = *lda_p;
  if (!CheckGetrf(name, m, n, lda, info)) return;
  if (m == 0 || n == 0) return;
  hb::Staged<T> sa;
  hb::StagedInts sp;
  if (!sa.In(a, lda, m, n, hb::kWsStageA, true)) return;
  if (!sp.In(ipiv, std::min(m, n), 0, false)) return;
  hb::ResetInfo();
  if (recursive) {
    hb::Getrf2<T>(m, n, sa.dev, sa.ld, sp.dev, hb::DeviceInfo());
  } else {
    hb::Getrf<T>(m, n, sa.dev, sa.ld, sp.dev, hb::DeviceInfo());
  }
  sa.Out();
  sp.Out();
  *info = hb::ReadInfo();
  hb::Finish(name);
}

template <typename T>
static void LaswpEntry(const char* name, const hwyblas_int* n_p, T* a,
                       const hwyblas_int* lda_p, const hwyblas_int* k1_p,
                       const hwyblas_int* k2_p, const hwyblas_int* ipiv,
                       const hwyblas_int* incx_p) {
  const int n = *n_p, lda = *lda_p, k1 = *k1_p, k2 = *k2_p, incx = *incx_p;
  if (incx == 0 || n <= 0) return;
  const int absinc = incx < 0 ? -incx : incx;
  const int count = k1 + (k2 - k1) * absinc;  // entries ipiv(1..count)
  if (count <= 0 || k2 < k1) return;
  hb::Staged<T> sa;
  hb::StagedInts sp;
  if (!sa.In(a, lda, lda, n, hb::kWsStageA, true)) return;
  if (!sp.In(ipiv, count, 0, true)) return;
  hb::Laswp<T>(n, sa.dev, sa.ld, k1, k2, sp.dev, incx);
  sa.Out();
  hb::Finish(name);
}

template <typename T>
static void GetrsEntry(const char* name, const char* trans, const hwyblas_int* n_p,
                       const hwyblas_int* nrhs_p, const T* a, const hwyblas_int* lda_p,
                       const hwyblas_int* ipiv, T* b, const hwyblas_int* ldb_p,
                       hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  const char t = hb::Up(*trans);
  const bool notran = (t == 'N');
  *info = 0;
  if (!notran && t != 'T' && t != 'C') *info = -1;
  else if (n < 0) *info = -2;
  else if (nrhs < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  else if (ldb < std::max(1, n)) *info = -8;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (n == 0 || nrhs == 0) return;
  hb::Staged<T> sa, sb;
  hb::StagedInts sp;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sp.In(ipiv, n, 0, true)) return;
  hb::Getrs<T>(!notran, n, nrhs, sa.dev, sa.ld, sp.dev, sb.dev, sb.ld);
  sb.Out();
  hb::Finish(name);
}

template <typename T>
static void GesvEntry(const char* name, const hwyblas_int* n_p, const hwyblas_int* nrhs_p,
                      T* a, const hwyblas_int* lda_p, hwyblas_int* ipiv, T* b,
                      const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  *info = 0;
  if (n < 0) *info = -1;
  else if (nrhs < 0) *info = -2;
  else if (lda < std::max(1, n)) *info = -4;
  else if (ldb < std::max(1, n)) *info = -7;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (n == 0) return;
  hb::Staged<T> sa, sb;
  hb::StagedInts sp;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sp.In(ipiv, n, 0, false)) return;
  hb::ResetInfo();
  hb::Getrf<T>(n, n, sa.dev, sa.ld, sp.dev, hb::DeviceInfo());
  const int finfo = hb::ReadInfo();
  if (finfo == 0 && nrhs > 0) {
    hb::Getrs<T>(false, n, nrhs, sa.dev, sa.ld, sp.dev, sb.dev, sb.ld);
  }
  sa.Out();
  sp.Out();
  if (finfo == 0) sb.Out();
  *info = finfo;
  hb::Finish(name);
}

// The complex LU family (zgetrf_, cgetrf_, ... : src/lapack/getrf.cc:505-553
// for T = c64 and c32): interleaved (re, im) arrays, leading dimensions in
// complex elements. A device array whose address is not aligned to a whole
// complex element is worked on in an aligned copy (the GEMM and TRSM updates
// move whole elements).
template <typename R>
struct ZWorkMatrix {
  hb::Staged<R> staged;
  R* dev = nullptr;
  int ld = 0;  // complex elements
  int rows = 0, cols = 0;
  bool copied = false;
  bool In(R* p, int ld_in, int rows_in, int cols_in, int slot, bool copy_in,
          int align_slot = hb::kWsZFactor) {
    rows = rows_in;
    cols = cols_in;
    if (!staged.In(p, 2 * ld_in, 2 * rows_in, cols_in, slot, copy_in)) return false;
    dev = staged.dev;
    ld = std::max(staged.ld / 2, 1);
    if (reinterpret_cast<uintptr_t>(dev) % (2 * sizeof(R)) == 0) return true;
    const size_t esz = 2 * sizeof(R);
    R* w = static_cast<R*>(hb::Workspace(align_slot, esz * rows * std::max(cols, 1)));
    if (w == nullptr) return false;
    if (copy_in && hb::Failed(cudaMemcpy2DAsync(w, esz * rows, dev, esz * ld, esz * rows, cols,
                                                cudaMemcpyDeviceToDevice, Ctx().stream),
                              "complex matrix copy"))
      return false;
    dev = w;
    ld = std::max(rows, 1);
    copied = true;
    return true;
  }
  void Out() {
    if (copied) {
      const size_t esz = 2 * sizeof(R);
      hb::Failed(cudaMemcpy2DAsync(staged.dev, esz * (staged.ld / 2), dev, esz * ld, esz * rows,
                                   cols, cudaMemcpyDeviceToDevice, Ctx().stream),
                 "complex matrix copy back");
    }
    staged.Out();
  }
};

template <typename R>
static void ZGetrfEntry(bool recursive, const char* name, const hwyblas_int* m_p,
                        const hwyblas_int* n_p, R* a, const hwyblas_int* lda_p,
                        hwyblas_int* ipiv, hwyblas_int* info) {
  const int m = *m_p, n = *n_p, lda = *lda_p;
  if (!CheckGetrf(name, m, n, lda, info)) return;
  if (m == 0 || n == 0) return;
  ZWorkMatrix<R> sa;
  hb::StagedInts sp;
  if (!sa.In(a, lda, m, n, hb::kWsStageA, true)) return;
  if (!sp.In(ipiv, std::min(m, n), 0, false)) return;
  hb::ResetInfo();
  hb::ZGetrf<R>(recursive, m, n, sa.dev, sa.ld, sp.dev, hb::DeviceInfo());
  sa.Out();
  sp.Out();
  *info = hb::ReadInfo();
  hb::Finish(name);
}

template <typename R>
static void ZLaswpEntry(const char* name, const hwyblas_int* n_p, R* a,
                        const hwyblas_int* lda_p, const hwyblas_int* k1_p,
                        const hwyblas_int* k2_p, const hwyblas_int* ipiv,
                        const hwyblas_int* incx_p) {
  const int n = *n_p, lda = *lda_p, k1 = *k1_p, k2 = *k2_p, incx = *incx_p;
  if (incx == 0 || n <= 0) return;
  const int absinc = incx < 0 ? -incx : incx;
  const int count = k1 + (k2 - k1) * absinc;
  if (count <= 0 || k2 < k1) return;
  hb::Staged<R> sa;
  hb::StagedInts sp;
  if (!sa.In(a, 2 * lda, 2 * lda, n, hb::kWsStageA, true)) return;
  if (!sp.In(ipiv, count, 0, true)) return;
  hb::ZLaswp<R>(n, sa.dev, sa.ld / 2, k1, k2, sp.dev, incx);
  sa.Out();
  hb::Finish(name);
}

template <typename R>
static void ZGetrsEntry(const char* name, const char* trans, const hwyblas_int* n_p,
                        const hwyblas_int* nrhs_p, const R* a, const hwyblas_int* lda_p,
                        const hwyblas_int* ipiv, R* b, const hwyblas_int* ldb_p,
                        hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  const int op = DecodeOp3(*trans);
  *info = 0;
  if (op < 0) *info = -1;
  else if (n < 0) *info = -2;
  else if (nrhs < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  else if (ldb < std::max(1, n)) *info = -8;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (n == 0 || nrhs == 0) return;
  ZWorkMatrix<R> sa, sb;
  hb::StagedInts sp;
  if (!sa.In(const_cast<R*>(a), lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true, hb::kWsZFactorB)) return;
  if (!sp.In(ipiv, n, 0, true)) return;
  hb::ZGetrs<R>(op, n, nrhs, sa.dev, sa.ld, sp.dev, sb.dev, sb.ld);
  sb.Out();
  hb::Finish(name);
}

template <typename R>
static void ZGesvEntry(const char* name, const hwyblas_int* n_p, const hwyblas_int* nrhs_p,
                       R* a, const hwyblas_int* lda_p, hwyblas_int* ipiv, R* b,
                       const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  *info = 0;
  if (n < 0) *info = -1;
  else if (nrhs < 0) *info = -2;
  else if (lda < std::max(1, n)) *info = -4;
  else if (ldb < std::max(1, n)) *info = -7;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (n == 0) return;
  ZWorkMatrix<R> sa, sb;
  hb::StagedInts sp;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true, hb::kWsZFactorB)) return;
  if (!sp.In(ipiv, n, 0, false)) return;
  hb::ResetInfo();
  hb::ZGetrf<R>(false, n, n, sa.dev, sa.ld, sp.dev, hb::DeviceInfo());
  const int finfo = hb::ReadInfo();
  if (finfo == 0 && nrhs > 0) hb::ZGetrs<R>(0, n, nrhs, sa.dev, sa.ld, sp.dev, sb.dev, sb.ld);
  sa.Out();
  sp.Out();
  if (finfo == 0) sb.Out();
  *info = finfo;
  hb::Finish(name);
}

// WORK(1) := v in the caller's array (host or device).
template <typename T>
static void StoreWork0(T* work, T v) {
  if (work == nullptr) return;
  if (hb::IsDevicePointer(work)) {
    hb::Failed(cudaMemcpyAsync(work, &v, sizeof(T), cudaMemcpyHostToDevice, Ctx().stream),
               "work(1)");
    hb::Failed(cudaStreamSynchronize(Ctx().stream), "sync");
  } else {
    *work = v;
  }
}

// xGETRI (src/lapack/getrf.cc:369-483): WORK(1) = max(1, 64 n) before the
// argument checks, lwork = -1 queries, lwork < 64 n narrows the blocks. The
// library's own workspace holds the block columns; the caller's WORK only
// reports sizes.
template <typename T>
static void GetriEntry(const char* name, const hwyblas_int* n_p, T* a,
                       const hwyblas_int* lda_p, const hwyblas_int* ipiv, T* work,
                       const hwyblas_int* lwork_p, hwyblas_int* info) {
  const int n = *n_p, lda = *lda_p, lwork = *lwork_p;
  StoreWork0<T>(work, static_cast<T>(std::max(1, n * 64)));
  const bool lquery = (lwork == -1);
  *info = 0;
  if (n < 0) *info = -1;
  else if (lda < std::max(1, n)) *info = -3;
  else if (lwork < std::max(1, n) && !lquery) *info = -6;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (lquery || n == 0) return;
  hb::Staged<T> sa;
  hb::StagedInts sp;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sp.In(ipiv, n, 0, true)) return;
  int iws = 0;
  const int r = hb::GetriFull<T>(n, sa.dev, sa.ld, sp.dev, lwork, &iws);
  sa.Out();
  hb::Finish(name);
  *info = r;
  if (r == 0) StoreWork0<T>(work, static_cast<T>(iws));
}

// xTRTRI / xTRTI2 (src/lapack/triangular.cc:18-166).
template <typename T>
static void TrtriEntry(bool unblocked, const char* name, const char* uplo, const char* diag,
                       const hwyblas_int* n_p, T* a, const hwyblas_int* lda_p,
                       hwyblas_int* info) {
  const int n = *n_p, lda = *lda_p;
  const char u = hb::Up(*uplo), d = hb::Up(*diag);
  *info = 0;
  if (u != 'U' && u != 'L') *info = -1;
  else if (d != 'N' && d != 'U') *info = -2;
  else if (n < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  if (n == 0) return;
  hb::Staged<T> sa;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  const int r = unblocked ? hb::Trti2Full<T>(u == 'U', d == 'U', n, sa.dev, sa.ld)
                          : hb::TrtriFull<T>(u == 'U', d == 'U', n, sa.dev, sa.ld);
  sa.Out();
  hb::Finish(name);
  *info = r;
}

// An array of `count` elements made available on the device (copied in and,
// by Out, back when it is host memory).
template <typename E>
struct StagedVec {
  E* dev = nullptr;
  E* host = nullptr;
  size_t count = 0;
  bool In(E* p, size_t n, int slot) {
    count = n;
    if (p == nullptr || n == 0) return true;
    if (hb::IsDevicePointer(p)) {
      dev = p;
      return true;
    }
    host = p;
    dev = static_cast<E*>(hb::Workspace(slot, sizeof(E) * n));
    if (dev == nullptr) return false;
    return !hb::Failed(cudaMemcpyAsync(dev, p, sizeof(E) * n, cudaMemcpyHostToDevice,
                                       Ctx().stream),
                       "copy in");
  }
  void Out() {
    if (host == nullptr || count == 0) return;
    hb::Failed(cudaMemcpyAsync(host, dev, sizeof(E) * count, cudaMemcpyDeviceToHost,
                               Ctx().stream),
               "copy out");
  }
};

// Stores v[0..n) into the caller's array p (host or device).
template <typename T>
static void StoreVector(T* p, const T* v, int n) {
  if (p == nullptr || n <= 0) return;
  if (hb::IsDevicePointer(p)) {
    hb::Failed(cudaMemcpyAsync(p, v, sizeof(T) * n, cudaMemcpyHostToDevice, Ctx().stream),
               "store");
    hb::Failed(cudaStreamSynchronize(Ctx().stream), "sync");
  } else {
    for (int i = 0; i < n; ++i) p[i] = v[i];
  }
}

// xGERFS (src/lapack/gesvx.cc:319-456, 796-806).
template <typename T>
static void GerfsEntry(const char* name, const char* trans, const hwyblas_int* n_p,
                       const hwyblas_int* nrhs_p, const T* a, const hwyblas_int* lda_p,
                       const T* af, const hwyblas_int* ldaf_p, const hwyblas_int* ipiv,
                       const T* b, const hwyblas_int* ldb_p, T* x, const hwyblas_int* ldx_p,
                       T* ferr, T* berr, T* work, hwyblas_int* iwork, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldaf = *ldaf_p, ldb = *ldb_p,
            ldx = *ldx_p;
  bool t = false;
  const bool vt = hb::DecodeOp(*trans, &t);
  *info = 0;
  if (!vt) *info = -1;
  else if (n < 0) *info = -2;
  else if (nrhs < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  else if (ldaf < std::max(1, n)) *info = -7;
  else if (ldb < std::max(1, n)) *info = -10;
  else if (ldx < std::max(1, n)) *info = -12;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return;
  }
  std::vector<T> fe(std::max(nrhs, 0), T(0)), be(std::max(nrhs, 0), T(0));
  if (n == 0 || nrhs == 0) {
    StoreVector<T>(ferr, fe.data(), nrhs);
    StoreVector<T>(berr, be.data(), nrhs);
    return;
  }
  hb::Staged<T> sa, saf, sb, sx;
  hb::StagedInts sp;
  StagedVec<T> sw;
  StagedVec<int> si;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!saf.In(af, ldaf, n, n, hb::kWsStageAF, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sx.In(x, ldx, n, nrhs, hb::kWsStageX, true)) return;
  if (!sp.In(ipiv, n, 0, true)) return;
  if (!sw.In(work, 3 * static_cast<size_t>(n), hb::kWsGerfsWork)) return;
  if (!si.In(iwork, static_cast<size_t>(n), hb::kWsGerfsIwork)) return;
  hb::GerfsFull<T>(t, n, nrhs, sa.dev, sa.ld, saf.dev, saf.ld, sp.dev, sb.dev, sb.ld, sx.dev,
                   sx.ld, fe.data(), be.data(), sw.dev, si.dev);
  sx.Out();
  sw.Out();
  si.Out();
  hb::Finish(name);
  StoreVector<T>(ferr, fe.data(), nrhs);
  StoreVector<T>(berr, be.data(), nrhs);
}
}  // extern "C++"

HWYBLAS_API void dgetrf_(const hwyblas_int* m, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv,
                         hwyblas_int* info) {
  GetrfEntry<double>(false, "DGETRF", m, n, a, lda, ipiv, info);
}

HWYBLAS_API void dgetrf2_(const hwyblas_int* m, const hwyblas_int* n,
                          double* a, const hwyblas_int* lda, hwyblas_int* ipiv,
                          hwyblas_int* info) {
  GetrfEntry<double>(true, "DGETRF2", m, n, a, lda, ipiv, info);
}

HWYBLAS_API void dlaswp_(const hwyblas_int* n, double* a, const hwyblas_int* lda,
                         const hwyblas_int* k1, const hwyblas_int* k2,
                         const hwyblas_int* ipiv, const hwyblas_int* incx) {
  LaswpEntry<double>("DLASWP", n, a, lda, k1, k2, ipiv, incx);
}

HWYBLAS_API void dgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const double* a,
                         const hwyblas_int* lda, const hwyblas_int* ipiv,
                         double* b, const hwyblas_int* ldb, hwyblas_int* info) {
  GetrsEntry<double>("DGETRS", trans, n, nrhs, a, lda, ipiv, b, ldb, info);
}

HWYBLAS_API void dgesv_(const hwyblas_int* n, const hwyblas_int* nrhs, double* a,
                        const hwyblas_int* lda, hwyblas_int* ipiv, double* b,
                        const hwyblas_int* ldb, hwyblas_int* info) {
  GesvEntry<double>("DGESV", n, nrhs, a, lda, ipiv, b, ldb, info);
}

HWYBLAS_API void sgetrf_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* ipiv,
                         hwyblas_int* info) {
  GetrfEntry<float>(false, "SGETRF", m, n, a, lda, ipiv, info);
}

HWYBLAS_API void sgetrf2_(const hwyblas_int* m, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* ipiv,
                          hwyblas_int* info) {
  GetrfEntry<float>(true, "SGETRF2", m, n, a, lda, ipiv, info);
}

HWYBLAS_API void slaswp_(const hwyblas_int* n, float* a, const hwyblas_int* lda,
                         const hwyblas_int* k1, const hwyblas_int* k2,
                         const hwyblas_int* ipiv, const hwyblas_int* incx) {
  LaswpEntry<float>("SLASWP", n, a, lda, k1, k2, ipiv, incx);
}

HWYBLAS_API void sgetrs_(const char* trans, const hwyblas_int* n,
                         const hwyblas_int* nrhs, const float* a,
                         const hwyblas_int* lda, const hwyblas_int* ipiv,
                         float* b, const hwyblas_int* ldb, hwyblas_int* info) {
  GetrsEntry<float>("SGETRS", trans, n, nrhs, a, lda, ipiv, b, ldb, info);
}

HWYBLAS_API void sgesv_(const hwyblas_int* n, const hwyblas_int* nrhs, float* a,
                        const hwyblas_int* lda, hwyblas_int* ipiv, float* b,
                        const hwyblas_int* ldb, hwyblas_int* info) {
  GesvEntry<float>("SGESV", n, nrhs, a, lda, ipiv, b, ldb, info);
}

// Complex LU (src/lapack/getrf.cc:548-549).
#define HB_ZLU(P, U, R)                                                                   \
  HWYBLAS_API void P##getrf_(const hwyblas_int* m, const hwyblas_int* n, R* a,            \
                             const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info) { \
    ZGetrfEntry<R>(false, U "GETRF", m, n, a, lda, ipiv, info);                          \
  }                                                                                       \
  HWYBLAS_API void P##getrf2_(const hwyblas_int* m, const hwyblas_int* n, R* a,           \
                              const hwyblas_int* lda, hwyblas_int* ipiv, hwyblas_int* info) { \
    ZGetrfEntry<R>(true, U "GETRF2", m, n, a, lda, ipiv, info);                          \
  }                                                                                       \
  HWYBLAS_API void P##laswp_(const hwyblas_int* n, R* a, const hwyblas_int* lda,          \
                             const hwyblas_int* k1, const hwyblas_int* k2,                \
                             const hwyblas_int* ipiv, const hwyblas_int* incx) {          \
    ZLaswpEntry<R>(U "LASWP", n, a, lda, k1, k2, ipiv, incx);                            \
  }                                                                                       \
  HWYBLAS_API void P##getrs_(const char* trans, const hwyblas_int* n,                     \
                             const hwyblas_int* nrhs, const R* a, const hwyblas_int* lda, \
                             const hwyblas_int* ipiv, R* b, const hwyblas_int* ldb,       \
                             hwyblas_int* info) {                                         \
    ZGetrsEntry<R>(U "GETRS", trans, n, nrhs, a, lda, ipiv, b, ldb, info);               \
  }                                                                                       \
  HWYBLAS_API void P##gesv_(const hwyblas_int* n, const hwyblas_int* nrhs, R* a,          \
                            const hwyblas_int* lda, hwyblas_int* ipiv, R* b,              \
                            const hwyblas_int* ldb, hwyblas_int* info) {                  \
    ZGesvEntry<R>(U "GESV", n, nrhs, a, lda, ipiv, b, ldb, info);                        \
  }
HB_ZLU(z, "Z", double)
HB_ZLU(c, "C", float)
#undef HB_ZLU

#define HB_GERFS(P, U, T)                                                                 \
  HWYBLAS_API void P##gerfs_(const char* trans, const hwyblas_int* n,                     \
                             const hwyblas_int* nrhs, const T* a, const hwyblas_int* lda, \
                             const T* af, const hwyblas_int* ldaf, const hwyblas_int* ipiv, \
                             const T* b, const hwyblas_int* ldb, T* x,                     \
                             const hwyblas_int* ldx, T* ferr, T* berr, T* work,            \
                             hwyblas_int* iwork, hwyblas_int* info) {                      \
    GerfsEntry<T>(#U "GERFS", trans, n, nrhs, a, lda, af, ldaf, ipiv, b, ldb, x, ldx, ferr, \
                  berr, work, iwork, info);                                               \
  }
HB_GERFS(d, D, double)
HB_GERFS(s, S, float)
#undef HB_GERFS

#define HB_GETRI(P, U, T)                                                                 \
  HWYBLAS_API void P##getri_(const hwyblas_int* n, T* a, const hwyblas_int* lda,          \
                             const hwyblas_int* ipiv, T* work, const hwyblas_int* lwork,  \
                             hwyblas_int* info) {                                         \
    GetriEntry<T>(#U "GETRI", n, a, lda, ipiv, work, lwork, info);                        \
  }                                                                                       \
  HWYBLAS_API void P##trtri_(const char* uplo, const char* diag, const hwyblas_int* n,    \
                             T* a, const hwyblas_int* lda, hwyblas_int* info) {           \
    TrtriEntry<T>(false, #U "TRTRI", uplo, diag, n, a, lda, info);                        \
  }                                                                                       \
  HWYBLAS_API void P##trti2_(const char* uplo, const char* diag, const hwyblas_int* n,    \
                             T* a, const hwyblas_int* lda, hwyblas_int* info) {           \
    TrtriEntry<T>(true, #U "TRTI2", uplo, diag, n, a, lda, info);                         \
  }
HB_GETRI(d, D, double)
HB_GETRI(s, S, float)
#undef HB_GETRI

static bool CheckPotrf(const char* name, const char* uplo, int n, int lda,
                       int* info, bool* upper) {
  const char u = hb::Up(*uplo);
  *upper = (u == 'U');
  *info = 0;
  if (!*upper && u != 'L') *info = -1;
  else if (n < 0) *info = -2;
  else if (lda < std::max(1, n)) *info = -4;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return false;
  }
  return true;
}

extern "C++" {
// The Cholesky family for T = double and float (the reference instantiates
// one template for both: src/lapack/potrf.cc:747-773, posv.cc).
template <typename T>
static void PotrfEntry(bool recursive, const char* name, const char* uplo,
                       const hwyblas_int* n_p, T* a, const hwyblas_int* lda_p,
                       hwyblas_int* info) {
  const int n = *n_p, lda = *lda_p;
  bool upper;
  if (!CheckPotrf(name, uplo, n, lda, info, &upper)) return;
  if (n == 0) return;
  hb::Staged<T> sa;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  hb::ResetInfo();
  if (recursive) {
    hb::Potrf2<T>(upper, n, sa.dev, sa.ld, hb::DeviceInfo());
  } else {
    hb::Potrf<T>(upper, n, sa.dev, sa.ld, hb::DeviceInfo());
  }
  sa.Out();
  *info = hb::ReadInfo();
  hb::Finish(name);
}

static bool CheckPos(const char* name, const char* uplo, int n, int nrhs, int lda, int ldb,
                     int* info, bool* upper) {
  const char u = hb::Up(*uplo);
  *upper = (u == 'U');
  *info = 0;
  if (!*upper && u != 'L') *info = -1;
  else if (n < 0) *info = -2;
  else if (nrhs < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  else if (ldb < std::max(1, n)) *info = -7;
  if (*info != 0) {
    hb::ReportError(name, -*info);
    return false;
  }
  return true;
}

template <typename T>
static void PotrsEntry(const char* name, const char* uplo, const hwyblas_int* n_p,
                       const hwyblas_int* nrhs_p, const T* a, const hwyblas_int* lda_p, T* b,
                       const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  bool upper;
  if (!CheckPos(name, uplo, n, nrhs, lda, ldb, info, &upper)) return;
  if (n == 0 || nrhs == 0) return;
  hb::Staged<T> sa, sb;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  hb::Potrs<T>(upper, n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld);
  sb.Out();
  hb::Finish(name);
}

template <typename T>
static void PosvEntry(const char* name, const char* uplo, const hwyblas_int* n_p,
                      const hwyblas_int* nrhs_p, T* a, const hwyblas_int* lda_p, T* b,
                      const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  bool upper;
  if (!CheckPos(name, uplo, n, nrhs, lda, ldb, info, &upper)) return;
  if (n == 0) return;
  hb::Staged<T> sa, sb;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  hb::ResetInfo();
  hb::Potrf<T>(upper, n, sa.dev, sa.ld, hb::DeviceInfo());
  const int finfo = hb::ReadInfo();
  if (finfo == 0 && nrhs > 0) hb::Potrs<T>(upper, n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld);
  sa.Out();
  if (finfo == 0) sb.Out();
  *info = finfo;
  hb::Finish(name);
}
// Complex HERK (src/level3.cc:85-140, 439-452): alpha and beta real.
template <typename R>
static void ZherkEntry(const char* name, const char* uplo, const char* trans,
                       const hwyblas_int* n_p, const hwyblas_int* k_p, const R* alpha,
                       const R* a, const hwyblas_int* lda_p, const R* beta, R* c,
                       const hwyblas_int* ldc_p) {
  const int n = *n_p, k = *k_p, lda = *lda_p, ldc = *ldc_p;
  const char u = hb::Up(*uplo);
  const int op = DecodeOp3(*trans);
  const bool no_trans = op == 0;
  const int rows_a = no_trans ? n : k;
  int info = 0;
  if (u != 'L' && u != 'U') info = 1;
  else if (op != 0 && op != 2) info = 2;
  else if (n < 0) info = 3;
  else if (k < 0) info = 4;
  else if (lda < std::max(1, rows_a)) info = 7;
  else if (ldc < std::max(1, n)) info = 10;
  if (info != 0) {
    hb::ReportError(name, info);
    return;
  }
  const R al = *alpha, be = *beta;
  if (n == 0 || ((al == R(0) || k == 0) && be == R(1))) return;
  const bool reads_a = !(al == R(0) || k == 0);
  ZWorkMatrix<R> sa, sc;
  if (reads_a && !sa.In(const_cast<R*>(a), lda, rows_a, no_trans ? k : n, hb::kWsStageA, true))
    return;
  if (!sc.In(c, ldc, n, n, hb::kWsStageC, true, hb::kWsZFactorB)) return;
  hb::ZherkFull<R>(u == 'L', op, n, k, al, sa.dev, sa.ld, be, sc.dev, sc.ld);
  sc.Out();
  hb::Finish(name);
}

template <typename R>
static void ZPotrfEntry(bool recursive, const char* name, const char* uplo,
                        const hwyblas_int* n_p, R* a, const hwyblas_int* lda_p,
                        hwyblas_int* info) {
  const int n = *n_p, lda = *lda_p;
  bool upper;
  if (!CheckPotrf(name, uplo, n, lda, info, &upper)) return;
  if (n == 0) return;
  ZWorkMatrix<R> sa;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  hb::ResetInfo();
  hb::ZPotrf<R>(recursive, upper, n, sa.dev, sa.ld, hb::DeviceInfo());
  sa.Out();
  *info = hb::ReadInfo();
  hb::Finish(name);
}

template <typename R>
static void ZPotrsEntry(const char* name, const char* uplo, const hwyblas_int* n_p,
                        const hwyblas_int* nrhs_p, const R* a, const hwyblas_int* lda_p, R* b,
                        const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  bool upper;
  if (!CheckPos(name, uplo, n, nrhs, lda, ldb, info, &upper)) return;
  if (n == 0 || nrhs == 0) return;
  ZWorkMatrix<R> sa, sb;
  if (!sa.In(const_cast<R*>(a), lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true, hb::kWsZFactorB)) return;
  hb::ZPotrs<R>(upper, n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld);
  sb.Out();
  hb::Finish(name);
}

template <typename R>
static void ZPosvEntry(const char* name, const char* uplo, const hwyblas_int* n_p,
                       const hwyblas_int* nrhs_p, R* a, const hwyblas_int* lda_p, R* b,
                       const hwyblas_int* ldb_p, hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p;
  bool upper;
  if (!CheckPos(name, uplo, n, nrhs, lda, ldb, info, &upper)) return;
  if (n == 0) return;
  ZWorkMatrix<R> sa, sb;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true, hb::kWsZFactorB)) return;
  hb::ResetInfo();
  hb::ZPotrf<R>(false, upper, n, sa.dev, sa.ld, hb::DeviceInfo());
  const int finfo = hb::ReadInfo();
  if (finfo == 0 && nrhs > 0) hb::ZPotrs<R>(upper, n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld);
  sa.Out();
  if (finfo == 0) sb.Out();
  *info = finfo;
  hb::Finish(name);
}
}  // extern "C++"

HWYBLAS_API void dpotrf_(const char* uplo, const hwyblas_int* n, double* a,
                         const hwyblas_int* lda, hwyblas_int* info) {
  PotrfEntry<double>(false, "DPOTRF", uplo, n, a, lda, info);
}

HWYBLAS_API void dpotrf2_(const char* uplo, const hwyblas_int* n, double* a,
                          const hwyblas_int* lda, hwyblas_int* info) {
  PotrfEntry<double>(true, "DPOTRF2", uplo, n, a, lda, info);
}

HWYBLAS_API void dpotrs_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const double* a, const hwyblas_int* lda, double* b,
                         const hwyblas_int* ldb, hwyblas_int* info) {
  PotrsEntry<double>("DPOTRS", uplo, n, nrhs, a, lda, b, ldb, info);
}

HWYBLAS_API void dposv_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                        double* a, const hwyblas_int* lda, double* b, const hwyblas_int* ldb,
                        hwyblas_int* info) {
  PosvEntry<double>("DPOSV", uplo, n, nrhs, a, lda, b, ldb, info);
}

// Complex Cholesky and HERK (src/lapack/potrf.cc, posv.cc at c64/c32;
// src/level3.cc:439-452).
#define HB_ZCHOL(P, U, R)                                                                 \
  HWYBLAS_API void P##potrf_(const char* uplo, const hwyblas_int* n, R* a,                \
                             const hwyblas_int* lda, hwyblas_int* info) {                 \
    ZPotrfEntry<R>(false, U "POTRF", uplo, n, a, lda, info);                             \
  }                                                                                       \
  HWYBLAS_API void P##potrf2_(const char* uplo, const hwyblas_int* n, R* a,               \
                              const hwyblas_int* lda, hwyblas_int* info) {                \
    ZPotrfEntry<R>(true, U "POTRF2", uplo, n, a, lda, info);                             \
  }                                                                                       \
  HWYBLAS_API void P##potrs_(const char* uplo, const hwyblas_int* n,                      \
                             const hwyblas_int* nrhs, const R* a, const hwyblas_int* lda, \
                             R* b, const hwyblas_int* ldb, hwyblas_int* info) {           \
    ZPotrsEntry<R>(U "POTRS", uplo, n, nrhs, a, lda, b, ldb, info);                      \
  }                                                                                       \
  HWYBLAS_API void P##posv_(const char* uplo, const hwyblas_int* n,                       \
                            const hwyblas_int* nrhs, R* a, const hwyblas_int* lda, R* b,  \
                            const hwyblas_int* ldb, hwyblas_int* info) {                  \
    ZPosvEntry<R>(U "POSV", uplo, n, nrhs, a, lda, b, ldb, info);                        \
  }                                                                                       \
  HWYBLAS_API void P##herk_(const char* uplo, const char* trans, const hwyblas_int* n,    \
                            const hwyblas_int* k, const R* alpha, const R* a,             \
                            const hwyblas_int* lda, const R* beta, R* c,                  \
                            const hwyblas_int* ldc) {                                     \
    ZherkEntry<R>(U "HERK", uplo, trans, n, k, alpha, a, lda, beta, c, ldc);             \
  }
HB_ZCHOL(z, "Z", double)
HB_ZCHOL(c, "C", float)
#undef HB_ZCHOL

// CBLAS complex HERK (src/cblas.cc:610-630, 1825-1841): row-major flips the
// triangle and swaps N and C (an invalid T stays invalid); error positions
// are the CBLAS argument numbers.
extern "C++" {
template <typename R>
static void CblasZherk(const char* name, const char* routine, CBLAS_LAYOUT layout,
                       CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans, hwyblas_int n, hwyblas_int k,
                       R alpha, const void* a, hwyblas_int lda, R beta, void* c,
                       hwyblas_int ldc) {
  if (!hb::ValidLayout(name, layout)) return;
  char uc = hb::UploChar(uplo), tc = hb::TransChar(trans);
  if (layout == CblasRowMajor) {
    uc = hb::FlipUplo(uc);
    if (tc == 'N') tc = 'C';
    else if (tc == 'C') tc = 'N';
  }
  hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11});
  ZherkEntry<R>(routine, &uc, &tc, &n, &k, &alpha, static_cast<const R*>(a), &lda, &beta,
                static_cast<R*>(c), &ldc);
}
}  // extern "C++"
HWYBLAS_API void cblas_zherk(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                             hwyblas_int n, hwyblas_int k, double alpha, const void* a,
                             hwyblas_int lda, double beta, void* c, hwyblas_int ldc) {
  CblasZherk<double>("cblas_zherk", "ZHERK", layout, uplo, trans, n, k, alpha, a, lda, beta,
                     c, ldc);
}
HWYBLAS_API void cblas_cherk(CBLAS_LAYOUT layout, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans,
                             hwyblas_int n, hwyblas_int k, float alpha, const void* a,
                             hwyblas_int lda, float beta, void* c, hwyblas_int ldc) {
  CblasZherk<float>("cblas_cherk", "CHERK", layout, uplo, trans, n, k, alpha, a, lda, beta,
                    c, ldc);
}

HWYBLAS_API void spotrf_(const char* uplo, const hwyblas_int* n, float* a,
                         const hwyblas_int* lda, hwyblas_int* info) {
  PotrfEntry<float>(false, "SPOTRF", uplo, n, a, lda, info);
}

HWYBLAS_API void spotrf2_(const char* uplo, const hwyblas_int* n, float* a,
                          const hwyblas_int* lda, hwyblas_int* info) {
  PotrfEntry<float>(true, "SPOTRF2", uplo, n, a, lda, info);
}

HWYBLAS_API void spotrs_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                         const float* a, const hwyblas_int* lda, float* b,
                         const hwyblas_int* ldb, hwyblas_int* info) {
  PotrsEntry<float>("SPOTRS", uplo, n, nrhs, a, lda, b, ldb, info);
}

HWYBLAS_API void sposv_(const char* uplo, const hwyblas_int* n, const hwyblas_int* nrhs,
                        float* a, const hwyblas_int* lda, float* b, const hwyblas_int* ldb,
                        hwyblas_int* info) {
  PosvEntry<float>("SPOSV", uplo, n, nrhs, a, lda, b, ldb, info);
}

// ---------------------------------------------------------------------------
// CBLAS.

HWYBLAS_API void cblas_xerbla(hwyblas_int p, const char* rout, const char* form,
                              ...) {
  if (p != 0) {
    fprintf(stderr, "Parameter %d to routine %s was incorrect\n",
            static_cast<int>(p), rout);
  }
  if (form != nullptr && *form != '\0') {
    va_list args;
    va_start(args, form);
    vfprintf(stderr, form, args);
    va_end(args);
  }
}


HWYBLAS_API void cblas_dgemm(const CBLAS_LAYOUT layout,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k,
                             const double alpha, const double* a,
                             const hwyblas_int lda, const double* b,
                             const hwyblas_int ldb, const double beta,
                             double* c, const hwyblas_int ldc) {
  hb::CblasGemm<double>("cblas_dgemm", layout, transa, transb, m, n, k, alpha, a,
                    lda, b, ldb, beta, c, ldc);
}

HWYBLAS_API void cblas_sgemm(const CBLAS_LAYOUT layout,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_TRANSPOSE transb, const hwyblas_int m,
                             const hwyblas_int n, const hwyblas_int k,
                             const float alpha, const float* a,
                             const hwyblas_int lda, const float* b,
                             const hwyblas_int ldb, const float beta, float* c,
                             const hwyblas_int ldc) {
  hb::CblasGemm<float>("cblas_sgemm", layout, transa, transb, m, n, k, alpha, a,
                   lda, b, ldb, beta, c, ldc);
}

extern "C++" {
template <typename T>
static void CblasTrsm(const char* name, const char* routine, const CBLAS_LAYOUT layout,
                      const CBLAS_SIDE side, const CBLAS_UPLO uplo,
                      const CBLAS_TRANSPOSE transa, const CBLAS_DIAG diag,
                      const hwyblas_int m_in, const hwyblas_int n_in, const T alpha,
                      const T* a, const hwyblas_int lda, T* b, const hwyblas_int ldb) {
  if (!hb::ValidLayout(name, layout)) return;
  char sc = hb::SideChar(side), uc = hb::UploChar(uplo);
  const char tc = hb::TransChar(transa), dc = hb::DiagChar(diag);
  int m = m_in, n = n_in;
  const bool row = (layout == CblasRowMajor);
  if (row) {
    sc = hb::FlipSide(sc);
    uc = hb::FlipUplo(uc);
    std::swap(m, n);
  }
  if (row) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 7, 6, 8, 9, 10, 11, 12});
    hb::TrsmEntry<T>(routine, &sc, &uc, &tc, &dc, &m, &n, &alpha, a, &lda, b, &ldb);
  } else {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12});
    hb::TrsmEntry<T>(routine, &sc, &uc, &tc, &dc, &m, &n, &alpha, a, &lda, b, &ldb);
  }
}

// CBLAS TRMM (src/cblas.cc:666-700): row-major is B^T := alpha B^T op(A)^T with
// the other side and triangle; op is unchanged.
template <typename T>
static void CblasTrmm(const char* name, const char* routine, const CBLAS_LAYOUT layout,
                      const CBLAS_SIDE side, const CBLAS_UPLO uplo,
                      const CBLAS_TRANSPOSE transa, const CBLAS_DIAG diag,
                      const hwyblas_int m_in, const hwyblas_int n_in, const T alpha,
                      const T* a, const hwyblas_int lda, T* b, const hwyblas_int ldb) {
  if (!hb::ValidLayout(name, layout)) return;
  char sc = hb::SideChar(side), uc = hb::UploChar(uplo);
  const char tc = hb::TransChar(transa), dc = hb::DiagChar(diag);
  int m = m_in, n = n_in;
  const bool row = (layout == CblasRowMajor);
  if (row) {
    sc = hb::FlipSide(sc);
    uc = hb::FlipUplo(uc);
    std::swap(m, n);
  }
  if (row) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 7, 6, 8, 9, 10, 11, 12});
    TrmmEntry<T>(routine, &sc, &uc, &tc, &dc, &m, &n, &alpha, a, &lda, b, &ldb);
  } else {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12});
    TrmmEntry<T>(routine, &sc, &uc, &tc, &dc, &m, &n, &alpha, a, &lda, b, &ldb);
  }
}

// CBLAS SYMM (src/cblas.cc:562-607): row-major is C^T = B^T A^T, A stored as
// the other triangle, with the other side and m, n swapped.
template <typename T>
static void CblasSymm(const char* name, const char* routine, const CBLAS_LAYOUT layout,
                      const CBLAS_SIDE side, const CBLAS_UPLO uplo, const hwyblas_int m_in,
                      const hwyblas_int n_in, const T alpha, const T* a,
                      const hwyblas_int lda, const T* b, const hwyblas_int ldb, const T beta,
                      T* c, const hwyblas_int ldc) {
  if (!hb::ValidLayout(name, layout)) return;
  char sc = hb::SideChar(side), uc = hb::UploChar(uplo);
  int m = m_in, n = n_in;
  const bool row = (layout == CblasRowMajor);
  if (row) {
    sc = hb::FlipSide(sc);
    uc = hb::FlipUplo(uc);
    std::swap(m, n);
  }
  if (row) {
    hb::CblasScope scope(name, {2, 3, 5, 4, 6, 7, 8, 9, 10, 11, 12, 13});
    SymmEntry<T>(routine, &sc, &uc, &m, &n, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
  } else {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13});
    SymmEntry<T>(routine, &sc, &uc, &m, &n, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
  }
}

// CBLAS SYR2K (src/cblas.cc:632-664): row-major flips uplo and N <-> T.
template <typename T>
static void CblasSyr2k(const char* name, const char* routine, const CBLAS_LAYOUT layout,
                       const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE trans,
                       const hwyblas_int n, const hwyblas_int k, const T alpha, const T* a,
                       const hwyblas_int lda, const T* b, const hwyblas_int ldb,
                       const T beta, T* c, const hwyblas_int ldc) {
  if (!hb::ValidLayout(name, layout)) return;
  char uc = hb::UploChar(uplo), tc = hb::TransChar(trans);
  if (layout == CblasRowMajor) {
    uc = hb::FlipUplo(uc);
    tc = (tc == 'N') ? 'T' : (tc == 'T' || tc == 'C') ? 'N' : tc;
  }
  hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13});
  Syr2kEntry<T>(routine, &uc, &tc, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
}

// CBLAS GEMMTR / GEMMT (src/cblas.cc:539-566): row-major is the column-major
// product of the swapped operands on the other triangle.
template <typename T>
static void CblasGemmtr(const char* name, const char* routine, const CBLAS_LAYOUT layout,
                        const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,
                        const CBLAS_TRANSPOSE transb, const hwyblas_int n,
                        const hwyblas_int k, const T alpha, const T* a,
                        const hwyblas_int lda, const T* b, const hwyblas_int ldb, const T beta,
                        T* c, const hwyblas_int ldc) {
  if (!hb::ValidLayout(name, layout)) return;
  const char ta = hb::TransChar(transa), tb = hb::TransChar(transb);
  const char uc = hb::UploChar(uplo);
  if (layout == CblasColMajor) {
    hb::CblasScope scope(name, {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14});
    GemmtrEntry<T>(routine, &uc, &ta, &tb, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc);
  } else {
    const char ur = hb::FlipUplo(uc);
    hb::CblasScope scope(name, {2, 4, 3, 5, 6, 7, 10, 11, 8, 9, 12, 13, 14});
    GemmtrEntry<T>(routine, &ur, &tb, &ta, &n, &k, &alpha, b, &ldb, a, &lda, &beta, c, &ldc);
  }
}
}  // extern "C++"

HWYBLAS_API void cblas_dtrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m_in,
                             const hwyblas_int n_in, const double alpha,
                             const double* a, const hwyblas_int lda, double* b,
                             const hwyblas_int ldb) {
  CblasTrsm<double>("cblas_dtrsm", "DTRSM", layout, side, uplo, transa, diag, m_in, n_in,
                    alpha, a, lda, b, ldb);
}

HWYBLAS_API void cblas_strsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side,
                             const CBLAS_UPLO uplo,
                             const CBLAS_TRANSPOSE transa,
                             const CBLAS_DIAG diag, const hwyblas_int m_in,
                             const hwyblas_int n_in, const float alpha,
                             const float* a, const hwyblas_int lda, float* b,
                             const hwyblas_int ldb) {
  CblasTrsm<float>("cblas_strsm", "STRSM", layout, side, uplo, transa, diag, m_in, n_in,
                   alpha, a, lda, b, ldb);
}

#define HB_CBLAS_L3(P, U, T)                                                                \
  HWYBLAS_API void cblas_##P##trmm(                                                         \
      const CBLAS_LAYOUT layout, const CBLAS_SIDE side, const CBLAS_UPLO uplo,              \
      const CBLAS_TRANSPOSE transa, const CBLAS_DIAG diag, const hwyblas_int m,             \
      const hwyblas_int n, const T alpha, const T* a, const hwyblas_int lda, T* b,          \
      const hwyblas_int ldb) {                                                              \
    CblasTrmm<T>("cblas_" #P "trmm", #U "TRMM", layout, side, uplo, transa, diag, m, n,   \
                 alpha, a, lda, b, ldb);                                                    \
  }                                                                                         \
  HWYBLAS_API void cblas_##P##symm(                                                         \
      const CBLAS_LAYOUT layout, const CBLAS_SIDE side, const CBLAS_UPLO uplo,              \
      const hwyblas_int m, const hwyblas_int n, const T alpha, const T* a,                  \
      const hwyblas_int lda, const T* b, const hwyblas_int ldb, const T beta, T* c,         \
      const hwyblas_int ldc) {                                                              \
    CblasSymm<T>("cblas_" #P "symm", #U "SYMM", layout, side, uplo, m, n, alpha, a, lda,  \
                 b, ldb, beta, c, ldc);                                                     \
  }                                                                                         \
  HWYBLAS_API void cblas_##P##syr2k(                                                        \
      const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE trans,        \
      const hwyblas_int n, const hwyblas_int k, const T alpha, const T* a,                  \
      const hwyblas_int lda, const T* b, const hwyblas_int ldb, const T beta, T* c,         \
      const hwyblas_int ldc) {                                                              \
    CblasSyr2k<T>("cblas_" #P "syr2k", #U "SYR2K", layout, uplo, trans, n, k, alpha, a,   \
                  lda, b, ldb, beta, c, ldc);                                               \
  }                                                                                         \
  HWYBLAS_API void cblas_##P##gemmtr(                                                       \
      const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,       \
      const CBLAS_TRANSPOSE transb, const hwyblas_int n, const hwyblas_int k,               \
      const T alpha, const T* a, const hwyblas_int lda, const T* b, const hwyblas_int ldb,  \
      const T beta, T* c, const hwyblas_int ldc) {                                          \
    CblasGemmtr<T>("cblas_" #P "gemmtr", #U "GEMMTR", layout, uplo, transa, transb, n, k, \
                   alpha, a, lda, b, ldb, beta, c, ldc);                                    \
  }                                                                                         \
  HWYBLAS_API void cblas_##P##gemmt(                                                        \
      const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE transa,       \
      const CBLAS_TRANSPOSE transb, const hwyblas_int n, const hwyblas_int k,               \
      const T alpha, const T* a, const hwyblas_int lda, const T* b, const hwyblas_int ldb,  \
      const T beta, T* c, const hwyblas_int ldc) {                                          \
    CblasGemmtr<T>("cblas_" #P "gemmt", #U "GEMMT", layout, uplo, transa, transb, n, k,   \
                   alpha, a, lda, b, ldb, beta, c, ldc);                                    \
  }

HB_CBLAS_L3(d, D, double)
HB_CBLAS_L3(s, S, float)
#undef HB_CBLAS_L3

HWYBLAS_API CBLAS_INDEX cblas_idamax(const hwyblas_int n, const double* x,
                                     const hwyblas_int incx) {
  const hwyblas_int i = idamax_(&n, x, &incx);
  return i > 0 ? static_cast<CBLAS_INDEX>(i - 1) : 0;
}

// ---------------------------------------------------------------------------
// Extensions.

HWYBLAS_API hwyblas_int hwyblas_dgemm_emulated(
    const char* transa, const char* transb, const hwyblas_int* m_p,
    const hwyblas_int* n_p, const hwyblas_int* k_p, const double* alpha_p,
    const double* a, const hwyblas_int* lda_p, const double* b,
    const hwyblas_int* ldb_p, const double* beta_p, double* c,
    const hwyblas_int* ldc_p, const hwyblas_int* slices_p) {
  const int m = *m_p, n = *n_p, k = *k_p, lda = *lda_p, ldb = *ldb_p,
            ldc = *ldc_p, slices = *slices_p;
  bool ta, tb;
  const bool va = hb::DecodeOp(*transa, &ta), vb = hb::DecodeOp(*transb, &tb);
  const int rows_a = ta ? k : m, rows_b = tb ? n : k;
  int info = 0;
  if (!va) info = 1;
  else if (!vb) info = 2;
  else if (m < 0) info = 3;
  else if (n < 0) info = 4;
  else if (k < 0) info = 5;
  else if (lda < std::max(1, rows_a)) info = 8;
  else if (ldb < std::max(1, rows_b)) info = 10;
  else if (ldc < std::max(1, m)) info = 13;
  else if (slices < 0 || slices > 8) info = 14;
  if (info != 0) {
    hb::ReportError("DGEMM_EMULATED", info);
    return -1;
  }
  const double alpha = *alpha_p, beta = *beta_p;
  if (m == 0 || n == 0) return 0;
  if ((k == 0 || alpha == 0.0) && beta == 1.0) return 0;
  hb::Staged<double> sa, sb, sc;
  const bool compute = !(k == 0 || alpha == 0.0);
  if (compute) {
    if (!sa.In(a, lda, rows_a, ta ? m : k, hb::kWsStageA, true)) return -1;
    if (!sb.In(b, ldb, rows_b, tb ? k : n, hb::kWsStageB, true)) return -1;
  }
  if (!sc.In(c, ldc, m, n, hb::kWsStageC, beta != 0.0)) return -1;
  int used = 0;
  long long copied = 0;  // columns of a host C already queued back
  if (!compute) {
    hb::ScaleMatrix<double>(m, n, beta, sc.dev, sc.ld, hb::kAll);
  } else {
    // A host C large enough for a few waves of tiles per block goes back in
    // column blocks on the side stream, each while the next is computed.
    hb::SideStream& side = hb::Side();
    int col_blocks = 1;
    std::function<void(int, int)> done;
    if (sc.host && side.ok) {
      const long long tiles = static_cast<long long>((m + 127) / 128) * ((n + 127) / 128);
      col_blocks = static_cast<int>(
          std::min<long long>(4, tiles / (6LL * hb::Ctx().num_sms)));
      done = [&](int n0, int nb) {
        cudaEventRecord(side.to_side, hb::Ctx().stream);
        cudaStreamWaitEvent(side.stream, side.to_side, 0);
        if (!hb::Failed(cudaMemcpy2DAsync(c + static_cast<long long>(n0) * ldc,
                                          sizeof(double) * ldc,
                                          sc.dev + static_cast<long long>(n0) * sc.ld,
                                          sizeof(double) * sc.ld, sizeof(double) * m, nb,
                                          cudaMemcpyDeviceToHost, side.stream),
                        "copy out"))
          copied += nb;
      };
    }
    // slices == 0: chosen from the inputs' exponent spread (emulated.cu).
    used = hb::DgemmEmulated(m, n, k, alpha, hb::ColMajor<double>(sa.dev, sa.ld, ta),
                             hb::ColMajor<double>(sb.dev, sb.ld, tb), beta, sc.dev,
                             sc.ld, slices, true, 0, false, col_blocks,
                             col_blocks > 1 ? &done : nullptr);
    if (copied > 0) {
      cudaEventRecord(side.to_main, side.stream);
      cudaStreamWaitEvent(hb::Ctx().stream, side.to_main, 0);
    }
  }
  if (copied != n) sc.Out();
  hb::Finish("DGEMM_EMULATED");
  return used;
}

// Slice count of the mixed solvers' trailing updates (calling thread).
static thread_local int t_mixed_slices = 4;

HWYBLAS_API int hwyblas_set_mixed_slices(int slices) {
  const int prev = t_mixed_slices;
  if (slices >= 1 && slices <= 8) t_mixed_slices = slices;
  return prev;
}

HWYBLAS_API void hwyblas_dgesv_mixed(const hwyblas_int* n_p, const hwyblas_int* nrhs_p,
                                     double* a, const hwyblas_int* lda_p,
                                     hwyblas_int* ipiv, const double* b,
                                     const hwyblas_int* ldb_p, double* x,
                                     const hwyblas_int* ldx_p, hwyblas_int* iter,
                                     hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p, ldx = *ldx_p;
  *info = 0;
  *iter = 0;
  if (n < 0) *info = -1;
  else if (nrhs < 0) *info = -2;
  else if (lda < std::max(1, n)) *info = -4;
  else if (ldb < std::max(1, n)) *info = -7;
  else if (ldx < std::max(1, n)) *info = -9;
  if (*info != 0) {
    hb::ReportError("DGESV_MIXED", -*info);
    return;
  }
  if (n == 0) return;
  hb::Staged<double> sa, sb, sx;
  hb::StagedInts sp;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sx.In(x, ldx, n, nrhs, hb::kWsStageX, false)) return;
  if (!sp.In(ipiv, n, 0, false)) return;
  int it = 0;
  const int finfo = hb::DgesvMixed(n, nrhs, sa.dev, sa.ld, sp.dev, sb.dev, sb.ld,
                                   sx.dev, sx.ld, t_mixed_slices, &it);
  if (finfo < 0) {
    hb::Finish("DGESV_MIXED");
    return;
  }
  if (it < 0) sa.Out();  // the FP64 factors, as DSGESV leaves them
  sp.Out();
  if (finfo == 0 && nrhs > 0) sx.Out();
  *iter = it;
  *info = finfo;
  hb::Finish("DGESV_MIXED");
}

HWYBLAS_API void hwyblas_dposv_mixed(const char* uplo, const hwyblas_int* n_p,
                                     const hwyblas_int* nrhs_p, double* a,
                                     const hwyblas_int* lda_p, const double* b,
                                     const hwyblas_int* ldb_p, double* x,
                                     const hwyblas_int* ldx_p, hwyblas_int* iter,
                                     hwyblas_int* info) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldb = *ldb_p, ldx = *ldx_p;
  const char u = hb::Up(*uplo);
  const bool upper = (u == 'U');
  *info = 0;
  *iter = 0;
  if (!upper && u != 'L') *info = -1;
  else if (n < 0) *info = -2;
  else if (nrhs < 0) *info = -3;
  else if (lda < std::max(1, n)) *info = -5;
  else if (ldb < std::max(1, n)) *info = -7;
  else if (ldx < std::max(1, n)) *info = -9;
  if (*info != 0) {
    hb::ReportError("DPOSV_MIXED", -*info);
    return;
  }
  if (n == 0) return;
  hb::Staged<double> sa, sb, sx;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sx.In(x, ldx, n, nrhs, hb::kWsStageX, false)) return;
  int it = 0;
  const int finfo = hb::DposvMixed(upper, n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld,
                                   sx.dev, sx.ld, t_mixed_slices, &it);
  if (finfo < 0) {
    hb::Finish("DPOSV_MIXED");
    return;
  }
  if (it < 0) sa.Out();
  if (finfo == 0 && nrhs > 0) sx.Out();
  *iter = it;
  *info = finfo;
  hb::Finish("DPOSV_MIXED");
}

HWYBLAS_API void hwyblas_dgemm_ddref(const char* transa, const char* transb,
                                     const hwyblas_int* m_p,
                                     const hwyblas_int* ncols_p,
                                     const hwyblas_int* k_p, const double* a,
                                     const hwyblas_int* lda_p, const double* b,
                                     const hwyblas_int* ldb_p,
                                     const hwyblas_int* n_p,
                                     const hwyblas_int* cols, double* out,
                                     const hwyblas_int* ldo_p) {
  const int m = *m_p, ncols = *ncols_p, k = *k_p, lda = *lda_p, ldb = *ldb_p,
            n = *n_p, ldo = *ldo_p;
  bool ta, tb;
  hb::DecodeOp(*transa, &ta);
  hb::DecodeOp(*transb, &tb);
  if (m <= 0 || ncols <= 0 || k <= 0 || n <= 0) return;
  hb::Staged<double> sa, sb, so;
  hb::StagedInts sj;
  if (!sa.In(a, lda, ta ? k : m, ta ? m : k, hb::kWsStageA, true)) return;
  if (!sb.In(b, ldb, tb ? n : k, tb ? k : n, hb::kWsStageB, true)) return;
  if (!so.In(out, ldo, m, ncols, hb::kWsStageC, false)) return;
  if (!sj.In(cols, ncols, 0, true)) return;
  hb::DgemmDoubleDouble(m, ncols, k, hb::ColMajor<double>(sa.dev, sa.ld, ta),
                        hb::ColMajor<double>(sb.dev, sb.ld, tb), sj.dev, so.dev,
                        so.ld);
  so.Out();
  hb::Finish("DGEMM_DDREF");
}

HWYBLAS_API void hwyblas_dresidual_dd(const hwyblas_int* n_p, const hwyblas_int* nrhs_p,
                                      const double* a, const hwyblas_int* lda_p,
                                      const double* x, const hwyblas_int* ldx_p,
                                      const double* b, const hwyblas_int* ldb_p, double* r,
                                      const hwyblas_int* ldr_p) {
  const int n = *n_p, nrhs = *nrhs_p, lda = *lda_p, ldx = *ldx_p, ldb = *ldb_p,
            ldr = *ldr_p;
  int info = 0;
  if (n < 0) info = 1;
  else if (nrhs < 0) info = 2;
  else if (lda < std::max(1, n)) info = 4;
  else if (ldx < std::max(1, n)) info = 6;
  else if (ldb < std::max(1, n)) info = 8;
  else if (ldr < std::max(1, n)) info = 10;
  if (info != 0) {
    hb::ReportError("DRESIDUAL_DD", info);
    return;
  }
  if (n == 0 || nrhs == 0) return;
  hb::Staged<double> sa, sx, sb, sr;
  if (!sa.In(a, lda, n, n, hb::kWsStageA, true)) return;
  if (!sx.In(x, ldx, n, nrhs, hb::kWsStageX, true)) return;
  if (!sb.In(b, ldb, n, nrhs, hb::kWsStageB, true)) return;
  if (!sr.In(r, ldr, n, nrhs, hb::kWsStageC, false)) return;
  double* part = static_cast<double*>(
      hb::Workspace(hb::kWsResidual, hb::ResidualDdPartBytes(n, nrhs)));
  if (part == nullptr) return;
  hb::ResidualDd(n, nrhs, sa.dev, sa.ld, sb.dev, sb.ld, sx.dev, sx.ld, sr.dev, sr.ld, part);
  sr.Out();
  hb::Finish("DRESIDUAL_DD");
}

HWYBLAS_API void hwyblas_set_stream(void* stream) {
  hb::Context& c = Ctx();
  c.stream = stream != nullptr ? static_cast<cudaStream_t>(stream) : c.own_stream;
}

HWYBLAS_API unsigned int hwyblas_set_leaf_wait_limit(unsigned int polls) {
  Ctx();
  return hb::SetLeafWaitLimit(polls);
}

HWYBLAS_API int hwyblas_last_cuda_error(void) {
  hb::Context& c = Ctx();
  const int e = c.last_error;
  c.last_error = 0;
  return e;
}

HWYBLAS_API void hwyblas_kernel_timer(int family) {
  std::lock_guard<std::mutex> lock(hb::g_timer_mu);
  hb::g_timer_family = family;
}

HWYBLAS_API double hwyblas_kernel_timer_read(int* launches) {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  {
    std::lock_guard<std::mutex> lock(hb::g_timer_mu);
    ev.swap(hb::g_timer_events);
  }
  double total = 0.0;
  for (auto& pr : ev) {
    float ms = 0.0f;
    cudaEventSynchronize(pr.second);
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) total += ms;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  if (launches != nullptr) *launches = static_cast<int>(ev.size());
  return total;
}

HWYBLAS_API uint64_t hwyblas_launch_count(void) {
  return hb::g_launches.load(std::memory_order_relaxed);
}

}  // extern "C"
