// Iterative refinement with error bounds (xGERFS, src/lapack/gesvx.cc:
// 319-456) and its condition estimator (xLACN2, src/lapack/trsen.cc:
// 2243-2366), real types, on the device.
//
// Per right-hand side: r = b - op(A) x and w = |b| + |op(A)| |x| (one pass
// over A), BERR = max_i |r_i| / w_i (with the safe-minimum guard), and while
// BERR > eps, it halves and fewer than 5 steps were taken, x += op(A)^-1 r
// through the LU factors. Then FERR: LACN2 estimates
// || inv(op(A)) diag(|r| + (n+1) eps w) ||_inf by reverse communication,
// each step being one solve with the factors; LACN2's control flow (a few
// integers and comparisons of scalars) runs on the host and every vector
// operation on the device.
//
// Rounding follows the reference: the op N residual is the GEMV axpy chain
// (fma per column in order, t = -x), the op T residual the GEMV dot form
// (lane l of N = 8 doubles / 16 floats chains rows i = l mod N, lanes summed
// by halves), w and the transposed sums are scalar loops with separate
// roundings, ASUM keeps four lane vectors as the reference's kernel, and the
// maxima are taken in index order with a > b ? a : b, so NaNs behave alike.
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace hb {

int RefLanesDouble();

namespace {

template <typename T>
__device__ __forceinline__ T MulR(T x, T y) {
  if constexpr (sizeof(T) == 8) return __dmul_rn(x, y);
  else return __fmul_rn(x, y);
}
template <typename T>
__device__ __forceinline__ T AddR(T x, T y) {
  if constexpr (sizeof(T) == 8) return __dadd_rn(x, y);
  else return __fadd_rn(x, y);
}
template <typename T>
__device__ __forceinline__ T FmaR(T x, T y, T z) {
  if constexpr (sizeof(T) == 8) return fma(x, y, z);
  else return fmaf(x, y, z);
}

// op N: r = b - A x (GEMV axpy chain), w = |b| + |A| |x| (column order).
template <typename T>
__global__ void ResidualNKernel(int n, const T* a, long long lda, const T* x, const T* b,
                                T* r, T* w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T y = b[i], s = fabs(b[i]);
  for (int k = 0; k < n; ++k) {
    const T aik = a[i + k * lda], xk = x[k];
    y = FmaR(aik, -xk, y);
    s = AddR(s, MulR(fabs(aik), fabs(xk)));
  }
  r[i] = y;
  w[i] = s;
}

// op T, residual: r_c = b_c + (-1 * dot(A(:, c), x)) with the dot in the
// GEMV dot form's lanes. `lanes` threads per column.
template <typename T>
__global__ void ResidualTKernel(int n, const T* a, long long lda, const T* x, const T* b, T* r,
                                int lanes) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = gt / lanes, l = gt % lanes;
  const bool active = c < n;
  T s = T(0);
  if (active) {
    const T* col = a + static_cast<long long>(c) * lda;
    const int full = n / lanes * lanes;
    for (int i = l; i < full; i += lanes) s = FmaR(col[i], x[i], s);
    if (full < n) {
      const int i = full + l;
      s = (i < n) ? FmaR(col[i], x[i], s) : FmaR(T(0), T(0), s);
    }
  }
  // Lane sum by halves: lane l takes lane l + h for h = lanes/2, ..., 1.
  for (int h = lanes / 2; h >= 1; h /= 2) {
    const T o = __shfl_down_sync(0xffffffffu, s, h, lanes);
    if (l < h) s = AddR(s, o);
  }
  if (active && l == 0) r[c] = AddR(b[c], MulR(T(-1), s));
}

// op T, w_k = |b_k| + sum_i |A(i, k)| |x_i| (the sum in row order).
template <typename T>
__global__ void AbsSumTKernel(int n, const T* a, long long lda, const T* x, const T* b, T* w) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const T* col = a + static_cast<long long>(k) * lda;
  T s = T(0);
  for (int i = 0; i < n; ++i) s = AddR(s, MulR(fabs(col[i]), fabs(x[i])));
  w[k] = AddR(fabs(b[k]), s);
}

// out[0] = max over i (in order, a > b ? a : b) of the componentwise
// backward error terms.
template <typename T>
__global__ void BerrKernel(int n, const T* r, const T* w, T safe1, T safe2, T* q, T* out) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    q[i] = (w[i] > safe2) ? fabs(r[i]) / w[i]
                          : AddR(fabs(r[i]), safe1) / AddR(w[i], safe1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T s = T(0);
    for (int i = 0; i < n; ++i) s = (s > q[i]) ? s : q[i];
    out[0] = s;
  }
}

// out[0] = max over i (in order) of |x_i|.
template <typename T>
__global__ void MaxAbsKernel(int n, const T* x, T* out) {
  T s = T(0);
  for (int i = 0; i < n; ++i) {
    const T v = fabs(x[i]);
    s = (s > v) ? s : v;
  }
  out[0] = s;
}

// AXPY in the reference's kernel order: blocks of 2 vectors as fma(alpha, x,
// y), the rest as y + alpha * x.
template <typename T>
__global__ void AxpyRefKernel(int n, T alpha, const T* x, T* y, int lanes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int blocked = n / (2 * lanes) * (2 * lanes);
  y[i] = (i < blocked) ? FmaR(alpha, x[i], y[i]) : AddR(y[i], MulR(x[i], alpha));
}

// w_i := |r_i| + (n+1) eps w_i (+ safe1 where w_i <= safe2).
template <typename T>
__global__ void FerrWeightKernel(int n, const T* r, T* w, T nzeps, T safe1, T safe2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T wi = w[i];
  const T v = AddR(fabs(r[i]), MulR(nzeps, wi));
  w[i] = (wi > safe2) ? v : AddR(v, safe1);
}

template <typename T>
__global__ void DiagScaleKernel(int n, const T* w, T* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = MulR(w[i], x[i]);
}

// ASUM in the reference kernel's order: lane vectors s0..s3 over blocks of
// 4 vectors, whole remaining vectors into s0, the zero-padded tail into s1,
// (s0 + s1) + (s2 + s3) per lane, lanes summed by halves. One thread per
// (vector, lane) slot; out[0] receives the sum.
template <typename T>
__global__ void AsumRefKernel(int n, const T* x, int lanes, T* out) {
  __shared__ T part[4][32];
  const int slot = threadIdx.x;  // 4 * lanes threads
  const int vec = slot / lanes, l = slot % lanes;
  const int blk = 4 * lanes;
  const int nblk = n / blk * blk;
  T s = T(0);
  for (int i = vec * lanes + l; i < nblk; i += blk) s = AddR(fabs(x[i]), s);
  const int tail = nblk + (n - nblk) / lanes * lanes;  // start of the partial vector
  if (vec == 0)
    for (int i = nblk; i < tail; i += lanes) s = AddR(fabs(x[i + l]), s);
  if (vec == 1 && tail < n) s = AddR((tail + l < n) ? fabs(x[tail + l]) : T(0), s);
  part[vec][l] = s;
  __syncthreads();
  if (slot == 0) {
    T lane[32];
    for (int k = 0; k < lanes; ++k)
      lane[k] = AddR(AddR(part[0][k], part[1][k]), AddR(part[2][k], part[3][k]));
    for (int h = lanes / 2; h >= 1; h /= 2)
      for (int k = 0; k < h; ++k) lane[k] = AddR(lane[k], lane[k + h]);
    out[0] = lane[0];
  }
}

// LACN2's vector steps.
template <typename T>
__global__ void FillKernel(int n, T v, T* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}
template <typename T>
__global__ void SignKernel(int n, T* x, int* isgn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T v = (x[i] >= T(0)) ? T(1) : T(-1);
  x[i] = v;
  isgn[i] = (v > T(0)) ? 1 : -1;
}
template <typename T>
__global__ void SignChangedKernel(int n, const T* x, const int* isgn, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = (x[i] >= T(0)) ? 1 : -1;
  if (s != isgn[i]) atomicExch(flag, 1);
}
template <typename T>
__global__ void UnitVectorKernel(int n, int j, T* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = (i == j) ? T(1) : T(0);
}
// x_i = (+1, -1, +1, ...) * (1 + i / (n - 1)).
template <typename T>
__global__ void AltSignKernel(int n, T* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T v = AddR(T(1), T(i) / T(n - 1));
  x[i] = (i % 2 == 0) ? v : -v;
}

int Blocks(int n) { return (n + 255) / 256; }

// Device buffers of one GERFS call.
template <typename T>
struct RefineBufs {
  T* rw;   // w: |b| + |op(A)||x|, then the FERR weights
  T* wk;   // residual, then LACN2's x
  T* vv;   // LACN2's v
  T* q;    // BERR terms
  T* sc;   // scalars
  int* isgn;
  int* flag;
};

template <typename T>
T ReadScalar(const T* d) {
  T h = T(0);
  Failed(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, Ctx().stream), "gerfs read");
  Failed(cudaStreamSynchronize(Ctx().stream), "gerfs sync");
  return h;
}

int ReadInt(const int* d) {
  int h = 0;
  Failed(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, Ctx().stream),
         "gerfs read");
  Failed(cudaStreamSynchronize(Ctx().stream), "gerfs sync");
  return h;
}

template <typename T>
T Asum(int n, const T* x, int lanes, T* out) {
  AsumRefKernel<T><<<1, 4 * lanes, 0, Ctx().stream>>>(n, x, lanes, out);
  CountLaunch();
  LaunchFailed("gerfs asum");
  return ReadScalar(out);
}

// LACN2 (real): the reference's state machine on the host, vectors on the
// device (x = wk, v = vv). Returns with *kase 0 when done.
template <typename T>
void Lacn2(int n, const RefineBufs<T>& bf, T* est, int* kase, int* isave, int lanes) {
  constexpr int itmax = 5;
  cudaStream_t st = Ctx().stream;
  T* x = bf.wk;
  const auto sign_vector = [&]() {
    SignKernel<T><<<Blocks(n), 256, 0, st>>>(n, x, bf.isgn);
    CountLaunch();
  };
  const auto unit_vector = [&]() {
    UnitVectorKernel<T><<<Blocks(n), 256, 0, st>>>(n, isave[1] - 1, x);
    CountLaunch();
    *kase = 1;
    isave[0] = 3;
  };
  const auto final_stage = [&]() {
    AltSignKernel<T><<<Blocks(n), 256, 0, st>>>(n, x);
    CountLaunch();
    *kase = 1;
    isave[0] = 5;
  };
  const auto iamax = [&]() {
    int* out = bf.flag + 1;
    Iamax<T>(n, x, 1, out);
    return ReadInt(out);
  };
  if (*kase == 0) {
    FillKernel<T><<<Blocks(n), 256, 0, st>>>(n, T(1) / T(n), x);
    CountLaunch();
    *kase = 1;
    isave[0] = 1;
    return;
  }
  switch (isave[0]) {
    default:
    case 1:
      if (n == 1) {
        Failed(cudaMemcpyAsync(bf.vv, x, sizeof(T), cudaMemcpyDeviceToDevice, st), "lacn2");
        *est = std::fabs(ReadScalar(x));
        *kase = 0;
        return;
      }
      *est = Asum<T>(n, x, lanes, bf.sc + 1);
      sign_vector();
      *kase = 2;
      isave[0] = 2;
      return;
    case 2:
      isave[1] = iamax();
      isave[2] = 2;
      unit_vector();
      return;
    case 3: {
      Failed(cudaMemcpyAsync(bf.vv, x, sizeof(T) * n, cudaMemcpyDeviceToDevice, st), "lacn2");
      const T estold = *est;
      *est = Asum<T>(n, bf.vv, lanes, bf.sc + 1);
      Failed(cudaMemsetAsync(bf.flag, 0, sizeof(int), st), "lacn2");
      SignChangedKernel<T><<<Blocks(n), 256, 0, st>>>(n, x, bf.isgn, bf.flag);
      CountLaunch();
      const bool changed = ReadInt(bf.flag) != 0;
      if (!changed || *est <= estold) {
        final_stage();
        return;
      }
      sign_vector();
      *kase = 2;
      isave[0] = 4;
      return;
    }
    case 4: {
      const int jlast = isave[1];
      isave[1] = iamax();
      const T xj = ReadScalar(x + jlast - 1), xm = ReadScalar(x + isave[1] - 1);
      if (xj != std::fabs(xm) && isave[2] < itmax) {
        isave[2] = isave[2] + 1;
        unit_vector();
        return;
      }
      final_stage();
      return;
    }
    case 5: {
      const T temp = T(2) * (Asum<T>(n, x, lanes, bf.sc + 1) / T(3 * n));
      if (temp > *est) {
        Failed(cudaMemcpyAsync(bf.vv, x, sizeof(T) * n, cudaMemcpyDeviceToDevice, st),
               "lacn2");
        *est = temp;
      }
      *kase = 0;
      return;
    }
  }
}

}  // namespace

// xGERFS after argument checks (n, nrhs > 0), device arrays. ferr and berr
// are host arrays of nrhs; work (3n) and iwork (n), when given (device),
// end with the reference's final workspace contents (w, r, v and the sign
// vector).
template <typename T>
void GerfsFull(bool trans, int n, int nrhs, const T* a, int lda, const T* af, int ldaf,
               const int* ipiv, const T* b, int ldb, T* x, int ldx, T* ferr, T* berr,
               T* work_dev, int* iwork_dev) {
  constexpr int itmax = 5;
  const int lanes = sizeof(T) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  cudaStream_t st = Ctx().stream;
  T* buf = static_cast<T*>(Workspace(kWsRefine, sizeof(T) * (4 * static_cast<size_t>(n) + 64)));
  int* ibuf =
      static_cast<int*>(Workspace(kWsRefineInt, sizeof(int) * (static_cast<size_t>(n) + 64)));
  if (buf == nullptr || ibuf == nullptr) return;
  // The caller's workspace contents, so that entries the call never writes
  // come back unchanged.
  if (work_dev != nullptr) {
    Failed(cudaMemcpyAsync(buf, work_dev, sizeof(T) * 3 * static_cast<size_t>(n),
                           cudaMemcpyDeviceToDevice, st),
           "gerfs work in");
  }
  if (iwork_dev != nullptr) {
    Failed(cudaMemcpyAsync(ibuf, iwork_dev, sizeof(int) * static_cast<size_t>(n),
                           cudaMemcpyDeviceToDevice, st),
           "gerfs iwork in");
  }
  RefineBufs<T> bf{buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, ibuf, ibuf + n};
  const int nz = n + 1;
  const T eps = std::numeric_limits<T>::epsilon() * T(0.5);
  const T safmin = std::numeric_limits<T>::min();
  const T safe1 = T(nz) * safmin;
  const T safe2 = safe1 / eps;
  for (int j = 0; j < nrhs; ++j) {
    T* xj = x + static_cast<long long>(j) * ldx;
    const T* bj = b + static_cast<long long>(j) * ldb;
    int count = 1;
    T lstres = T(3);
    for (;;) {
      if (!trans) {
        ResidualNKernel<T><<<Blocks(n), 256, 0, st>>>(n, a, lda, xj, bj, bf.wk, bf.rw);
        CountLaunch();
      } else {
        const long long threads = static_cast<long long>(n) * lanes;
        ResidualTKernel<T><<<static_cast<int>((threads + 255) / 256), 256, 0, st>>>(
            n, a, lda, xj, bj, bf.wk, lanes);
        AbsSumTKernel<T><<<Blocks(n), 256, 0, st>>>(n, a, lda, xj, bj, bf.rw);
        CountLaunch(2);
      }
      BerrKernel<T><<<1, 1024, 0, st>>>(n, bf.wk, bf.rw, safe1, safe2, bf.q, bf.sc);
      CountLaunch();
      if (LaunchFailed("gerfs residual")) return;
      berr[j] = ReadScalar(bf.sc);
      if (berr[j] > eps && T(2) * berr[j] <= lstres && count <= itmax) {
        Getrs<T>(trans, n, 1, af, ldaf, ipiv, bf.wk, n);
        AxpyRefKernel<T><<<Blocks(n), 256, 0, st>>>(n, T(1), bf.wk, xj, lanes);
        CountLaunch();
        lstres = berr[j];
        count = count + 1;
        continue;
      }
      break;
    }
    FerrWeightKernel<T><<<Blocks(n), 256, 0, st>>>(n, bf.wk, bf.rw, T(nz) * eps, safe1, safe2);
    CountLaunch();
    int kase = 0;
    int isave[3] = {0, 0, 0};
    for (;;) {
      Lacn2<T>(n, bf, &ferr[j], &kase, isave, lanes);
      if (kase == 0) break;
      if (kase == 1) {
        Getrs<T>(!trans, n, 1, af, ldaf, ipiv, bf.wk, n);
        DiagScaleKernel<T><<<Blocks(n), 256, 0, st>>>(n, bf.rw, bf.wk);
        CountLaunch();
      } else {
        DiagScaleKernel<T><<<Blocks(n), 256, 0, st>>>(n, bf.rw, bf.wk);
        CountLaunch();
        Getrs<T>(trans, n, 1, af, ldaf, ipiv, bf.wk, n);
      }
      if (LaunchFailed("gerfs estimate")) return;
    }
    MaxAbsKernel<T><<<1, 1, 0, st>>>(n, xj, bf.sc + 2);
    CountLaunch();
    const T lx = ReadScalar(bf.sc + 2);
    if (lx != T(0)) ferr[j] = ferr[j] / lx;
  }
  if (work_dev != nullptr) {
    Failed(cudaMemcpyAsync(work_dev, buf, sizeof(T) * 3 * static_cast<size_t>(n),
                           cudaMemcpyDeviceToDevice, st),
           "gerfs work");
  }
  if (iwork_dev != nullptr) {
    Failed(cudaMemcpyAsync(iwork_dev, ibuf, sizeof(int) * static_cast<size_t>(n),
                           cudaMemcpyDeviceToDevice, st),
           "gerfs iwork");
  }
}
template void GerfsFull<double>(bool, int, int, const double*, int, const double*, int,
                                const int*, const double*, int, double*, int, double*, double*,
                                double*, int*);
template void GerfsFull<float>(bool, int, int, const float*, int, const float*, int,
                               const int*, const float*, int, float*, int, float*, float*,
                               float*, int*);

}  // namespace hb
