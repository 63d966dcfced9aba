// FP64-accurate GEMM on the INT8 tensor cores (Ozaki scheme, splitting into
// integer slices, after Ootomo, Ozaki and Yokota, "DGEMM on integer matrix
// multiplication unit", IJHPCA 2024).
//
// Every row i of op(A) is scaled by 2^-(e_i+2) (e_i: frexp exponent of the
// row's largest |a|, so x = a 2^-(e_i+2) lies in [-1/4, 1/4)) and cut into S
// balanced base-256 digits: for s = 1..S: y = 256 x; d_s = floor(y), plus 1
// if y - floor(y) >= 1/2; x = y - d_s. Each step is exact and keeps x in
// [-1/2, 1/2), so d_1 is in [-64, 64] and the others in [-128, 128]; a digit
// of 128 is rewritten as -128 with a carry of 1 into the digit above (the top
// digit has room for it), so every digit fits signed 8 bits and the errors
// have either sign. a = 2^(e_i+2) (sum_s d_s 256^-s + r), |r| <= 256^-S / 2:
// 8S - 1 bits per value. Columns of op(B) are split the same way with
// exponents f_j. Then
//
//   A B ~ diag(2^(e+2)) [ sum_{l=0}^{S-1} 256^-(l+2) T_l ] diag(2^(f+2)),
//   T_l = sum_{p+q=l} A_p B_q^T          (p, q = 0-based slice indices),
//
// dropping the products of slices with p + q >= S. Every T_l is an exact
// INT32 tensor-core product (|T_l| <= (l+1) K 2^14 < 2^31 for K below the
// chunk limit) and the S levels are recombined in FP64 with a compensated
// (TwoSum) accumulation, smallest level first, then scaled by
// alpha 2^(e_i + f_j + 4) and merged with beta C.
//
// Kernel: one CTA per 128 x 128 tile of C and a range of levels [L0, L1]
// (at most 4: their INT32 accumulators fill the 512 tensor-memory columns).
// A producer warp streams, per k block, the slices of op(A) and op(B) that the
// levels need (128 x KB bytes each) into shared memory with TMA; a single
// thread issues tcgen05.mma kind::i8 for every slice pair of those levels in
// that k block, so each loaded slice tile feeds several products; four
// epilogue warps then read the accumulators back (tcgen05.ld), recombine them
// in FP64 and write either an FP64 partial sum W (first pass) or C. S <= 4
// runs in one pass; S = 5..8 run levels 4..S-1 first into W, then levels
// 0..3 plus W into C. (N = 128 keeps the tensor core's shared-memory operand
// reads at 8 KB per 64-cycle MMA; N = 64 would need 6 KB per 32 cycles,
// more than shared memory delivers.)
#include <cuda.h>

#include <algorithm>
#include <functional>
#include <climits>
#include <cmath>
#include <cstdio>

#include "device.cuh"
#include "internal.h"

namespace hb {

bool MakeTensorMap2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem,
                     const void* base, long long rows, long long cols,
                     long long ld, int box_rows, int box_cols,
                     CUtensorMapSwizzle swizzle);
template <typename T>
const T* Canonical(View<T> x, int rows, int cols, int slot, long long* ld_out);

namespace {

constexpr int kZeroExp = -100000;  // exponent of an all-zero row / column
constexpr int kEBM = 128, kEBN = 128;
constexpr int kEpiWarps = 4;
constexpr int kEThreads = (2 + kEpiWarps) * 32;  // producer, MMA, epilogue

// ---------------------------------------------------------------------------
// Exponents: e[o] = frexp exponent of max_k |x(o, k)| (kZeroExp if all 0).

__global__ void FillIntKernel(int* p, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// x(o, k) = data[o * os + k * is]; reduction over k for every o.
__global__ void ExpOuterContigKernel(View<double> x, int outer, int inner,
                                     int* exps, int* nonfinite) {
  // os == 1: consecutive threads take consecutive o; blockIdx.y a k chunk.
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= outer) return;
  const int k0 = blockIdx.y * 256, k1 = min(inner, k0 + 256);
  double mx = 0.0;
  bool bad = false;
  for (int k = k0; k < k1; ++k) {
    const double v = x.data[o * x.rs + k * x.cs];
    bad |= !isfinite(v);
    mx = fmax(mx, fabs(v));
  }
  if (bad) atomicOr(nonfinite, 1);
  if (mx > 0.0) {
    int e;
    frexp(mx, &e);
    atomicMax(&exps[o], e);
  }
}

__global__ void ExpInnerContigKernel(View<double> x, int outer, int inner,
                                     int* exps, int* nonfinite) {
  // is == 1: a warp per o, lanes along k.
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int lane = threadIdx.x % 32;
  if (warp >= outer) return;
  const double* row = x.data + static_cast<long long>(warp) * x.rs;
  double mx = 0.0;
  bool bad = false;
  for (int k = lane; k < inner; k += 32) {
    const double v = row[k];
    bad |= !isfinite(v);
    mx = fmax(mx, fabs(v));
  }
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    bad |= __shfl_xor_sync(0xffffffffu, bad ? 1 : 0, off) != 0;
  }
  if (lane == 0) {
    if (bad) atomicOr(nonfinite, 1);
    if (mx > 0.0) {
      int e;
      frexp(mx, &e);
      exps[warp] = e;
    }
  }
}

// Splits a value into S balanced base-256 digits (see the file comment).
template <int S>
__device__ __forceinline__ void SplitValue(double a, int e, int8_t (&d)[S]) {
  double x = (e == kZeroExp) ? 0.0 : ldexp(a, -(e + 2));
  int di[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const double y = x * 256.0;
    double t = floor(y);
    if (y - t >= 0.5) t = t + 1.0;
    di[s] = static_cast<int>(t);
    x = y - t;
  }
  // 128 = -128 + 256: carry into the more significant digit.
#pragma unroll
  for (int s = S - 1; s > 0; --s) {
    if (di[s] == 128) {
      di[s] = -128;
      di[s - 1] += 1;
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) d[s] = static_cast<int8_t>(di[s]);
}

// Slices of x (outer x inner) into out[s][o][kp] (K-major int8). is == 1:
// a thread takes 8 consecutive k of one o.
template <int S>
__global__ void SplitInnerContigKernel(View<double> x, int outer, int inner,
                                       const int* exps, int8_t* out,
                                       long long kp) {
  const long long tid = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long groups = (inner + 7) / 8;
  const long long o = tid / groups;
  const int k0 = static_cast<int>(tid % groups) * 8;
  if (o >= outer) return;
  const int e = exps[o];
  uint64_t packed[S];
#pragma unroll
  for (int s = 0; s < S; ++s) packed[s] = 0;
  const double* row = x.data + o * x.rs;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int k = k0 + j;
    const double a = (k < inner) ? row[k] : 0.0;
    int8_t d[S];
    SplitValue<S>(a, e, d);
#pragma unroll
    for (int s = 0; s < S; ++s)
      packed[s] |= static_cast<uint64_t>(static_cast<uint8_t>(d[s])) << (8 * j);
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    *reinterpret_cast<uint64_t*>(out + (static_cast<long long>(s) * outer + o) * kp + k0) =
        packed[s];
  }
}

// os == 1: a 64 (o) x 64 (k) tile through shared memory (read along o, write
// along k).
template <int S>
__global__ void __launch_bounds__(512)
    SplitOuterContigKernel(View<double> x, int outer, int inner,
                           const int* exps, int8_t* out, long long kp) {
  __shared__ double tile[64][65];  // [k][o]
  const int o0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  for (int idx = threadIdx.x; idx < 64 * 64; idx += blockDim.x) {
    const int ol = idx % 64, kl = idx / 64;
    const int o = o0 + ol, k = k0 + kl;
    tile[kl][ol] = (o < outer && k < inner) ? x.data[o * x.rs + k * x.cs] : 0.0;
  }
  __syncthreads();
  const int ol = threadIdx.x % 64, kq = threadIdx.x / 64;  // 8 groups of 8 k
  const int o = o0 + ol;
  if (o >= outer) return;
  const int e = exps[o];
  uint64_t packed[S];
#pragma unroll
  for (int s = 0; s < S; ++s) packed[s] = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int8_t d[S];
    SplitValue<S>(tile[kq * 8 + j][ol], e, d);
#pragma unroll
    for (int s = 0; s < S; ++s)
      packed[s] |= static_cast<uint64_t>(static_cast<uint8_t>(d[s])) << (8 * j);
  }
  const int k = k0 + kq * 8;
  if (k >= inner) return;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    *reinterpret_cast<uint64_t*>(out + (static_cast<long long>(s) * outer + o) * kp + k) =
        packed[s];
  }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers.

__device__ __forceinline__ void TmemLoad32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,"
      "%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,"
      "%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]),
        "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct OzakiParams {
  int m, n, k;
  const int* row_exp;
  const int* col_exp;
  double alpha, beta;
  double* c;
  long long ldc;
  double* w;  // FP64 partial sums of the first pass (m x n, leading dim m)
  int* timeout_flag;
  int lower_only;  // skip the tiles strictly above the diagonal of C
  // op(B)'s slice rows: slice sl of column j (of this launch's n) is row
  // sl * b_rows + b_off + j of the slice array (a launch over a block of C's
  // columns reads its columns of the whole array).
  int b_rows, b_off;
};

// Tile of this CTA in groups of 16 tile rows: consecutive CTAs walk down a
// 16-tile band column by column, so a wave of ~148 CTAs covers a compact
// 16 x 9 block of C and shares its slice tiles in L2.
__device__ __forceinline__ void TileOrigin(int m, int n, int* m0, int* n0) {
  constexpr int kGroup = 16;
  const int tiles_m = (m + kEBM - 1) / kEBM, tiles_n = (n + kEBN - 1) / kEBN;
  const int pid = blockIdx.x;
  const int per_group = kGroup * tiles_n;
  const int first_m = (pid / per_group) * kGroup;
  const int gm = min(tiles_m - first_m, kGroup);
  const int in_group = pid % per_group;
  *m0 = (first_m + in_group % gm) * kEBM;
  *n0 = (in_group / gm) * kEBN;
}

template <int S, int L0, int L1, int KB>
struct OzakiCfg {
  static constexpr int kNA = (L1 < S - 1 ? L1 : S - 1) + 1;  // slices loaded
  static constexpr int kNLev = L1 - L0 + 1;
  static constexpr int kATile = kEBM * KB;  // one slice of op(A)
  static constexpr int kBTile = kEBN * KB;
  static constexpr int kStage = kNA * (kATile + kBTile);
  static constexpr int kStagesRaw = (200 * 1024) / kStage;
  static constexpr int kStages = kStagesRaw > 8 ? 8 : kStagesRaw;
  static constexpr int kBarOffset = kStages * kStage;
  static constexpr int kSmem = kBarOffset + 256 + 1024;
  static constexpr int kTmemCols = kNLev * kEBN <= 128 ? 128
                                 : kNLev * kEBN <= 256 ? 256 : 512;
  static_assert(kNLev * kEBN <= 512, "accumulators exceed tensor memory");
  static_assert(kStages >= 2, "stage too large");
};

// kFinal: write C (reading W first if kReadW); else write the pass's FP64
// partial sum to W.
template <int S, int L0, int L1, int KB, bool kFinal, bool kReadW>
__global__ void __launch_bounds__(kEThreads, 1)
    OzakiGemmKernel(const __grid_constant__ CUtensorMap tm_a,
                    const __grid_constant__ CUtensorMap tm_b, OzakiParams p) {
  using Cfg = OzakiCfg<S, L0, L1, KB>;
  constexpr int kStages = Cfg::kStages;
  constexpr int kNA = Cfg::kNA;
  int m0, n0;
  TileOrigin(p.m, p.n, &m0, &n0);
  // A product whose lower triangle alone is wanted (a symmetric rank-k
  // update): tiles strictly above the diagonal return before any set-up.
  if (p.lower_only && n0 >= m0 + kEBM) return;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024 - (SmemAddr(smem_raw) & 1023)) & 1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Cfg::kBarOffset);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_full + 1);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      MbarInit(&full[s], 1);
      MbarInit(&empty[s], 1);
    }
    MbarInit(acc_full, 1);
    FenceBarrierInit();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(SmemAddr(tmem_slot)), "r"(Cfg::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nkb = (p.k + KB - 1) / KB;

  if (warp == 0) {
    if (lane == 0) {
      PrefetchTmap(&tm_a);
      PrefetchTmap(&tm_b);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % kStages, round = kb / kStages;
        if (round > 0 && !MbarWait(&empty[s], (round - 1) & 1, p.timeout_flag)) break;
        uint8_t* st = smem + s * Cfg::kStage;
        MbarArriveExpectTx(&full[s], Cfg::kStage);
#pragma unroll
        for (int sl = 0; sl < kNA; ++sl) {
          TmaLoad2d(st + sl * Cfg::kATile, &tm_a, kb * KB, sl * p.m + m0, &full[s]);
          TmaLoad2d(st + kNA * Cfg::kATile + sl * Cfg::kBTile, &tm_b, kb * KB,
                    sl * p.b_rows + p.b_off + n0, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // Instruction descriptor: D s32, A/B signed 8-bit, both K-major,
      // N = 128, M = 128.
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) |
                             (static_cast<uint32_t>(kEBN >> 3) << 17) |
                             (static_cast<uint32_t>(kEBM >> 4) << 24);
      for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb % kStages, round = kb / kStages;
        if (!MbarWait(&full[s], round & 1, p.timeout_flag)) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = SmemAddr(smem + s * Cfg::kStage);
#pragma unroll
        for (int l = L0; l <= L1; ++l) {
#pragma unroll
          for (int pa = 0; pa <= l; ++pa) {
            const int qb = l - pa;
            if (pa >= S || qb >= S) continue;
#pragma unroll
            for (int kk = 0; kk < KB / 32; ++kk) {
              const uint64_t da = SmemDesc(st + pa * Cfg::kATile + kk * 32, KB);
              const uint64_t db =
                  SmemDesc(st + kNA * Cfg::kATile + qb * Cfg::kBTile + kk * 32, KB);
              const uint32_t acc = (kb == 0 && pa == 0 && kk == 0) ? 0u : 1u;
              MmaI8(tmem + (l - L0) * kEBN, da, db, idesc, acc);
            }
          }
        }
        MmaCommit(&empty[s]);
      }
      MmaCommit(acc_full);
    }
  } else {
    // Epilogue warps 2..5: TMEM lanes 32 (warp % 4) .. + 31 = tile rows.
    const int q = warp % 4;
    const int row = m0 + 32 * q + lane;
    const bool ok = MbarWait(acc_full, 0, p.timeout_flag);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      const int e_row = (row < p.m) ? p.row_exp[row] : kZeroExp;
#pragma unroll 1
      for (int cc = 0; cc < kEBN / 32; ++cc) {
        double sum[32], comp[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          comp[j] = 0.0;
          const int col = n0 + cc * 32 + j;
          sum[j] = (kReadW && row < p.m && col < p.n)
                       ? p.w[row + static_cast<long long>(col) * p.m] : 0.0;
        }
#pragma unroll
        for (int l = L1; l >= L0; --l) {
          uint32_t r[32];
          TmemLoad32(tmem + (static_cast<uint32_t>(32 * q) << 16) + (l - L0) * kEBN + cc * 32, r);
          const double wgt = ldexp(1.0, -8 * (l + 2));
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const double v = static_cast<double>(static_cast<int>(r[j])) * wgt;
            // TwoSum: sum + v = s + err exactly.
            const double s2 = sum[j] + v;
            const double bb = s2 - sum[j];
            const double err = (sum[j] - (s2 - bb)) + (v - bb);
            sum[j] = s2;
            comp[j] = comp[j] + err;
          }
        }
        if (row >= p.m) continue;
        if constexpr (!kFinal) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + cc * 32 + j;
            if (col < p.n) p.w[row + static_cast<long long>(col) * p.m] = sum[j] + comp[j];
          }
        } else {
          // All loads of the chunk (column exponents, C) are issued before
          // its stores, which the compiler cannot reorder them across.
          int f[32];
          double cin[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            sum[j] += comp[j];
            const int col = n0 + cc * 32 + j;
            f[j] = (col < p.n) ? p.col_exp[col] : kZeroExp;
            cin[j] = (col < p.n && p.beta != 0.0) ? p.c[row + col * p.ldc] : 0.0;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + cc * 32 + j;
            if (col >= p.n) continue;
            double v = 0.0;
            if (f[j] != kZeroExp && e_row != kZeroExp) v = ldexp(sum[j], e_row + f[j] + 4);
            const double r = p.alpha * v;
            p.c[row + col * p.ldc] = (p.beta == 0.0) ? r : fma(p.beta, cin[j], r);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 ::"r"(tmem), "r"(Cfg::kTmemCols));
  }
}

// Reference-precision product for error measurement: every C(i, j) of the
// selected columns as a double-double sum of exact products (TwoProduct by
// FMA, TwoSum accumulation), rounded once at the end.
__global__ void DoubleDoubleGemmKernel(int m, int ncols, int k, View<double> a,
                                       View<double> b, const int* cols,
                                       double* out, long long ldo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y;
  if (i >= m || jj >= ncols) return;
  const int j = cols[jj];
  double hi = 0.0, lo = 0.0;
  for (int p = 0; p < k; ++p) {
    const double x = a.data[i * a.rs + p * a.cs];
    const double y = b.data[p * b.rs + static_cast<long long>(j) * b.cs];
    const double ph = x * y;
    const double pl = fma(x, y, -ph);
    const double s = hi + ph;
    const double bb = s - hi;
    const double e = (hi - (s - bb)) + (ph - bb);
    hi = s;
    lo = lo + (e + pl);
  }
  out[i + jj * ldo] = hi + lo;
}

// ---------------------------------------------------------------------------
// Automatic slice count.
//
// The emulated product's error grows with how far the products a(i,p) b(p,j)
// sit below the scales 2^e_i 2^f_j that the slicing is relative to. With
// E = max e_i and F = max f_j, the statistic
//
//   rho = K (sum_i 4^(e_i - E)) (sum_j 4^(f_j - F))
//         / sum_p (sum_i (a(i,p) 2^-E)^2) (sum_j (b(p,j) 2^-F)^2)   (>= 1)
//
// compares the squared scales with the squared products, and
// beta = log2(rho) / 2 is the number of bits the data loses to its exponent
// spread. Measured on B200 (normwise error against a double-double product,
// spreads 0..30 and graded columns, K = 64..8192) the error of S slices
// relative to the plain FP64 path's is at most
//
//   r(S) = 2^(beta + 52.57 - 8 S + max(0, (8 - log2 K) / 2)) + 0.04,
//
// (the last term: both paths round the same result; the K term: FP64 chains
// shorter than the reference's 256-long chunks are more accurate). The call
// takes the smallest S with r(S) <= 1/2 and runs the plain FP64 path when no
// S <= 8 qualifies. Every reduction below runs in a fixed order, so the same
// inputs always get the same S.

constexpr int kSumSqRowsP = 64;     // rows of a p-contiguous chunk
constexpr int kSumSqRowsO = 1024;   // rows of an o-contiguous chunk

__global__ void MaxExpKernel(const int* exps, int n, int* out) {
  __shared__ int s[1024];
  int mx = kZeroExp;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = max(mx, exps[i]);
  s[threadIdx.x] = mx;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) s[threadIdx.x] = max(s[threadIdx.x], s[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// part[c * inner + p] = sum over the rows o of chunk c of (x(o, p) 2^-E)^2.
// x.cs == 1: a thread per p, looping over the chunk's rows.
__global__ void SumSqPContigKernel(View<double> x, int outer, int inner,
                                   const int* emax, double* part) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= inner) return;
  const int E = *emax;
  const int o0 = blockIdx.y * kSumSqRowsP, o1 = min(outer, o0 + kSumSqRowsP);
  double s = 0.0;
  if (E != kZeroExp) {
    for (int o = o0; o < o1; ++o) {
      const double v = ldexp(x.data[o * x.rs + p * x.cs], -E);
      s = fma(v, v, s);
    }
  }
  part[static_cast<long long>(blockIdx.y) * inner + p] = s;
}

// x.rs == 1: a warp per p, lanes along the chunk's rows, fixed shuffle tree.
__global__ void SumSqOContigKernel(View<double> x, int outer, int inner,
                                   const int* emax, double* part) {
  const int p = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (p >= inner) return;
  const int E = *emax;
  const int o0 = blockIdx.y * kSumSqRowsO, o1 = min(outer, o0 + kSumSqRowsO);
  double s = 0.0;
  if (E != kZeroExp) {
    for (int o = o0 + lane; o < o1; o += 32) {
      const double v = ldexp(x.data[o * x.rs + p * x.cs], -E);
      s = fma(v, v, s);
    }
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) part[static_cast<long long>(blockIdx.y) * inner + p] = s;
}

__device__ double BlockSum(double v, double* s) {
  s[threadIdx.x] = v;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
    __syncthreads();
  }
  const double r = s[0];
  __syncthreads();
  return r;
}

struct AutoArgs {
  const int* row_exp;
  const int* col_exp;
  int m, n, k;
  const int* emax;      // [0] E of op(A), [1] F of op(B)
  const double* part_a;  // [chunks_a][k]
  const double* part_b;  // [chunks_b][k]
  int chunks_a, chunks_b;
  int* slices_out;      // the chosen S (0: the plain path)
};

// One block of 1024 threads: the statistic and the slice count.
__global__ void AutoSlicesKernel(AutoArgs g) {
  __shared__ double s[1024];
  const int E = g.emax[0], F = g.emax[1];
  double sa = 0.0, sb = 0.0, q = 0.0;
  if (E != kZeroExp && F != kZeroExp) {
    for (int i = threadIdx.x; i < g.m; i += blockDim.x)
      if (g.row_exp[i] != kZeroExp) sa += ldexp(1.0, 2 * (g.row_exp[i] - E));
    for (int j = threadIdx.x; j < g.n; j += blockDim.x)
      if (g.col_exp[j] != kZeroExp) sb += ldexp(1.0, 2 * (g.col_exp[j] - F));
    for (int p = threadIdx.x; p < g.k; p += blockDim.x) {
      double ca = 0.0, rb = 0.0;
      for (int c = 0; c < g.chunks_a; ++c) ca += g.part_a[static_cast<long long>(c) * g.k + p];
      for (int c = 0; c < g.chunks_b; ++c) rb += g.part_b[static_cast<long long>(c) * g.k + p];
      q = fma(ca, rb, q);
    }
  }
  sa = BlockSum(sa, s);
  sb = BlockSum(sb, s);
  q = BlockSum(q, s);
  if (threadIdx.x == 0) {
    int S = 1;
    if (q > 0.0) {
      const double rho = fmax(1.0, static_cast<double>(g.k) * sa * sb / q);
      const double beta = 0.5 * log2(rho);
      const double kterm = fmax(0.0, 0.5 * (8.0 - log2(static_cast<double>(g.k))));
      S = 0;
      for (int c = 1; c <= 8; ++c) {
        if (exp2(beta + 52.57 - 8.0 * c + kterm) + 0.04 <= 0.5) {
          S = c;
          break;
        }
      }
    }
    *g.slices_out = S;
  }
}

void SumSquares(View<double> x, int outer, int inner, const int* emax, double* part,
                int* chunks, cudaStream_t st) {
  if (x.rs == 1) {
    *chunks = (outer + kSumSqRowsO - 1) / kSumSqRowsO;
    const dim3 grid((inner + 7) / 8, *chunks);
    SumSqOContigKernel<<<grid, 256, 0, st>>>(x, outer, inner, emax, part);
  } else {
    *chunks = (outer + kSumSqRowsP - 1) / kSumSqRowsP;
    const dim3 grid((inner + 255) / 256, *chunks);
    SumSqPContigKernel<<<grid, 256, 0, st>>>(x, outer, inner, emax, part);
  }
  CountLaunch();
  LaunchFailed("ozaki auto statistics");
}

template <int S>
void LaunchSplit(View<double> x, int outer, int inner, const int* exps,
                 int8_t* out, long long kp, cudaStream_t st) {
  if (x.cs == 1 && x.rs != 1) {
    // op(X)(o, k) contiguous along k.
    const long long threads = static_cast<long long>(outer) * ((inner + 7) / 8);
    SplitInnerContigKernel<S><<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(
        x, outer, inner, exps, out, kp);
  } else {
    const dim3 grid((outer + 63) / 64, (inner + 63) / 64);
    SplitOuterContigKernel<S><<<grid, 512, 0, st>>>(x, outer, inner, exps, out, kp);
  }
}

void SplitDispatch(int S, View<double> x, int outer, int inner, const int* exps,
                   int8_t* out, long long kp, cudaStream_t st) {
  switch (S) {
    case 1: LaunchSplit<1>(x, outer, inner, exps, out, kp, st); break;
    case 2: LaunchSplit<2>(x, outer, inner, exps, out, kp, st); break;
    case 3: LaunchSplit<3>(x, outer, inner, exps, out, kp, st); break;
    case 4: LaunchSplit<4>(x, outer, inner, exps, out, kp, st); break;
    case 5: LaunchSplit<5>(x, outer, inner, exps, out, kp, st); break;
    case 6: LaunchSplit<6>(x, outer, inner, exps, out, kp, st); break;
    case 7: LaunchSplit<7>(x, outer, inner, exps, out, kp, st); break;
    default: LaunchSplit<8>(x, outer, inner, exps, out, kp, st); break;
  }
  CountLaunch();
  LaunchFailed("ozaki split");
}

void Exponents(View<double> x, int outer, int inner, int* exps, int* nonfinite,
               cudaStream_t st) {
  FillIntKernel<<<(outer + 255) / 256, 256, 0, st>>>(exps, outer, kZeroExp);
  if (x.cs == 1 && x.rs != 1) {
    ExpInnerContigKernel<<<(outer + 7) / 8, 256, 0, st>>>(x, outer, inner, exps,
                                                          nonfinite);
  } else {
    // Row-major reductions over k chunks (view along o contiguous).
    View<double> v = x;
    const dim3 grid((outer + 255) / 256, (inner + 255) / 256);
    ExpOuterContigKernel<<<grid, 256, 0, st>>>(v, outer, inner, exps, nonfinite);
  }
  CountLaunch(2);
  LaunchFailed("ozaki exponents");
}

template <int S, int L0, int L1, int KB, bool kFinal, bool kReadW>
bool LaunchOzaki(const CUtensorMap& ma, const CUtensorMap& mb,
                 const OzakiParams& p, cudaStream_t st) {
  using Cfg = OzakiCfg<S, L0, L1, KB>;
  auto* kernel = OzakiGemmKernel<S, L0, L1, KB, kFinal, kReadW>;
  static bool configured = false;
  if (!configured) {
    if (Failed(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    Cfg::kSmem),
               "ozaki smem attribute"))
      return false;
    configured = true;
  }
  const long long tiles =
      static_cast<long long>((p.m + kEBM - 1) / kEBM) * ((p.n + kEBN - 1) / kEBN);
  cudaEvent_t t0 = KernelTimerStart(kFamilyOzakiGemm, st);
  kernel<<<static_cast<unsigned>(tiles), kEThreads, Cfg::kSmem, st>>>(ma, mb, p);
  KernelTimerStop(t0, st);
  CountLaunch();
  return !LaunchFailed("ozaki gemm");
}

// k-block bytes of each pass: the stage of the slices it loads must leave
// room for at least two stages (KB = 32 for the 8-slice pass: 64 KB).
constexpr int KbSingle(int S) { return S <= 2 ? 128 : 64; }
constexpr int kKbHigh = 32, kKbLow = 64;

// One slice-product pass: the maps cover `slices` slices of op(A) / op(B)
// with k blocks of `kb` bytes.
struct PassMaps {
  CUtensorMap a, b;
};

bool GemmDispatch(int S, const PassMaps& single, const PassMaps& high,
                  const PassMaps& low, const OzakiParams& p, cudaStream_t st) {
  switch (S) {
    case 1: return LaunchOzaki<1, 0, 0, KbSingle(1), true, false>(single.a, single.b, p, st);
    case 2: return LaunchOzaki<2, 0, 1, KbSingle(2), true, false>(single.a, single.b, p, st);
    case 3: return LaunchOzaki<3, 0, 2, KbSingle(3), true, false>(single.a, single.b, p, st);
    case 4: return LaunchOzaki<4, 0, 3, KbSingle(4), true, false>(single.a, single.b, p, st);
    case 5:
      return LaunchOzaki<5, 4, 4, kKbHigh, false, false>(high.a, high.b, p, st) &&
             LaunchOzaki<5, 0, 3, kKbLow, true, true>(low.a, low.b, p, st);
    case 6:
      return LaunchOzaki<6, 4, 5, kKbHigh, false, false>(high.a, high.b, p, st) &&
             LaunchOzaki<6, 0, 3, kKbLow, true, true>(low.a, low.b, p, st);
    case 7:
      return LaunchOzaki<7, 4, 6, kKbHigh, false, false>(high.a, high.b, p, st) &&
             LaunchOzaki<7, 0, 3, kKbLow, true, true>(low.a, low.b, p, st);
    default:
      return LaunchOzaki<8, 4, 7, kKbHigh, false, false>(high.a, high.b, p, st) &&
             LaunchOzaki<8, 0, 3, kKbLow, true, true>(low.a, low.b, p, st);
  }
}

CUtensorMapSwizzle SwizzleOf(int kb) {
  return kb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                   : (kb == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

bool MakePassMaps(PassMaps* pm, const int8_t* sa, const int8_t* sb, int kc, int m,
                  int n, int slices, long long kp, int kb) {
  return MakeTensorMap2d(&pm->a, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, sa, kc,
                         static_cast<long long>(slices) * m, kp, kb, kEBM, SwizzleOf(kb)) &&
         MakeTensorMap2d(&pm->b, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, sb, kc,
                         static_cast<long long>(slices) * n, kp, kb, kEBN, SwizzleOf(kb));
}

}  // namespace

// Largest K for which every level sum fits INT32: S K 2^14 < 2^31.
int OzakiMaxK(int S) { return static_cast<int>((2147483647LL / (S * 16384LL)) / 128 * 128); }

// Returns the slice count used (0 if the plain FP64 path ran instead: the
// inputs were not finite, or slices == 0 found no S <= 8 as accurate as it).
int DgemmEmulated(int m, int n, int k, double alpha, View<double> a,
                  View<double> b, double beta, double* c, int ldc, int slices,
                  bool check_finite, int ws_set, bool lower_only, int col_blocks,
                  const std::function<void(int, int)>* block_done) {
  const int ws_emul = ws_set ? kWsEmul2 : kWsEmul;
  const int ws_acc = ws_set ? kWsEmulAcc2 : kWsEmulAcc;
  const int ws_w = ws_set ? kWsEmulW2 : kWsEmulW;
  Context& ctx = Ctx();
  cudaStream_t st = ctx.stream;
  const bool automatic = (slices == 0);
  // op(B)(p, j): outer j, inner p -> element (j, p) at rs_b * p + cs_b * j.
  View<double> bt;
  bt.data = b.data;
  bt.rs = b.cs;
  bt.cs = b.rs;
  // Workspace: ints [row exponents m | column exponents n | nonfinite, S,
  // E, F, ...] then, for the automatic slice count, the per-p partial sums
  // of squares of op(A) and op(B).
  const int chunks_a = a.rs == 1 ? (m + kSumSqRowsO - 1) / kSumSqRowsO
                                 : (m + kSumSqRowsP - 1) / kSumSqRowsP;
  const int chunks_b = bt.rs == 1 ? (n + kSumSqRowsO - 1) / kSumSqRowsO
                                  : (n + kSumSqRowsP - 1) / kSumSqRowsP;
  const size_t int_bytes = (sizeof(int) * (m + n + 64) + 255) / 256 * 256;
  const size_t part_bytes =
      automatic ? sizeof(double) * static_cast<size_t>(chunks_a + chunks_b) * k : 0;
  char* acc = static_cast<char*>(Workspace(ws_acc, int_bytes + part_bytes));
  int* exps = reinterpret_cast<int*>(acc);
  int* row_exp = exps;
  int* col_exp = exps + m;
  int* flags = exps + m + n;  // [0] nonfinite, [1] automatic S, [2..3] E, F
  cudaMemsetAsync(flags, 0, sizeof(int) * 2, st);
  Exponents(a, m, k, row_exp, flags, st);
  Exponents(bt, n, k, col_exp, flags, st);
  if (automatic) {
    double* part_a = reinterpret_cast<double*>(acc + int_bytes);
    double* part_b = part_a + static_cast<size_t>(chunks_a) * k;
    MaxExpKernel<<<1, 1024, 0, st>>>(row_exp, m, flags + 2);
    MaxExpKernel<<<1, 1024, 0, st>>>(col_exp, n, flags + 3);
    CountLaunch(2);
    int ca = 0, cb = 0;
    SumSquares(a, m, k, flags + 2, part_a, &ca, st);
    SumSquares(bt, n, k, flags + 3, part_b, &cb, st);
    AutoArgs g;
    g.row_exp = row_exp;
    g.col_exp = col_exp;
    g.m = m;
    g.n = n;
    g.k = k;
    g.emax = flags + 2;
    g.part_a = part_a;
    g.part_b = part_b;
    g.chunks_a = ca;
    g.chunks_b = cb;
    g.slices_out = flags + 1;
    AutoSlicesKernel<<<1, 1024, 0, st>>>(g);
    CountLaunch();
    if (LaunchFailed("ozaki auto slices")) return -1;
  }
  int host_flags[2] = {0, 0};
  if (check_finite || automatic) {
    cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, st);
    if (Failed(cudaStreamSynchronize(st), "ozaki exponents")) return -1;
  }
  if (host_flags[0] || (automatic && host_flags[1] == 0)) {
    // Inf/NaN cannot be sliced, and a spread too wide for 8 slices would
    // lose accuracy: the plain FP64 path runs (and propagates Inf/NaN).
    Dgemm(m, n, k, alpha, a, b, beta, c, ldc, kAll);
    return 0;
  }
  const int S = automatic ? host_flags[1] : std::min(8, std::max(1, slices));
  const int kmax = OzakiMaxK(S);
  const int kchunk = std::min(k, kmax);
  const long long kp = (static_cast<long long>(kchunk) + 15) / 16 * 16;
  int8_t* slices_a = static_cast<int8_t*>(
      Workspace(ws_emul, static_cast<size_t>(S) * (static_cast<size_t>(m) + n) * kp + 256));
  int8_t* slices_b = slices_a + static_cast<size_t>(S) * m * kp;
  OzakiParams p;
  p.m = m;
  p.n = n;
  p.row_exp = row_exp;
  p.col_exp = col_exp;
  p.alpha = alpha;
  p.c = c;
  p.ldc = ldc;
  p.w = (S > 4) ? static_cast<double*>(Workspace(ws_w, sizeof(double) *
                                                            static_cast<size_t>(m) * n))
                : nullptr;
  p.timeout_flag = ctx.dev_status;
  p.lower_only = lower_only ? 1 : 0;
  p.b_rows = n;
  p.b_off = 0;
  // Column blocks (one k chunk, a full C): the products run block by block
  // and block_done(first column, columns) is called as each block's
  // launches are queued, so that the caller can move the block while the
  // next one is computed. Each element's arithmetic is the same as unblocked.
  const int blocks =
      (col_blocks > 1 && block_done != nullptr && kchunk == k && !lower_only) ? col_blocks : 1;
  if (blocks > 1) {
    SplitDispatch(S, a, m, k, row_exp, slices_a, kp, st);
    SplitDispatch(S, bt, n, k, col_exp, slices_b, kp, st);
    PassMaps single, high, low;
    bool ok;
    if (S <= 4) {
      ok = MakePassMaps(&single, slices_a, slices_b, k, m, n, S, kp, KbSingle(S));
    } else {
      ok = MakePassMaps(&high, slices_a, slices_b, k, m, n, S, kp, kKbHigh) &&
           MakePassMaps(&low, slices_a, slices_b, k, m, n, S, kp, kKbLow);
    }
    if (!ok) {
      Failed(cudaErrorInvalidValue, "ozaki tensor map");
      return -1;
    }
    p.k = k;
    p.beta = beta;
    // Block widths: multiples of the tile width, as even as possible.
    const int tiles_n = (n + kEBN - 1) / kEBN;
    for (int blk = 0, t0 = 0; blk < blocks; ++blk) {
      const int t1 = static_cast<int>(static_cast<long long>(tiles_n) * (blk + 1) / blocks);
      const int n0 = t0 * kEBN, nb = std::min(n, t1 * kEBN) - n0;
      t0 = t1;
      if (nb <= 0) continue;
      OzakiParams q = p;
      q.n = nb;
      q.col_exp = col_exp + n0;
      q.c = c + static_cast<long long>(n0) * ldc;
      q.w = p.w ? p.w + static_cast<long long>(n0) * m : nullptr;
      q.b_off = n0;
      if (!GemmDispatch(S, single, high, low, q, st)) return -1;
      (*block_done)(n0, nb);
    }
    return S;
  }
  for (int k0 = 0; k0 < k; k0 += kchunk) {
    const int kc = std::min(kchunk, k - k0);
    SplitDispatch(S, a.sub(0, k0), m, kc, row_exp, slices_a, kp, st);
    SplitDispatch(S, bt.sub(0, k0), n, kc, col_exp, slices_b, kp, st);
    PassMaps single, high, low;
    bool ok;
    if (S <= 4) {
      ok = MakePassMaps(&single, slices_a, slices_b, kc, m, n, S, kp, KbSingle(S));
    } else {
      ok = MakePassMaps(&high, slices_a, slices_b, kc, m, n, S, kp, kKbHigh) &&
           MakePassMaps(&low, slices_a, slices_b, kc, m, n, S, kp, kKbLow);
    }
    if (!ok) {
      Failed(cudaErrorInvalidValue, "ozaki tensor map");
      return -1;
    }
    p.k = kc;
    p.beta = (k0 == 0) ? beta : 1.0;
    if (!GemmDispatch(S, single, high, low, p, st)) return -1;
  }
  return S;
}

void DgemmDoubleDouble(int m, int ncols, int k, View<double> a, View<double> b,
                       const int* cols, double* out, int ldo) {
  const dim3 grid((m + 127) / 128, ncols);
  DoubleDoubleGemmKernel<<<grid, 128, 0, Ctx().stream>>>(m, ncols, k, a, b, cols,
                                                         out, ldo);
  CountLaunch();
  LaunchFailed("double-double gemm");
}

}  // namespace hb
