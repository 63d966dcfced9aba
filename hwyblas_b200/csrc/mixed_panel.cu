// LU panels of the mixed-precision dgesv (factor in reduced precision, refine
// in FP64). Only a stable pivoted LU is needed here, not the reference's
// recursive order (lapack.cc keeps that for the plain path), so a panel is
// factored right-looking over 32-column sub-panels, each with few launches:
//
//   leaf         pivot search, interchanges and scaling of the sub-panel over
//                all of the panel's rows, by tournament pivoting (one
//                cooperative launch, no per-column exchange between CTAs);
//   swap+solve   the sub-panel's interchanges on every other column of the
//                panel, and U12 = L11^{-1} A12 on the columns to its right;
//   update       A22 -= L21 U12 (rank 32, one DMMA pass over A22).
//
// Pivots are LAPACK-style (row i interchanged with row ipiv[i], 1-based) and
// end relative to the panel's first row.
#include <algorithm>
#include <climits>
#include <cmath>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

template <typename T>
T* At(T* a, long long lda, long long i, long long j) {
  return a + i + j * lda;
}

// Interchanges and triangular solve of one sub-panel. The sub-panel [c, c + w)
// has just been factored by the leaf, which left its pivots relative to row c
// in piv[0..w). Columns [0, left) (earlier sub-panels) get the w
// interchanges; columns [rbeg, rbeg + right) get them and then
// U12 = L11^{-1} A12 on their rows [c, c + w) (L11 unit lower). The w
// interchanges touch at most 2w rows: warp 0 replays them once on slot
// indices (slot s < w is row c + s, the others are the distinct pivot rows
// below the block), then each column is one gather over the slots.
constexpr int kSwapCols = 32;  // columns per CTA
__global__ void __launch_bounds__(256)
    PanelSwapSolveKernel(int w, int c, int left, int rbeg, int right, double* a,
                         long long lda, const int* piv) {
  __shared__ int s_row[64];    // slot -> row
  __shared__ int s_src[64];    // slot -> slot whose value ends there
  __shared__ int s_pslot[32];  // interchange i -> slot of its pivot row
  __shared__ int s_nslots;
  __shared__ double s_l[32][33];
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int lblocks = (left + kSwapCols - 1) / kSwapCols;
  const bool is_right = static_cast<int>(blockIdx.x) >= lblocks;
  const int col0 = is_right ? rbeg + (static_cast<int>(blockIdx.x) - lblocks) * kSwapCols
                            : static_cast<int>(blockIdx.x) * kSwapCols;
  const int ncols = min(kSwapCols, is_right ? rbeg + right - col0 : left - col0);
  if (warp == 0) {
    const int p = lane < w ? c + piv[lane] - 1 : -1;
    const bool below = lane < w && p >= c + w;
    // Lanes with the same pivot row share one slot: the lowest lane leads.
    const unsigned peers = __match_any_sync(0xffffffffu, below ? p : -(lane + 2));
    const int leader = __ffs(peers) - 1;
    const unsigned leaders = __ballot_sync(0xffffffffu, below && leader == lane);
    const int rank = __popc(leaders & ((1u << leader) - 1u));
    if (lane < w) {
      s_row[lane] = c + lane;
      s_pslot[lane] = below ? w + rank : p - c;
      if (below && leader == lane) s_row[w + rank] = p;
    }
    if (lane == 0) s_nslots = w + __popc(leaders);
    __syncwarp();
    if (lane == 0) {
      const int ns = s_nslots;
      for (int s = 0; s < ns; ++s) s_src[s] = s;
      for (int i = 0; i < w; ++i) {
        const int t = s_pslot[i], v = s_src[i];
        s_src[i] = s_src[t];
        s_src[t] = v;
      }
    }
  }
  if (is_right) {
    for (int idx = tid; idx < 32 * 32; idx += 256) {
      const int i = idx % 32, k = idx / 32;
      s_l[i][k] = (i < w && k < w) ? a[c + i + static_cast<long long>(c + k) * lda] : 0.0;
    }
  }
  __syncthreads();
  const int ns = s_nslots;
  const int r0 = lane < ns ? s_row[lane] : 0;
  const int r1 = lane + 32 < ns ? s_row[lane + 32] : 0;
  const int src0 = lane < ns ? s_src[lane] : 0;
  const int src1 = lane + 32 < ns ? s_src[lane + 32] : 0;
  for (int j = warp; j < ncols; j += 8) {
    double* col = a + static_cast<long long>(col0 + j) * lda;
    const double v0 = lane < ns ? col[r0] : 0.0;
    const double v1 = lane + 32 < ns ? col[r1] : 0.0;
    const double g00 = __shfl_sync(0xffffffffu, v0, src0 & 31);
    const double g01 = __shfl_sync(0xffffffffu, v1, src0 & 31);
    const double g10 = __shfl_sync(0xffffffffu, v0, src1 & 31);
    const double g11 = __shfl_sync(0xffffffffu, v1, src1 & 31);
    double n0 = src0 < 32 ? g00 : g01;
    const double n1 = src1 < 32 ? g10 : g11;
    if (is_right) {
      // Forward substitution with the unit lower L11 (lane i holds row i).
      for (int k = 0; k < w - 1; ++k) {
        const double xk = __shfl_sync(0xffffffffu, n0, k);
        if (lane > k && lane < w) n0 = fma(-s_l[lane][k], xk, n0);
      }
    }
    if (lane < ns) col[r0] = n0;
    if (lane + 32 < ns) col[r1] = n1;
  }
}

// C -= A B for the mixed panels' rank-w updates (w <= 32): A m x w, B w x n,
// C m x n, column-major. The reference-order DMMA GEMM streams K in chunks
// and is built for large K; here K is one MMA k-extent of 32, so the cost is
// C's read and write. One CTA per 128 x 32 tile of C: -A's 128 x 32 and B's
// 32 x 32 in padded shared memory, each warp's 16 x 32 block of C loaded
// straight into its m16n8k8 accumulators, 4 k-steps, stored back.
constexpr int kRkM = 128, kRkN = 32, kRkK = 32;
constexpr int kRkLda = kRkM + 4;  // conflict-free A fragments
constexpr int kRkLdb = kRkK + 4;  // conflict-free B fragments
// With lower_only, tiles wholly above C's diagonal are skipped.
__global__ void __launch_bounds__(256)
    PanelRankUpdateKernel(int m, int n, int kw, const double* a, long long lda,
                          const double* b, long long ldb, double* c, long long ldc,
                          bool lower_only) {
  __shared__ __align__(16) double sa[kRkK * kRkLda];  // sa[k * kRkLda + row] = -A
  __shared__ __align__(16) double sb[kRkN * kRkLdb];  // sb[col * kRkLdb + k] = B
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, t = lane & 3;
  const int r0 = blockIdx.x * kRkM, c0 = blockIdx.y * kRkN;
  if (lower_only && c0 >= r0 + kRkM) return;
  for (int idx = tid; idx < kRkK * kRkM; idx += 256) {
    const int k = idx / kRkM, r = idx % kRkM;
    sa[k * kRkLda + r] = (k < kw && r0 + r < m) ? -a[r0 + r + k * lda] : 0.0;
  }
  for (int idx = tid; idx < kRkN * kRkK; idx += 256) {
    const int col = idx / kRkK, k = idx % kRkK;
    sb[col * kRkLdb + k] = (k < kw && c0 + col < n) ? b[k + (c0 + col) * ldb] : 0.0;
  }
  // Warp w: rows w*16 .. +16, all 32 columns of the tile.
  double d[4][4];
  const int row = r0 + warp * 16 + g;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int col = c0 + j * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int rr = row + (e >> 1) * 8, cc = col + (e & 1);
      d[j][e] = (rr < m && cc < n) ? c[rr + cc * ldc] : 0.0;
    }
  }
  __syncthreads();
#pragma unroll
  for (int kk = 0; kk < kRkK / 8; ++kk) {
    const int lr = warp * 16 + g, k0 = kk * 8 + t;
    const double a0 = sa[k0 * kRkLda + lr];
    const double a1 = sa[k0 * kRkLda + lr + 8];
    const double a2 = sa[(k0 + 4) * kRkLda + lr];
    const double a3 = sa[(k0 + 4) * kRkLda + lr + 8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = j * 8 + g;
      const double b0 = sb[col * kRkLdb + k0];
      const double b1 = sb[col * kRkLdb + k0 + 4];
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
          "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
          : "+d"(d[j][0]), "+d"(d[j][1]), "+d"(d[j][2]), "+d"(d[j][3])
          : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int col = c0 + j * 8 + 2 * t;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int rr = row + (e >> 1) * 8, cc = col + (e & 1);
      if (rr < m && cc < n) c[rr + cc * ldc] = d[j][e];
    }
  }
}

// Cholesky of one 32-column sub-panel of a diagonal block (the mixed
// dposv's FP64 diagonal blocks; a stable Cholesky is all that is needed, not
// the reference's recursive order). The sub-panel is m rows x w columns
// (w <= 32) at a, its top w x w block on the diagonal. Every CTA factors
// that block in registers (one warp, left-looking), then solves its 128
// rows below it, X L11^T = A21, one row per thread with the row in
// registers. It stores L21 in place and, transposed, into the strip to the
// right of the diagonal block (rows 0..w, columns w..m), where the rank-w
// update reads it as its right operand. L11 overwrites the block that every
// CTA reads first, so the last CTA to have read it (an arrival counter,
// zero between launches) stores it: no CTA waits for another. A pivot that
// is not positive records INFO (global column col0 + j + 1, the first one
// only) and is replaced by 1 so that what follows stays finite; kernels see
// a recorded INFO and do nothing.
constexpr int kChRows = 128;
__global__ void __launch_bounds__(kChRows)
    CholSubPanelKernel(int m, int w, double* a, long long lda, int* info, int col0,
                       unsigned int* arrivals) {
  __shared__ double s_l[32][33];
  __shared__ double s_x[32][kChRows + 1];
  __shared__ double s_rinv[32];
  __shared__ int s_bad;
  __shared__ bool s_last;
  if (*info != 0) return;
  const int tid = threadIdx.x, lane = tid % 32;
  for (int idx = tid; idx < 32 * 32; idx += kChRows) {
    const int i = idx % 32, j = idx / 32;
    s_l[i][j] = (i < w && j <= i) ? a[i + j * lda] : 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(arrivals, 1u) == gridDim.x - 1;
    if (s_last) *arrivals = 0u;  // every CTA has arrived: reset for the next launch
  }
  if (tid < 32) {
    // Warp 0, lane i holding row i in registers; left-looking:
    // l_ij = (a_ij - sum_{k<j} l_ik l_jk) / l_jj, row j's entries by shuffle.
    double row[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) row[k] = s_l[lane][k];
    int bad = -1;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < w) {
        double acc = row[j];
#pragma unroll
        for (int k = 0; k < j; ++k)
          acc = fma(-row[k], __shfl_sync(0xffffffffu, row[k], j), acc);
        const double d = __shfl_sync(0xffffffffu, acc, j);
        const bool ok = d > 0.0;  // false on NaN
        if (!ok && bad < 0) bad = j;
        const double l = ok ? sqrt(d) : 1.0;
        if (lane == j) row[j] = l;
        else if (lane > j) row[j] = acc / l;
      }
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) s_l[lane][k] = (lane < w && k <= lane) ? row[k] : 0.0;
    __syncwarp();
    if (lane < w) s_rinv[lane] = 1.0 / s_l[lane][lane];
    if (lane == 0) s_bad = bad;
  }
  __syncthreads();
  if (s_last) {
    if (tid == 0 && s_bad >= 0) *info = col0 + s_bad + 1;
    for (int idx = tid; idx < 32 * 32; idx += kChRows) {
      const int i = idx % 32, j = idx / 32;
      if (i < w && j <= i) a[i + j * lda] = s_l[i][j];
    }
  }
  // Rows below: x_j = (a_j - sum_{k<j} x_k l_jk) / l_jj.
  const int r = w + static_cast<int>(blockIdx.x) * kChRows + tid;
  if (r < m) {
    double x[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) x[j] = j < w ? a[r + j * lda] : 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < w) {
        double acc = x[j];
#pragma unroll
        for (int k = 0; k < j; ++k) acc = fma(-x[k], s_l[j][k], acc);
        x[j] = acc * s_rinv[j];
      }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < w) {
        a[r + j * lda] = x[j];
        s_x[j][tid] = x[j];
      }
    }
  }
  __syncthreads();
  // The transposed strip: rows 0..w, columns w + blockIdx.x * 128 + i.
  const int rows = min(kChRows, m - w - static_cast<int>(blockIdx.x) * kChRows);
  for (int idx = tid; idx < 32 * kChRows; idx += kChRows) {
    const int j = idx % 32, i = idx / 32;
    if (j < w && i < rows)
      a[j + (w + static_cast<long long>(blockIdx.x) * kChRows + i) * lda] = s_x[j][i];
  }
}

// Each sub-panel's pivots are relative to its first row c = (i / ib) * ib;
// make them relative to the panel's first row.
__global__ void PanelPivotOffsetKernel(int mn, int ib, int* ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mn) ipiv[i] += (i / ib) * ib;
}

// Tournament-pivoting leaf (CALU's TSLU) for an m x w block, w <= 32, in one
// cooperative launch of ceil(m / 512) CTAs. Partial pivoting over all m rows
// needs an exchange across CTAs for every column; a tournament needs none:
//
//   level 0   each CTA runs partial pivoting on its 512 rows (two a thread,
//             in registers) and proposes the w rows it picked, with their
//             original values;
//   merges    the last of up to 16 sibling CTAs to finish (an arrival
//             counter per tree node) runs partial pivoting on their
//             16 x 32 candidates, and so on up to the root, whose picks, in
//             its order, are the pivots; the root publishes U11 (its picked
//             rows after elimination), their original values and the
//             LAPACK-style ipiv;
//   apply     every CTA waits for the root and writes its rows:
//             (row after the interchanges) * U11^{-1}, i.e. L21, and for the
//             first w rows their L11 part next to U11.
//
// The factors are those of partial pivoting with the tournament's pivot
// order, a stable choice in practice (Grigori, Demmel, Xiang: "CALU: a
// communication optimal LU factorization algorithm", SIAM J. Matrix Anal.
// Appl. 32(4), 2011), and the mixed solver's refinement works from them.
constexpr int kTnRows = 512;      // rows per CTA, two a thread
constexpr int kTnThreads = 256;
constexpr int kTnRpt = kTnRows / kTnThreads;  // rows per thread
constexpr int kTnWarps = kTnThreads / 32;
constexpr int kTnW = 32;
constexpr int kTnFan = 16;        // candidate sets per merge: 16 x 32 rows
constexpr int kTnMaxLevels = 3;   // <= 148 CTAs -> 10 -> 1
constexpr int kTnMaxNodes = 160;
constexpr int kTnLd = kTnW + 1;   // padded row stride of the original rows
constexpr int kTnSmem = kTnRows * kTnLd * 8;

struct TnArgs {
  int m, w;
  double* a;
  long long lda;
  int* ipiv;
  int* info;
  int info_base;
  double* cand;            // [node][column][32] candidates' original values
  int* cidx;               // [node][32] their rows (relative to the leaf)
  int* ncand;              // [node]
  unsigned int* counters;  // [node] arrivals; the last arriver resets it
  double* top;             // [32][32] the leaf's original first w rows
  double* lu;              // [32][32] U11 rows in pivot order, shifted: U(k, k + j)
  double* wo;              // [32][32] the picked rows' original values, in order
  int* moved;              // [0] count, then (row, top row) pairs
  unsigned int* done;      // root finished: set to epoch
  unsigned int epoch;
  int levels;              // merge levels above level 0
  int lsize[kTnMaxLevels];
  int lbase[kTnMaxLevels];
  int* timeout_flag;
};

struct TnShared {
  double prow[2][kTnWarps][kTnW];  // each warp's best row (double-buffered by step)
  unsigned int bk[2][kTnWarps];    // its key (0: none)
  int bi[2][kTnWarps];             // its local row
  double rp[2][kTnWarps];          // 1 / its pivot value (0 for a zero pivot)
  int sel[kTnW];             // local row picked at each step
  int gid[kTnRows];          // local row -> leaf row
  __align__(16) double us[kTnW][kTnW];  // U11 rows shifted: us[k][j] = U(k, k + j)
  double rinv[kTnW];
  int mvrow[kTnW], mvsrc[kTnW];
  int content[2 * kTnW], posrow[2 * kTnW];
  int zero, last, ok;
};

// Pivot key of a value: the bits of |x| rounded up to float, plus 1 (positive
// floats order as their bits; 0 is left for "no candidate"; NaN sorts above
// infinity). A tournament only needs a large pivot, not the exact maximum.
__device__ __forceinline__ unsigned int TnKey(double x) {
  return __float_as_uint(__double2float_ru(fabs(x))) + 1u;
}

// 1 / x by two Newton steps x_{i+1} = x_i (2 - a x_i) from the float
// reciprocal (24 -> 48 -> full bits, within an ulp or two: a multiplier, not
// a result); exact division where the float seed would overflow or flush.
__device__ __forceinline__ double TnRecip(double a) {
  if (a == 0.0) return 0.0;  // a zero column: multipliers 0
  const double m = fabs(a);
  if (!(m > 1e-30 && m < 1e30)) return 1.0 / a;
  double r = static_cast<double>(__frcp_rn(static_cast<float>(a)));
  r = fma(r, fma(-a, r, 1.0), r);
  r = fma(r, fma(-a, r, 1.0), r);
  return r;
}

// Steps k0 .. min(k0 + 8, w) - 1 of the partial pivoting, on registers
// whose live columns fit the first WB (the other registers hold zeros).
// Returns false once there is nothing left to do (w reached or no rows).
template <int WB>
__device__ __forceinline__ bool TnSteps(double (&v)[kTnRpt][kTnW], bool (&act)[kTnRpt], int k0,
                                        int w, bool root, TnShared& s, int tid, int lane,
                                        int warp, int& nsel) {
#pragma unroll 1
  for (int kk = 0; kk < 8; ++kk) {
    const int k = k0 + kk;
    if (k >= w) return false;
    const int buf = k & 1;
    unsigned int mine = 0u;
    int mr = 0;
#pragma unroll
    for (int r = 0; r < kTnRpt; ++r) {
      const unsigned int kr = act[r] ? TnKey(v[r][0]) : 0u;
      if (kr > mine) mine = kr, mr = r;
    }
    const unsigned int wmax = __reduce_max_sync(0xffffffffu, mine);
    const unsigned int holders = __ballot_sync(0xffffffffu, wmax != 0u && mine == wmax);
    const int owner = holders ? __ffs(holders) - 1 : 0;
    if (holders == 0u) {
      if (lane == 0) s.bk[buf][warp] = 0u;
    } else if (lane == owner) {
      double2* dst = reinterpret_cast<double2*>(s.prow[buf][warp]);
      double piv = v[0][0];
#pragma unroll
      for (int r = 1; r < kTnRpt; ++r)
        if (mr == r) piv = v[r][0];
      s.rp[buf][warp] = TnRecip(piv);
#pragma unroll
      for (int j = 0; j < WB / 2; ++j) {
        double2 x = make_double2(v[0][2 * j], v[0][2 * j + 1]);
#pragma unroll
        for (int r = 1; r < kTnRpt; ++r)
          if (mr == r) x = make_double2(v[r][2 * j], v[r][2 * j + 1]);
        dst[j] = x;
      }
      s.bk[buf][warp] = wmax;
      s.bi[buf][warp] = tid + mr * kTnThreads;
    }
    __syncthreads();
    // Block maximum: lane q reads warp q's key (ties to the lower warp).
    const unsigned int okey = lane < kTnWarps ? s.bk[buf][lane] : 0u;
    const unsigned int gk = __reduce_max_sync(0xffffffffu, okey);
    if (gk == 0u) return false;
    const int gw = __ffs(__ballot_sync(0xffffffffu, lane < kTnWarps && okey == gk)) - 1;
    const int gi = s.bi[buf][gw];
    nsel = k + 1;
    if (tid == 0) s.sel[k] = gi;
#pragma unroll
    for (int r = 0; r < kTnRpt; ++r)
      if (gi == tid + r * kTnThreads) act[r] = false;
    const double* pr = s.prow[buf][gw];
    if (root && warp == kTnWarps - 1) {
      // U11 row k, shifted: us[k][j] = U(k, k + j).
      s.us[k][lane] = lane < WB ? pr[lane] : 0.0;
      if (lane == 0 && pr[0] == 0.0 && s.zero == INT_MAX) s.zero = k;
    }
    const double rp = s.rp[buf][gw];
    double prv[WB];
    const double2* pr2 = reinterpret_cast<const double2*>(pr);
#pragma unroll
    for (int q = 0; q < WB / 2; ++q) {
      const double2 x = pr2[q];
      prv[2 * q] = x.x;
      prv[2 * q + 1] = x.y;
    }
#pragma unroll
    for (int r = 0; r < kTnRpt; ++r) {
      if (act[r]) {
        const double l = v[r][0] * rp;
#pragma unroll
        for (int j = 1; j < WB; ++j) v[r][j - 1] = fma(-l, prv[j], v[r][j]);
        v[r][WB - 1] = 0.0;
      }
    }
  }
  return true;
}

// Partial pivoting over the CTA's active rows (local row tid + r * threads).
// Registers hold each row shifted: before step k, v[r][0..w-k) are columns
// k..w-1 and the rest zeros; the steps run in blocks of 8 whose register
// width shrinks with the live columns. Each step picks the largest key
// (ties: lower lane, then the thread's first row, then the lower warp),
// takes that row out of the active set and eliminates the others, shifting
// them one register left. At the root, U11 is recorded. Returns the number
// of picks (fewer than w only if rows run out).
__device__ __forceinline__ int TnGepp(double (&v)[kTnRpt][kTnW], bool (&act)[kTnRpt], int w,
                                      bool root, TnShared& s, int tid, int lane, int warp) {
  int nsel = 0;
  if (TnSteps<32>(v, act, 0, w, root, s, tid, lane, warp, nsel) &&
      TnSteps<24>(v, act, 8, w, root, s, tid, lane, warp, nsel) &&
      TnSteps<16>(v, act, 16, w, root, s, tid, lane, warp, nsel))
    TnSteps<8>(v, act, 24, w, root, s, tid, lane, warp, nsel);
  __syncthreads();
  return nsel;
}

// The apply step's substitution l = x U11^{-1} for steps k0 .. k0 + 7 (the
// thread's rows together, so each U11 row is read once), width WB.
template <int WB>
__device__ __forceinline__ void TnSolveSteps(double (&x)[kTnRpt][kTnW], int k0, int w,
                                             const TnShared& s, double* const (&out)[kTnRpt],
                                             const int (&g)[kTnRpt], long long lda) {
#pragma unroll 1
  for (int kk = 0; kk < 8; ++kk) {
    const int k = k0 + kk;
    if (k >= w) return;
    double uk[WB];
    const double2* u2 = reinterpret_cast<const double2*>(s.us[k]);
#pragma unroll
    for (int q = 0; q < WB / 2; ++q) {
      const double2 t = u2[q];
      uk[2 * q] = t.x;
      uk[2 * q + 1] = t.y;
    }
    const double ri = s.rinv[k];
#pragma unroll
    for (int r = 0; r < kTnRpt; ++r) {
      const double l = x[r][0] * ri;
      // The first w rows keep their L11 part and take U11.
      if (out[r] != nullptr) out[r][k * lda] = g[r] < w && k >= g[r] ? s.us[g[r]][k - g[r]] : l;
#pragma unroll
      for (int j = 1; j < WB; ++j) x[r][j - 1] = fma(-l, uk[j], x[r][j]);
      x[r][WB - 1] = 0.0;
    }
  }
}

__global__ void __launch_bounds__(kTnThreads, 1) TournamentLeafKernel(TnArgs p) {
  extern __shared__ __align__(16) double tn_orig[];  // [kTnRows][kTnLd] original rows
  __shared__ TnShared s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int w = p.w;
  const long long lda = p.lda;
  const int row0 = blockIdx.x * kTnRows;
  double v[kTnRpt][kTnW];
  bool act[kTnRpt];

  // Level 0: this CTA's rows, in registers and (original values) in shared
  // memory; CTA 0 also keeps the leaf's first w rows for the apply step.
  if (tid == 0) s.zero = INT_MAX;
#pragma unroll
  for (int r = 0; r < kTnRpt; ++r) {
    const int li = tid + r * kTnThreads, g = row0 + li;
    act[r] = g < p.m;
    s.gid[li] = g;
#pragma unroll
    for (int j = 0; j < kTnW; ++j) {
      const double x = (act[r] && j < w) ? p.a[g + j * lda] : 0.0;
      v[r][j] = x;
      tn_orig[li * kTnLd + j] = x;
    }
  }
  if (blockIdx.x == 0) {
    for (int idx = tid; idx < kTnW * kTnW; idx += kTnThreads) {
      const int i = idx / kTnW, j = idx % kTnW;
      p.top[idx] = (i < w && j < w) ? p.a[i + j * lda] : 0.0;
    }
  }
  __syncthreads();

  int level = 0, node = blockIdx.x;
  bool root = false;
  while (true) {
    root = level == p.levels;
    const int nsel = TnGepp(v, act, w, root, s, tid, lane, warp);
    if (root) break;
    // This node's candidates: their leaf rows and original values.
    const int gnode = p.lbase[level] + node;
    for (int idx = tid; idx < kTnW * kTnW; idx += kTnThreads) {
      const int j = idx / kTnW, kk = idx % kTnW;
      if (kk < nsel)
        p.cand[(static_cast<long long>(gnode) * kTnW + j) * kTnW + kk] =
            tn_orig[s.sel[kk] * kTnLd + j];
    }
    if (tid < nsel) p.cidx[gnode * kTnW + tid] = s.gid[s.sel[tid]];
    if (tid == 0) p.ncand[gnode] = nsel;
    // Arrive at the parent; the last of its children merges.
    const int parent = node / kTnFan;
    const int children = min(kTnFan, p.lsize[level] - parent * kTnFan);
    const int pnode = p.lbase[level + 1] + parent;
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      const unsigned int old = atomicAdd(&p.counters[pnode], 1u);
      const int last = old + 1 == static_cast<unsigned int>(children);
      if (last) {
        p.counters[pnode] = 0;  // ready for the next launch
        __threadfence();
      }
      s.last = last;
    }
    __syncthreads();
    if (!s.last) break;
    ++level;
    node = parent;
    const int cbase = p.lbase[level - 1] + parent * kTnFan;
#pragma unroll
    for (int r = 0; r < kTnRpt; ++r) {
      const int li = tid + r * kTnThreads, ci = li / kTnW, k = li % kTnW;
      const int cn = cbase + ci;
      const int nc = ci < children ? __ldcg(&p.ncand[cn]) : 0;
      act[r] = k < nc;
      s.gid[li] = act[r] ? __ldcg(&p.cidx[cn * kTnW + k]) : -1;
#pragma unroll
      for (int j = 0; j < kTnW; ++j) {
        const double x =
            (act[r] && j < w)
                ? __ldcg(&p.cand[(static_cast<long long>(cn) * kTnW + j) * kTnW + k])
                : 0.0;
        v[r][j] = x;
        tn_orig[li * kTnLd + j] = x;
      }
    }
    __syncthreads();
  }

  if (root) {
    // U11 (recorded by the pivoting), the picked rows' original values, the
    // first zero pivot, and ipiv.
    for (int idx = tid; idx < kTnW * kTnW; idx += kTnThreads) {
      const int i = idx / kTnW, j = idx % kTnW;
      p.lu[idx] = s.us[i][j];
      p.wo[idx] = i < w ? tn_orig[s.sel[i] * kTnLd + j] : 0.0;
    }
    if (warp == 0) {
      // Replay the interchanges on slots: 0..w-1 are the leaf's first rows,
      // then the picked rows below them; content = row whose values are there.
      const int g = lane < w ? s.gid[s.sel[lane]] : -1;
      const bool extra = lane < w && g >= w;
      const unsigned em = __ballot_sync(0xffffffffu, extra);
      const int er = __popc(em & ((1u << lane) - 1u));
      if (lane < w) s.posrow[lane] = lane, s.content[lane] = lane;
      if (extra) s.posrow[w + er] = g, s.content[w + er] = g;
      const int ns = w + __popc(em);
      __syncwarp();
      for (int i = 0; i < w; ++i) {
        const int gi = __shfl_sync(0xffffffffu, g, i);
        const bool h0 = lane < ns && s.content[lane] == gi;
        const bool h1 = lane + 32 < ns && s.content[lane + 32] == gi;
        const unsigned b0 = __ballot_sync(0xffffffffu, h0);
        const unsigned b1 = __ballot_sync(0xffffffffu, h1);
        const int t = b0 ? __ffs(b0) - 1 : 32 + __ffs(b1) - 1;
        if (lane == 0) {
          p.ipiv[i] = s.posrow[t] + 1;
          const int c = s.content[i];
          s.content[i] = s.content[t];
          s.content[t] = c;
        }
        __syncwarp();
      }
      // The picked rows below the first w now hold first rows.
      if (w + lane < ns) {
        p.moved[1 + 2 * lane] = s.posrow[w + lane];
        p.moved[2 + 2 * lane] = s.content[w + lane];
      }
      if (lane == 0) p.moved[0] = ns - w;
    }
    __syncthreads();
    if (tid == 0) {
      if (s.zero < w) atomicCAS(p.info, 0, p.info_base + s.zero + 1);
      __threadfence();
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p.done), "r"(p.epoch)
                   : "memory");
    }
  }

  // Apply: wait for the root, then write this CTA's rows.
  if (tid == 0) {
    uint32_t polls = 0;
    int good = 1;
    while (true) {
      unsigned int d;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(d) : "l"(p.done) : "memory");
      if (d == p.epoch) break;
      if ((++polls & 255u) == 0 &&
          (*reinterpret_cast<volatile int*>(p.timeout_flag) != 0 || polls >= kMaxPolls)) {
        atomicExch(p.timeout_flag, 1);
        good = 0;
        break;
      }
    }
    s.ok = good;
  }
  __syncthreads();
  if (!s.ok) return;
  for (int idx = tid; idx < kTnW * kTnW; idx += kTnThreads) {
    const int i = idx / kTnW, j = idx % kTnW;
    s.us[i][j] = (i < w && i + j < w) ? __ldcg(&p.lu[idx]) : 0.0;
  }
  const int nm = __ldcg(&p.moved[0]);
  if (tid < nm) {
    s.mvrow[tid] = __ldcg(&p.moved[1 + 2 * tid]);
    s.mvsrc[tid] = __ldcg(&p.moved[2 + 2 * tid]);
  }
  __syncthreads();
  if (tid < w) s.rinv[tid] = s.us[tid][0] != 0.0 ? 1.0 / s.us[tid][0] : 0.0;
  __syncthreads();
  const bool own_in_smem = level == 0;  // a merging CTA reloaded its shared rows
  // The rows' values after the interchanges: a picked row (the first w
  // rows), a first row moved down, or the row itself.
  double x[kTnRpt][kTnW];
  double* out[kTnRpt];
  int g[kTnRpt];
#pragma unroll
  for (int r = 0; r < kTnRpt; ++r) {
    const int li = tid + r * kTnThreads;
    g[r] = row0 + li;
    out[r] = g[r] < p.m ? p.a + g[r] : nullptr;
    int src = -1;
    for (int q = 0; q < nm; ++q)
      if (s.mvrow[q] == g[r]) src = s.mvsrc[q];
    // One source a row, then one batch of loads: scratch rows (zero beyond
    // w), this CTA's rows in shared memory, or the row in the matrix.
    if (out[r] == nullptr) {
#pragma unroll
      for (int j = 0; j < kTnW; ++j) x[r][j] = 0.0;
    } else if (g[r] < w || src >= 0) {
      const double* sp = g[r] < w ? p.wo + g[r] * kTnW : p.top + src * kTnW;
#pragma unroll
      for (int j = 0; j < kTnW; ++j) x[r][j] = __ldcg(sp + j);
    } else if (own_in_smem) {
#pragma unroll
      for (int j = 0; j < kTnW; ++j) x[r][j] = tn_orig[li * kTnLd + j];
    } else {
#pragma unroll
      for (int j = 0; j < kTnW; ++j) x[r][j] = j < w ? out[r][j * lda] : 0.0;
    }
  }
  // l = x U11^{-1}, one column a step: l_k = x_k / u_kk, then the rest of x
  // loses l_k * U(k, :) and shifts one register left.
  TnSolveSteps<32>(x, 0, w, s, out, g, lda);
  TnSolveSteps<24>(x, 8, w, s, out, g, lda);
  TnSolveSteps<16>(x, 16, w, s, out, g, lda);
  TnSolveSteps<8>(x, 24, w, s, out, g, lda);
}

// Co-resident CTAs of the tournament leaf (one a SM with its shared memory).
int TournamentCapacity() {
  static int capacity = -1;
  if (capacity < 0) {
    cudaFuncSetAttribute(TournamentLeafKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kTnSmem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, TournamentLeafKernel,
                                                      kTnThreads, kTnSmem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
    capacity = std::min(Ctx().num_sms * per_sm, kTnMaxNodes - 12);
  }
  return capacity;
}

bool TournamentFits(int m) {
  return (m + kTnRows - 1) / kTnRows <= TournamentCapacity();
}

// The tournament leaf on an m x w block (m >= w, w <= 32): ipiv relative to
// the block's first row, *info as GetrfLeaf. Requires TournamentFits(m).
void TournamentLeaf(int m, int w, double* a, int lda, int* ipiv, int* info, int info_base) {
  Context& ctx = Ctx();
  const int c0 = (m + kTnRows - 1) / kTnRows;
  TnArgs p = {};
  p.m = m;
  p.w = w;
  p.a = a;
  p.lda = lda;
  p.ipiv = ipiv;
  p.info = info;
  p.info_base = info_base;
  p.lsize[0] = c0;
  p.lbase[0] = 0;
  int L = 0;
  while (p.lsize[L] > 1) {
    p.lsize[L + 1] = (p.lsize[L] + kTnFan - 1) / kTnFan;
    p.lbase[L + 1] = p.lbase[L] + p.lsize[L];
    ++L;
  }
  p.levels = L;
  // Scratch: candidates, then the small arrays; counters and the done flag
  // are zeroed whenever the workspace is new.
  const size_t cand_bytes = sizeof(double) * kTnMaxNodes * kTnW * kTnW;
  const size_t small_bytes = sizeof(double) * 3 * kTnW * kTnW;
  const size_t int_elems = kTnMaxNodes * kTnW + kTnMaxNodes + (1 + 2 * kTnW);
  const size_t zero_elems = kTnMaxNodes + 1;  // counters, done
  uint8_t* ws = static_cast<uint8_t*>(
      Workspace(kWsTourney, cand_bytes + small_bytes + sizeof(int) * (int_elems + zero_elems)));
  if (ws == nullptr) return;
  p.cand = reinterpret_cast<double*>(ws);
  p.top = p.cand + kTnMaxNodes * kTnW * kTnW;
  p.lu = p.top + kTnW * kTnW;
  p.wo = p.lu + kTnW * kTnW;
  p.cidx = reinterpret_cast<int*>(p.wo + kTnW * kTnW);
  p.ncand = p.cidx + kTnMaxNodes * kTnW;
  p.moved = p.ncand + kTnMaxNodes;
  p.counters = reinterpret_cast<unsigned int*>(p.moved + 1 + 2 * kTnW);
  p.done = p.counters + kTnMaxNodes;
  static thread_local const void* zeroed = nullptr;
  static thread_local unsigned int epoch = 0;
  if (zeroed != ws || epoch == 0xffffffffu) {
    cudaMemsetAsync(p.counters, 0, sizeof(unsigned int) * zero_elems, ctx.stream);
    zeroed = ws;
    epoch = 0;
  }
  p.epoch = ++epoch;
  p.timeout_flag = ctx.dev_status;
  void* args[] = {&p};
  cudaEvent_t t0 = KernelTimerStart(kFamilyLuLeaf, ctx.stream);
  Failed(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(TournamentLeafKernel), c0,
                                     kTnThreads, args, kTnSmem, ctx.stream),
         "mixed tournament leaf");
  KernelTimerStop(t0, ctx.stream);
  CountLaunch();
}

// Leaf width of the mixed panels: 32 columns where the rows fit the
// 32-column cluster leaf (16 CTAs of 832 rows), else the 16-column leaf.
int PanelLeafWidth(int m) { return m <= 16 * 832 ? 32 : 16; }

}  // namespace

namespace {

// A stream for the panels' wide rank updates, at a priority between the
// look-ahead stream's (highest) and the default, and two events to order it
// against the stream the panel runs on.
struct PanelSide {
  cudaStream_t stream = nullptr;
  cudaEvent_t to_side = nullptr, to_panel = nullptr;
  bool ok = false;
};
PanelSide& GetPanelSide() {
  static thread_local PanelSide ps;
  static thread_local bool tried = false;
  if (!tried) {
    tried = true;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int prio = greatest < least ? greatest + 1 : greatest;
    ps.ok = cudaStreamCreateWithPriority(&ps.stream, cudaStreamNonBlocking, prio) ==
                cudaSuccess &&
            cudaEventCreateWithFlags(&ps.to_side, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&ps.to_panel, cudaEventDisableTiming) == cudaSuccess;
    if (!ps.ok) cudaGetLastError();
  }
  return ps;
}

void RankUpdate(int mr, int nr, int w, const double* l21, const double* u12, double* a22,
                int lda, cudaStream_t st, bool lower_only = false) {
  if (mr <= 0 || nr <= 0) return;
  PanelRankUpdateKernel<<<dim3((mr + kRkM - 1) / kRkM, (nr + kRkN - 1) / kRkN), 256, 0, st>>>(
      mr, nr, w, l21, lda, u12, lda, a22, lda, lower_only);
  CountLaunch();
  LaunchFailed("mixed panel update");
}

}  // namespace

// Sub-panel c's update is split: the next sub-panel's columns first, on the
// panel's stream, so that the next leaf can start; the columns beyond them
// on a side stream, overlapping that leaf. The next interchange+solve kernel
// touches those columns, so it waits for the side stream.
void MixedPanel(int m, int nc, double* a, int lda, int* ipiv, int* info, int col0) {
  Context& ctx = Ctx();
  const cudaStream_t st = ctx.stream;
  PanelSide& side = GetPanelSide();
  const bool tourney = TournamentFits(m);
  const int ib = tourney ? kTnW : PanelLeafWidth(m);
  const int mn = std::min(m, nc);
  if (mn <= 0) return;
  bool side_pending = false;
  for (int c = 0; c < mn; c += ib) {
    const int w = std::min(ib, mn - c);
    if (tourney)
      TournamentLeaf(m - c, w, At(a, lda, c, c), lda, ipiv + c, info, col0 + c);
    else
      GetrfLeaf<double>(m - c, w, At(a, lda, c, c), lda, ipiv + c, info, col0 + c, ib);
    if (side_pending) {
      cudaStreamWaitEvent(st, side.to_panel, 0);
      side_pending = false;
    }
    const int right = nc - c - w;
    const int blocks =
        (c + kSwapCols - 1) / kSwapCols + (right + kSwapCols - 1) / kSwapCols;
    if (blocks > 0) {
      PanelSwapSolveKernel<<<blocks, 256, 0, st>>>(w, c, c, c + w, right, a, lda, ipiv + c);
      CountLaunch();
      LaunchFailed("mixed panel interchanges");
    }
    const int mr = m - c - w;
    if (right <= 0 || mr <= 0) continue;
    const int near = std::min(right, ib);
    const double* l21 = At(a, lda, c + w, c);
    RankUpdate(mr, near, w, l21, At(a, lda, c, c + w), At(a, lda, c + w, c + w), lda, st);
    if (right > near) {
      const int far0 = c + w + near;
      if (side.ok) {
        cudaEventRecord(side.to_side, st);
        cudaStreamWaitEvent(side.stream, side.to_side, 0);
      }
      RankUpdate(mr, right - near, w, l21, At(a, lda, c, far0), At(a, lda, c + w, far0), lda,
                 side.ok ? side.stream : st);
      if (side.ok) {
        cudaEventRecord(side.to_panel, side.stream);
        side_pending = true;
      }
    }
  }
  if (side_pending) cudaStreamWaitEvent(st, side.to_panel, 0);
  PanelPivotOffsetKernel<<<(mn + 255) / 256, 256, 0, st>>>(mn, ib, ipiv);
  CountLaunch();
  LaunchFailed("mixed panel pivots");
}

// Lower Cholesky of an n x n diagonal block, right-looking over 32-column
// sub-panels: the sub-panel kernel, then the rank-32 update of the block's
// lower trailing part. The block's upper triangle is scratch (it receives
// the transposed panels); *info as PotrfPanel sets it; `arrivals` is one
// device word of scratch for this stream.
void CholBlock(int n, double* a, int lda, int* info, int col0, unsigned int* arrivals) {
  const cudaStream_t st = Ctx().stream;
  cudaMemsetAsync(arrivals, 0, sizeof(unsigned int), st);
  for (int c = 0; c < n; c += 32) {
    const int w = std::min(32, n - c), m = n - c, below = m - w;
    const int grid = std::max(1, (below + kChRows - 1) / kChRows);
    CholSubPanelKernel<<<grid, kChRows, 0, st>>>(m, w, At(a, lda, c, c), lda, info,
                                                 col0 + c, arrivals);
    CountLaunch();
    LaunchFailed("mixed cholesky panel");
    if (below > 0)
      RankUpdate(below, below, w, At(a, lda, c + w, c), At(a, lda, c, c + w),
                 At(a, lda, c + w, c + w), lda, st, true);
  }
}

}  // namespace hb
