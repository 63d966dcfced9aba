// LU panels of the mixed-precision dgesv (factor in reduced precision, refine
// in FP64). Only a stable pivoted LU is needed here, not the reference's
// recursive order (lapack.cc keeps that for the plain path), so a panel is
// factored right-looking over 32-column sub-panels, each with few launches:
//
//   leaf         pivot search, interchanges and scaling of the sub-panel over
//                all of the panel's rows;
//   swap+solve   the sub-panel's interchanges on every other column of the
//                panel, and U12 = L11^{-1} A12 on the columns to its right;
//   update       A22 -= L21 U12 (rank 32, the DMMA GEMM).
//
// Pivots are LAPACK-style (row i interchanged with row ipiv[i], 1-based) and
// end relative to the panel's first row.
#include <algorithm>

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

// Each sub-panel's pivots are relative to its first row c = (i / ib) * ib;
// make them relative to the panel's first row.
__global__ void PanelPivotOffsetKernel(int mn, int ib, int* ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mn) ipiv[i] += (i / ib) * ib;
}

// Leaf width of the mixed panels: 32 columns where the rows fit the
// 32-column cluster leaf (16 CTAs of 832 rows), else the 16-column leaf.
int PanelLeafWidth(int m) { return m <= 16 * 832 ? 32 : 16; }

}  // namespace

void MixedPanel(int m, int nc, double* a, int lda, int* ipiv, int* info, int col0) {
  Context& ctx = Ctx();
  const int ib = PanelLeafWidth(m);
  const int mn = std::min(m, nc);
  if (mn <= 0) return;
  for (int c = 0; c < mn; c += ib) {
    const int w = std::min(ib, mn - c);
    GetrfLeaf<double>(m - c, w, At(a, lda, c, c), lda, ipiv + c, info, col0 + c, ib);
    const int right = nc - c - w;
    const int blocks =
        (c + kSwapCols - 1) / kSwapCols + (right + kSwapCols - 1) / kSwapCols;
    if (blocks > 0) {
      PanelSwapSolveKernel<<<blocks, 256, 0, ctx.stream>>>(w, c, c, c + w, right, a, lda,
                                                           ipiv + c);
      CountLaunch();
      LaunchFailed("mixed panel interchanges");
    }
    if (right > 0 && m - c - w > 0)
      GemmFull<double>(false, false, m - c - w, right, w, -1.0, At(a, lda, c + w, c), lda,
                       At(a, lda, c, c + w), lda, 1.0, At(a, lda, c + w, c + w), lda);
  }
  PanelPivotOffsetKernel<<<(mn + 255) / 256, 256, 0, ctx.stream>>>(mn, ib, ipiv);
  CountLaunch();
  LaunchFailed("mixed panel pivots");
}

}  // namespace hb
