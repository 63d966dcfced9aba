// FP64 GEMM on the FP64 tensor pipe (DMMA), bit-identical to the reference.
//
// The reference computes every C element as a sequential FMA chain over k,
// restarted from 0 every KC = 256 (src/gemm_kernel-inl.h:72, 161-176;
// src/gemm-inl.h:176-178), and merges each chunk as r = alpha*acc, then
// C = r + C (beta 1), fma(C, beta, r) (other beta, first chunk only) or r
// (beta 0, C not read) (src/gemm_kernel-inl.h:182-224). Tiles of a triangular
// C that cross the diagonal are merged as r + beta*C instead
// (src/gemm-inl.h:110-130, 219-225).
//
// mma.sync.m16n8k8.f64 accumulates its 8 products in ascending k as a chain
// of correctly rounded FMAs starting from the C operand (measured on B200 on
// random operands spanning 2^-20..2^20: 38400 of 38400 outputs identical to
// the sequential chain), so chaining the MMAs in ascending k and restarting
// the accumulator every 256 reproduces the reference bit for bit.
//
// Tiling: a CTA computes a 128 x 64 tile of C with 8 consumer warps (32 x 32
// each: 2 x 4 MMAs per k8 step) and one producer warp that streams 16-deep k
// slices of op(A) (eight 16 x 16 boxes, M-contiguous) and op(B) (16 x 64,
// K-contiguous) into a 4-stage shared-memory ring with TMA (128-byte swizzle:
// the 16-byte chunk c of row r lands at chunk c ^ (r & 7)) and mbarriers.
// Which tile row/column each MMA row/column computes is a free choice, made so
// that every shared load is conflict free: MMA rows g and g+8 of a 16-row
// block take the adjacent tile rows 2c(g), 2c(g)+1 with c = [0,4,1,5,2,6,3,7]
// (one 16-byte load per A fragment pair; the 8 lanes of each 128-bit load
// phase hit 8 distinct chunks), and MMA column g takes tile column
// [0,2,4,6,1,3,5,7][g] of its 8-column block (the 16 lanes of each 64-bit
// load phase hit 16 distinct 8-byte slots).
#include <cuda.h>

#include <algorithm>
#include <cstdio>

#include "device.cuh"
#include "internal.h"

namespace hb {
namespace {

constexpr int kBM = 128, kBN = 64, kBK = 16, kStages = 4;
constexpr int kConsumerWarps = 8;
constexpr int kThreads = (kConsumerWarps + 1) * 32;
constexpr int kTileABytes = kBM * kBK * 8;  // 8 boxes of 16 (m) x 16 (k)
constexpr int kABoxBytes = 16 * kBK * 8;
constexpr int kTileBBytes = kBN * kBK * 8;
constexpr int kStageBytes = kTileABytes + kTileBBytes;
constexpr int kKtPerChunk = 256 / kBK;  // k-slices per reference KC chunk
constexpr int kSmemBytes = kStages * kStageBytes + 2 * kStages * 8 + 1024;

struct GemmParams {
  int m, n, k;
  double alpha, beta;
  double* c;
  long long ldc;
  int part;
  int tri;  // Tri: which operand is triangular (TRMM)
  // Split over the KC chunks of k: work item (tile, chunk) writes the
  // chunk's raw accumulators to partial[(chunk * n + j) * m + i].
  double* partial;
  int nchunks;
  int* timeout_flag;
  const int* guard;
};

// k range [*kb, *ke) that the reference multiplies for C(i, j) when an
// operand is triangular: NonZeroRange of the AVX-512 double micro-tile (MR 16,
// NR 12, MC 96, NC 4080) holding C(i, j) (src/gemm-inl.h:62-85). Row tiles
// start at multiples of 16 (MC is a multiple of MR); column tiles at
// multiples of 12 within NC blocks.
__device__ __forceinline__ void TriRange(const GemmParams& p, int i, int j, int* kb,
                                         int* ke) {
  *kb = 0;
  *ke = p.k;
  if (p.tri == kTriALower || p.tri == kTriAUpper) {
    const int i0 = i & ~15, mr = min(16, p.m - i0);
    if (p.tri == kTriALower) *ke = min(p.k, i0 + mr);
    else *kb = i0;
  } else if (p.tri == kTriBLower || p.tri == kTriBUpper) {
    constexpr int NR = 12, NC = 4080;
    const int jc = j / NC * NC, jr = (j - jc) / NR * NR;
    const int nr = min(NR, min(NC, p.n - jc) - jr);
    if (p.tri == kTriBLower) *kb = jc + jr;
    else *ke = min(p.k, jc + jr + nr);
  }
}

// The k-slices (of kBK) a tile of C needs: the union of its elements' ranges.
__device__ __forceinline__ void TileKRange(const GemmParams& p, int m0, int n0, int kt_total,
                                           int* kt_lo, int* kt_hi) {
  *kt_lo = 0;
  *kt_hi = kt_total;
  int kb, ke;
  switch (p.tri) {
    case kTriALower:
      TriRange(p, min(p.m, m0 + kBM) - 1, 0, &kb, &ke);
      *kt_hi = (ke + kBK - 1) / kBK;
      break;
    case kTriAUpper:
      *kt_lo = m0 / kBK;
      break;
    case kTriBLower:
      TriRange(p, 0, n0, &kb, &ke);
      *kt_lo = kb / kBK;
      break;
    case kTriBUpper:
      TriRange(p, 0, min(p.n, n0 + kBN) - 1, &kb, &ke);
      *kt_hi = (ke + kBK - 1) / kBK;
      break;
    default:
      break;
  }
}

// Whether C(i, j) lies in a micro-tile of the reference's AVX-512 double
// kernel (MR 16, NR 12, MC 96, NC 4080) that crosses the diagonal
// (src/gemm-inl.h:93-106; src/gemm_kernel-inl.h:64-74).
__device__ __forceinline__ bool InCrossingTile(int part, int m, int n, int i,
                                               int j) {
  constexpr int MR = 16, NR = 12, MC = 96, NC = 4080;
  const int ic = i / MC * MC, mcb = min(MC, m - ic);
  const int ir = (i - ic) / MR * MR, mr = min(MR, mcb - ir);
  const int jc = j / NC * NC, ncb = min(NC, n - jc);
  const int jr = (j - jc) / NR * NR, nr = min(NR, ncb - jr);
  const int i0 = ic + ir, j0 = jc + jr;
  if (part == kLower) return !(i0 > j0 + nr - 1);
  return !(i0 + mr - 1 < j0);
}

__device__ __forceinline__ bool InPart(const GemmParams& p, int i, int j) {
  if (i >= p.m || j >= p.n) return false;
  if (p.part == kLower) return i >= j;
  if (p.part == kUpper) return i <= j;
  return true;
}

// Tile `tile` in groups of 16 tile rows: consecutive tiles walk down a band
// of 16 tile rows column by column, so the tiles in flight at once form a
// compact block of C and share their A and B tiles in L2.
__device__ __forceinline__ void TileOrigin(int tile, int tiles_m, int tiles_n,
                                           int* m0, int* n0) {
  const int per_group = 16 * tiles_n;
  const int first_m = (tile / per_group) * 16;
  const int gm = min(tiles_m - first_m, 16);
  const int in_group = tile % per_group;
  *m0 = (first_m + in_group % gm) * kBM;
  *n0 = (in_group / gm) * kBN;
}

// Tiles entirely outside a triangular C part are skipped.
__device__ __forceinline__ bool SkipTile(const GemmParams& p, int m0, int n0) {
  if (p.part == kLower && m0 + kBM - 1 < n0) return true;
  if (p.part == kUpper && m0 > n0 + kBN - 1) return true;
  return false;
}

__device__ __forceinline__ void Dmma(double (&d)[4], const double (&a)[4],
                                     double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

// Producer cursor: the TMA loads of the CTA's k-slices in order, across
// tile boundaries (kt = -1: the current tile's slices are not yet known).
struct Producer {
  int tile, kt, kt_hi, gs;
};

// The k-slices [*lo, *hi) of work item w (a tile, or a tile's chunk when
// split); false when the tile lies outside C's part.
template <bool kTri, bool kSplit>
__device__ __forceinline__ bool WorkRange(const GemmParams& p, int w, int tiles_m, int tiles_n,
                                          int kt_total, int* m0, int* n0, int* lo, int* hi) {
  const int tile = kSplit ? w / p.nchunks : w;
  TileOrigin(tile, tiles_m, tiles_n, m0, n0);
  if (SkipTile(p, *m0, *n0)) return false;
  *lo = 0;
  *hi = kt_total;
  if constexpr (kTri) TileKRange(p, *m0, *n0, kt_total, lo, hi);
  if constexpr (kSplit) {
    const int c = w % p.nchunks;
    *lo = max(*lo, c * kKtPerChunk);
    *hi = min(*hi, (c + 1) * kKtPerChunk);
  }
  return true;
}

template <bool kTri, bool kSplit>
__device__ __forceinline__ bool IssueNext(Producer& pr, const GemmParams& p,
                                          int tiles_m, int tiles_n, int kt_total,
                                          uint8_t* smem, uint64_t* full,
                                          uint64_t* empty, const CUtensorMap* tm_a,
                                          const CUtensorMap* tm_b) {
  const int num_tiles = tiles_m * tiles_n;
  const int num_work = kSplit ? num_tiles * p.nchunks : num_tiles;
  int m0 = 0, n0 = 0;
  while (pr.tile < num_work) {
    if constexpr (!kTri && !kSplit) {
      TileOrigin(pr.tile, tiles_m, tiles_n, &m0, &n0);
      if (!SkipTile(p, m0, n0)) break;
    } else {
      int lo, hi;
      if (WorkRange<kTri, kSplit>(p, pr.tile, tiles_m, tiles_n, kt_total, &m0, &n0, &lo,
                                  &hi)) {
        if (pr.kt >= 0) break;
        if (lo < hi) {
          pr.kt = lo;
          pr.kt_hi = hi;
          break;
        }
      }
    }
    pr.tile += gridDim.x;
    if constexpr (kTri || kSplit) pr.kt = -1;
  }
  if (pr.tile >= num_work) return true;
  const int s = pr.gs % kStages, round = pr.gs / kStages;
  if (round > 0 && !MbarWait(&empty[s], (round - 1) & 1, p.timeout_flag)) return false;
  uint8_t* st = smem + s * kStageBytes;
  MbarArriveExpectTx(&full[s], kStageBytes);
#pragma unroll
  for (int b = 0; b < kBM / 16; ++b)
    TmaLoad2d(st + b * kABoxBytes, tm_a, m0 + 16 * b, pr.kt * kBK, &full[s]);
  TmaLoad2d(st + kTileABytes, tm_b, pr.kt * kBK, n0, &full[s]);
  ++pr.gs;
  if (++pr.kt == ((kTri || kSplit) ? pr.kt_hi : kt_total)) {
    pr.kt = (kTri || kSplit) ? -1 : 0;
    pr.tile += gridDim.x;
  }
  return true;
}

// 168 registers: nine warps of a CTA share the 16K registers of each SM
// sub-partition three at a time.
//
// kTri (TRMM): each tile loads only the k-slices its elements need; a 16-row
// MMA block is exactly one reference row micro-tile, so for a triangular
// op(A) its MMAs run only inside that tile's k range. Reference column
// micro-tiles are 12 wide, so an 8-column MMA block of a triangular op(B) can
// span two ranges: its k8 steps inside both run as MMAs, those outside both
// are skipped, and the (at most two) steps in between run as per-element FMA
// chains over the in-range k only, in the MMA's own ascending order. A chunk
// whose range is empty for an element leaves it unmerged, as the reference
// skips that micro-tile (src/gemm-inl.h:202-209).
template <int kTriKind, bool kSplit>
__global__ void __maxnreg__(168)
    DgemmDmmaKernel(const __grid_constant__ CUtensorMap tm_a,
                    const __grid_constant__ CUtensorMap tm_b, GemmParams p) {
  // kTriKind: 0 no triangular operand, 1 op(A) triangular, 2 op(B).
  constexpr bool kTri = kTriKind != 0, kTriA = kTriKind == 1, kTriB = kTriKind == 2;
  if (p.guard != nullptr && *p.guard != 0) return;
  // Persistent: CTA b computes tiles b, b + gridDim.x, ... The producer
  // streams the k-slices across tile boundaries (the stage counter gs runs
  // over all of the CTA's k-slices), so the next tile's loads overlap this
  // tile's epilogue.
  const int tiles_m = (p.m + kBM - 1) / kBM, tiles_n = (p.n + kBN - 1) / kBN;
  const int num_tiles = tiles_m * tiles_n;
  const int num_work = kSplit ? num_tiles * p.nchunks : num_tiles;

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024 - (SmemAddr(smem_raw) & 1023)) & 1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      MbarInit(&full[s], 1);
      MbarInit(&empty[s], kConsumerWarps);
    }
    FenceBarrierInit();
  }
  __syncthreads();
  const int kt_total = (p.k + kBK - 1) / kBK;
  if (warp == kConsumerWarps) {
    // Producer warp: one lane streams the k-slices through the ring.
    if (lane == 0) {
      PrefetchTmap(&tm_a);
      PrefetchTmap(&tm_b);
      Producer pr{static_cast<int>(blockIdx.x), (kTri || kSplit) ? -1 : 0, 0, 0};
      while (pr.tile < num_work) {
        if (!IssueNext<kTri, kSplit>(pr, p, tiles_m, tiles_n, kt_total, smem, full, empty,
                                     &tm_a, &tm_b))
          return;
      }
    }
    return;
  }

  const int wm = warp % 4, wn = warp / 4;
  const int g = lane >> 2, t = lane & 3;
  // Tile-row pair of MMA rows (g, g+8) and tile columns of MMA columns 2t,
  // 2t+1 (see the file comment).
  const int cg = (g >> 1) + 4 * (g & 1);
  const int ccol0 = 2 * ((2 * t) & 3) + ((2 * t) >> 2);
  const int ccol1 = 2 * ((2 * t + 1) & 3) + ((2 * t + 1) >> 2);
  const int bcol = 2 * (g & 3) + (g >> 2);  // tile column of this lane's B
  int gs = 0;
  for (int w = blockIdx.x; w < num_work; w += gridDim.x) {
    int m0, n0, kt_lo = 0, kt_hi = kt_total;
    if constexpr (!kTri && !kSplit) {
      TileOrigin(w, tiles_m, tiles_n, &m0, &n0);
      if (SkipTile(p, m0, n0)) continue;
    } else {
      if (!WorkRange<kTri, kSplit>(p, w, tiles_m, tiles_n, kt_total, &m0, &n0, &kt_lo,
                                   &kt_hi))
        continue;
      if (kSplit && kt_lo >= kt_hi) continue;
    }
    // Element e of MMA (mb, nb) is C(row0 + mb*16 + (e >> 1),
    // col0 + nb*8 + (e & 1 ? ccol1 : ccol0)).
    const int row0 = m0 + wm * 32 + 2 * cg, col0 = n0 + wn * 32;
    double acc[2][4][4];
    // C_in, loaded before the MMAs so that the loads overlap them, then the
    // running value merged at the end of every 256-deep chunk.
    double cacc[2][4][4];
    uint32_t in_part = 0, crossing = 0;
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
      for (int nb = 0; nb < 4; ++nb)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int bit = (mb * 4 + nb) * 4 + e;
          const int i = row0 + mb * 16 + (e >> 1);
          const int j = col0 + nb * 8 + ((e & 1) ? ccol1 : ccol0);
          acc[mb][nb][e] = 0.0;
          const bool inside = InPart(p, i, j);
          if (inside) in_part |= 1u << bit;
          if (inside && p.part != kAll && InCrossingTile(p.part, p.m, p.n, i, j))
            crossing |= 1u << bit;
          cacc[mb][nb][e] =
              (!kSplit && inside && p.beta != 0.0) ? p.c[i + j * p.ldc] : 0.0;
        }
    // kTri: k ranges of the 16-row blocks [xb, xe) (op(A) triangular), and the
    // union [ub, ue) and intersection [ib, ie) of the ranges of the 8-column
    // blocks' columns (op(B) triangular; ranges are monotone in j, so the
    // first and last columns bound them). Blocks wholly outside C get empty
    // ranges.
    int xb[2] = {0, 0}, xe[2] = {p.k, p.k};
    int ub[4] = {0, 0, 0, 0}, ue[4] = {p.k, p.k, p.k, p.k};
    int ib[4] = {0, 0, 0, 0}, ie[4] = {p.k, p.k, p.k, p.k};
    if constexpr (kTri) {
      const int fr = m0 + wm * 32;
#pragma unroll
      for (int mb = 0; mb < 2; ++mb) {
        if (fr + mb * 16 >= p.m) {
          xb[mb] = xe[mb] = 0;
        } else if (kTriA) {
          TriRange(p, fr + mb * 16, 0, &xb[mb], &xe[mb]);
        }
      }
#pragma unroll
      for (int nb = 0; nb < 4; ++nb) {
        if constexpr (!kTriB) break;
        const int j0 = col0 + nb * 8, j1 = min(j0 + 7, p.n - 1);
        if (j0 >= p.n) {
          ub[nb] = ue[nb] = ib[nb] = ie[nb] = 0;
        } else {
          int b0, e0, b1, e1;
          TriRange(p, 0, j0, &b0, &e0);
          TriRange(p, 0, j1, &b1, &e1);
          ub[nb] = min(b0, b1);
          ib[nb] = max(b0, b1);
          ue[nb] = max(e0, e1);
          ie[nb] = min(e0, e1);
        }
      }
    }

    // Merge of chunk `chunk` (256 deep) into the running C values.
    const auto merge = [&](int chunk) {
      const bool first = (chunk == 0);
      const int c_lo = chunk * 256, c_hi = min(p.k, c_lo + 256);
#pragma unroll
      for (int mb = 0; mb < 2; ++mb)
#pragma unroll
        for (int nb = 0; nb < 4; ++nb)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int bit = (mb * 4 + nb) * 4 + e;
            bool skip = false;
            if constexpr (kTriA) {
              // The range is the 16-row block's.
              if (!first) skip = max(xb[mb], c_lo) >= min(xe[mb], c_hi);
            } else if constexpr (kTriB) {
              if (!first) {
                int kb, ke;
                TriRange(p, row0 + mb * 16 + (e >> 1),
                         col0 + nb * 8 + ((e & 1) ? ccol1 : ccol0), &kb, &ke);
                skip = max(kb, c_lo) >= min(ke, c_hi);
              }
            }
            const double r = p.alpha * acc[mb][nb][e];
            double& cv = cacc[mb][nb][e];
            if (skip) {
              // Outside the element's k range: not merged.
            } else if (!first || p.beta == 1.0) {
              cv = r + cv;
            } else if (p.beta == 0.0) {
              cv = r;
            } else if ((crossing >> bit) & 1u) {
              const double bc = p.beta * cv;
              cv = r + bc;
            } else {
              cv = fma(cv, p.beta, r);
            }
            acc[mb][nb][e] = 0.0;
          }
    };
    // Chunk 0 lies before the tile's first k-slice: its k range is empty for
    // every element, and the reference still applies beta (with alpha * 0).
    if (kTri && !kSplit && !(kt_lo < kt_hi && kt_lo < kKtPerChunk)) merge(0);

    for (int kt = kt_lo; kt < kt_hi; ++kt, ++gs) {
      const int s = gs % kStages, round = gs / kStages;
      if (!MbarWait(&full[s], round & 1, p.timeout_flag)) return;
      const double* sa = reinterpret_cast<const double*>(smem + s * kStageBytes);
      const uint8_t* sb = smem + s * kStageBytes + kTileABytes;
#pragma unroll
      for (int ks = 0; ks < kBK / 8; ++ks) {
        double af[2][4];
        const int klo = ks * 8 + t, khi = klo + 4;
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const uint8_t* box = reinterpret_cast<const uint8_t*>(sa) +
                               (wm * 2 + mb) * kABoxBytes;
          const double2 lo = *reinterpret_cast<const double2*>(
              box + klo * 128 + ((cg ^ (klo & 7)) << 4));
          const double2 hi = *reinterpret_cast<const double2*>(
              box + khi * 128 + ((cg ^ (khi & 7)) << 4));
          af[mb][0] = lo.x;
          af[mb][1] = lo.y;
          af[mb][2] = hi.x;
          af[mb][3] = hi.y;
        }
        const int kg = kt * kBK + ks * 8, kend = min(kg + 8, p.k);
#pragma unroll
        for (int nb = 0; nb < 4; ++nb) {
          const int r = wn * 32 + nb * 8 + bcol;
          const int k0 = ks * 8 + t, k1 = k0 + 4;
          const double b0 = *reinterpret_cast<const double*>(
              sb + r * 128 + (((k0 >> 1) ^ (r & 7)) << 4) + ((k0 & 1) << 3));
          const double b1 = *reinterpret_cast<const double*>(
              sb + r * 128 + (((k1 >> 1) ^ (r & 7)) << 4) + ((k1 & 1) << 3));
          if constexpr (!kTri) {
            Dmma(acc[0][nb], af[0], b0, b1);
            Dmma(acc[1][nb], af[1], b0, b1);
          } else if constexpr (kTriA) {
            if (kg >= p.k) continue;
#pragma unroll
            for (int mb = 0; mb < 2; ++mb)
              if (kg >= xb[mb] && kg < xe[mb]) Dmma(acc[mb][nb], af[mb], b0, b1);
          } else {
            if (kg >= p.k || kend <= ub[nb] || kg >= ue[nb]) continue;
            if (kg >= ib[nb] && kend <= ie[nb]) {
#pragma unroll
              for (int mb = 0; mb < 2; ++mb)
                if (kg >= xb[mb] && kg < xe[mb]) Dmma(acc[mb][nb], af[mb], b0, b1);
              continue;
            }
            // Per-element chains (only for a triangular op(B), whose op(A)
            // blocks all need every k).
#pragma unroll
            for (int mb = 0; mb < 2; ++mb) {
              const uint8_t* box = reinterpret_cast<const uint8_t*>(sa) +
                                   (wm * 2 + mb) * kABoxBytes;
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                const int col = (e & 1) ? ccol1 : ccol0;
                const int rc = wn * 32 + nb * 8 + col;
                int kb, ke;
                TriRange(p, 0, col0 + nb * 8 + col, &kb, &ke);
                double a_acc = acc[mb][nb][e];
                for (int q = 0; q < 8; ++q) {
                  const int kk = ks * 8 + q, kq = kg + q;
                  if (kq < kb || kq >= ke) continue;
                  const double av = *reinterpret_cast<const double*>(
                      box + kk * 128 + ((cg ^ (kk & 7)) << 4) + (e >> 1) * 8);
                  const double bv = *reinterpret_cast<const double*>(
                      sb + rc * 128 + (((kk >> 1) ^ (rc & 7)) << 4) + ((kk & 1) << 3));
                  a_acc = fma(av, bv, a_acc);
                }
                acc[mb][nb][e] = a_acc;
              }
            }
          }
        }
      }
      // The stage was read through the generic proxy and will be rewritten
      // by TMA (the async proxy): the proxy fence orders this warp's reads
      // before the release. Without it B200 showed stale-stage reads (one
      // warp's 16 x 32 block wrong in about 1 of 4 GEMMs of 8128^2 x 64).
      __syncwarp();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (lane == 0) MbarArrive(&empty[s]);

      // End of a reference KC chunk: merge into the running C value.
      if (!kSplit && ((kt + 1) % kKtPerChunk == 0 || kt + 1 == kt_hi))
        merge(kt / kKtPerChunk);
    }

    // Epilogue: write C, or the chunk's raw accumulators.
    const long long pbase =
        kSplit ? static_cast<long long>(w % p.nchunks) * p.n * static_cast<long long>(p.m) : 0;
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
      for (int nb = 0; nb < 4; ++nb)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int bit = (mb * 4 + nb) * 4 + e;
          if (!((in_part >> bit) & 1u)) continue;
          const int i = row0 + mb * 16 + (e >> 1);
          const int j = col0 + nb * 8 + ((e & 1) ? ccol1 : ccol0);
          if constexpr (kSplit) {
            p.partial[pbase + static_cast<long long>(j) * p.m + i] = acc[mb][nb][e];
          } else {
            p.c[i + j * p.ldc] = cacc[mb][nb][e];
          }
        }
  }
}

// The merge after a split launch: for each element of C's part, the chunks
// in order, exactly as the tile kernel merges them (a chunk outside a
// triangular operand's range for the element is skipped; chunk 0 still
// applies beta, with a zero accumulator when its range is empty).
__global__ void __launch_bounds__(256) DgemmSplitMergeKernel(GemmParams p) {
  if (p.guard != nullptr && *p.guard != 0) return;
  const long long total = static_cast<long long>(p.m) * p.n;
  const long long plane = total;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % p.m), j = static_cast<int>(e / p.m);
    if (!InPart(p, i, j)) continue;
    const bool crossing = p.part != kAll && InCrossingTile(p.part, p.m, p.n, i, j);
    int kb = 0, ke = p.k;
    if (p.tri != kTriNone) TriRange(p, i, j, &kb, &ke);
    double cv = 0.0;
    for (int c = 0; c < p.nchunks; ++c) {
      const bool nonempty = max(c * 256, kb) < min(min(p.k, c * 256 + 256), ke);
      if (!nonempty && c != 0) continue;
      const double acc = nonempty ? p.partial[c * plane + e] : 0.0;
      const double r = p.alpha * acc;
      if (c != 0 || p.beta == 1.0) {
        if (c == 0) cv = p.c[i + j * p.ldc];
        cv = r + cv;
      } else if (p.beta == 0.0) {
        cv = r;
      } else {
        const double cin = p.c[i + j * p.ldc];
        if (crossing) {
          const double bc = p.beta * cin;
          cv = r + bc;
        } else {
          cv = fma(cin, p.beta, r);
        }
      }
    }
    p.c[i + j * p.ldc] = cv;
  }
}

// Short products (k <= 64, inside one reference chunk): the LU's trailing
// updates C -= L21 U12 at k = nb = 64 and the TRSM recursion's updates. At
// such k the tile kernel's TMA ring barely fills before a tile ends, and each
// tile then waits on its C. Here small CTAs (4 warps, three an SM) each walk
// 64 x 32 tiles of C: cp.async brings the tile's A (64 x k), B (k x 32) and
// C into shared memory, each warp computes 32 x 16 of the tile with m16n8k8
// chains over k in ascending order from zero (the reference's chain), then
// merges alpha*acc into C with the reference's rules and stores straight
// from registers. The CTAs of an SM overlap one another's loads and
// products. (Measured on B200 at 16384 x 16384 x 64: 19.7 TFLOP/s, against
// 16.8 for one 8-warp CTA an SM that prefetched the next 64 x 64 tile and
// 12 for the tile kernel; every variant gave the same bits.) Operand rows
// are padded to 68 doubles and C's to 66, which makes every fragment and
// accumulator access conflict free. Canonical operands only (column-major,
// 16-byte aligned base and leading dimension), no triangular operand; a
// triangular C part (SYRK) skips the tiles outside it and merges with the
// reference's crossing-tile rule.
constexpr int kSkM = 64, kSkN = 32, kSkK = 64;
constexpr int kSkLdAB = kSkK + 4;   // shared row stride of A and B (doubles)
constexpr int kSkLdBt = kSkN + 4;   // of a transposed B (k rows of 32)
constexpr int kSkLdC = kSkM + 2;    // shared row stride of C
constexpr int kSkSizeB = kSkK * kSkLdBt;  // >= kSkN * kSkLdAB
constexpr int kSkSmemBytes = (kSkK * kSkLdAB + kSkSizeB + kSkN * kSkLdC) * 8;
constexpr int kSkThreads = 128;
constexpr int kSkPerSm = 3;

__device__ __forceinline__ void ShortKTile(int tile, int tiles_m, int tiles_n, int* m0,
                                           int* n0) {
  constexpr int kGroup = 16;  // bands of 16 tile rows, walked column by column
  const int per_group = kGroup * tiles_n;
  const int first_m = (tile / per_group) * kGroup;
  const int gm = min(tiles_m - first_m, kGroup);
  const int in_group = tile % per_group;
  *m0 = (first_m + in_group % gm) * kSkM;
  *n0 = (in_group / gm) * kSkN;
}

// kTA / kTB: op(A) = A^T (A(i, q) at a[q + i lda]) / op(B) = B^T; shared
// memory keeps each operand's contiguous index contiguous.
template <bool kTA, bool kTB, bool kPart>
__global__ void __launch_bounds__(kSkThreads, kSkPerSm)
    DgemmShortKKernel(GemmParams p, const double* __restrict__ a, long long lda,
                      const double* __restrict__ b, long long ldb) {
  if (p.guard != nullptr && *p.guard != 0) return;
  extern __shared__ __align__(16) double sk_smem[];
  double* sA = sk_smem;                   // sA[q][i] (kTA: sA[i][q]) = op(A)(m0 + i, q)
  double* sB = sA + kSkK * kSkLdAB;       // sB[j][q] (kTB: sB[q][j]) = op(B)(q, n0 + j)
  double* sC = sB + kSkSizeB;             // sC[j][i] = C(m0 + i, n0 + j)
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp % 2, wn = warp / 2;  // warp tile: rows 32 wm, columns 16 wn
  const int tiles_m = (p.m + kSkM - 1) / kSkM, tiles_n = (p.n + kSkN - 1) / kSkN;
  const int tiles = tiles_m * tiles_n;
  const int k = p.k;
  const bool read_c = p.beta != 0.0;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    int m0, n0;
    ShortKTile(tile, tiles_m, tiles_n, &m0, &n0);
    if (kPart &&
        ((p.part == kLower && m0 + kSkM - 1 < n0) || (p.part == kUpper && m0 > n0 + kSkN - 1)))
      continue;  // wholly outside C's part
    __syncthreads();  // the previous tile's reads are done
    // 16-byte chunks (two doubles along the contiguous index); chunks past
    // the matrices' edges read only their valid doubles and are zero-filled.
    for (int ch = tid; ch < kSkK * kSkM / 2; ch += kSkThreads) {
      if (!kTA) {
        const int q = ch / (kSkM / 2), r2 = (ch % (kSkM / 2)) * 2;
        const int rows = min(2, p.m - m0 - r2);
        const bool ok = q < k && rows > 0;
        CpAsync16(sA + q * kSkLdAB + r2, ok ? a + (m0 + r2) + q * lda : a, ok ? rows * 8 : 0);
      } else {
        const int i = ch / (kSkK / 2), q2 = (ch % (kSkK / 2)) * 2;
        const int qs = min(2, k - q2);
        const bool ok = m0 + i < p.m && qs > 0;
        CpAsync16(sA + i * kSkLdAB + q2, ok ? a + q2 + (m0 + i) * lda : a, ok ? qs * 8 : 0);
      }
    }
    for (int ch = tid; ch < kSkN * kSkK / 2; ch += kSkThreads) {
      if (!kTB) {
        const int j = ch / (kSkK / 2), q2 = (ch % (kSkK / 2)) * 2;
        const int qs = min(2, k - q2);
        const bool ok = n0 + j < p.n && qs > 0;
        CpAsync16(sB + j * kSkLdAB + q2, ok ? b + q2 + (n0 + j) * ldb : b, ok ? qs * 8 : 0);
      } else {
        const int q = ch / (kSkN / 2), j2 = (ch % (kSkN / 2)) * 2;
        const int cols = min(2, p.n - n0 - j2);
        const bool ok = q < k && cols > 0;
        CpAsync16(sB + q * kSkLdBt + j2, ok ? b + (n0 + j2) + q * ldb : b, ok ? cols * 8 : 0);
      }
    }
    if (read_c) {
      for (int ch = tid; ch < kSkN * kSkM / 2; ch += kSkThreads) {
        const int j = ch / (kSkM / 2), r2 = (ch % (kSkM / 2)) * 2;
        const int rows = min(2, p.m - m0 - r2);
        const bool ok = n0 + j < p.n && rows > 0;
        CpAsync16(sC + j * kSkLdC + r2, ok ? p.c + (m0 + r2) + (n0 + j) * p.ldc : p.c,
                  ok ? rows * 8 : 0);
      }
    }
    CpAsyncCommit();
    CpAsyncWait<0>();
    __syncthreads();
    double acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    const int steps = (k + 7) / 8;
    for (int ks = 0; ks < steps; ++ks) {
      double af[2][4], bf[2][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = wm * 32 + i * 16 + g, q = ks * 8 + t4;
        if (!kTA) {
          const double* pa = sA + q * kSkLdAB + row;
          af[i][0] = pa[0];
          af[i][1] = pa[8];
          af[i][2] = pa[4 * kSkLdAB];
          af[i][3] = pa[4 * kSkLdAB + 8];
        } else {
          const double* pa = sA + row * kSkLdAB + q;
          af[i][0] = pa[0];
          af[i][1] = pa[8 * kSkLdAB];
          af[i][2] = pa[4];
          af[i][3] = pa[8 * kSkLdAB + 4];
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int col = wn * 16 + j * 8 + g, q = ks * 8 + t4;
        if (!kTB) {
          const double* pb = sB + col * kSkLdAB + q;
          bf[j][0] = pb[0];
          bf[j][1] = pb[4];
        } else {
          const double* pb = sB + q * kSkLdBt + col;
          bf[j][0] = pb[0];
          bf[j][1] = pb[4 * kSkLdBt];
        }
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
              "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1]), "+d"(acc[i][j][2]),
                "+d"(acc[i][j][3])
              : "d"(af[i][0]), "d"(af[i][1]), "d"(af[i][2]), "d"(af[i][3]), "d"(bf[j][0]),
                "d"(bf[j][1]));
    }
    // Merge (each element read and written by its own thread).
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int r = wm * 32 + i * 16 + g + (e >> 1) * 8;
          const int c = wn * 16 + j * 8 + 2 * t4 + (e & 1);
          if (!kPart && m0 + r < p.m && n0 + c < p.n) {
            const double v = p.alpha * acc[i][j][e];
            const double cin = sC[c * kSkLdC + r];
            p.c[(m0 + r) + static_cast<long long>(n0 + c) * p.ldc] =
                p.beta == 1.0 ? v + cin : p.beta == 0.0 ? v : fma(cin, p.beta, v);
          } else if (kPart && InPart(p, m0 + r, n0 + c)) {
            const double v = p.alpha * acc[i][j][e];
            const double cin = sC[c * kSkLdC + r];
            double cv;
            if (p.beta == 1.0) {
              cv = v + cin;
            } else if (p.beta == 0.0) {
              cv = v;
            } else if (InCrossingTile(p.part, p.m, p.n, m0 + r, n0 + c)) {
              const double bc = p.beta * cin;
              cv = v + bc;
            } else {
              cv = fma(cin, p.beta, v);
            }
            p.c[(m0 + r) + static_cast<long long>(n0 + c) * p.ldc] = cv;
          }
        }
  }
}

// Small products: one thread per C element, the same FMA chain over k in
// chunks of 256 and the same merges as the tensor-core kernel (so the same
// bits), without its TMA pipeline whose fixed costs dominate tiny shapes.
__global__ void __launch_bounds__(256)
    DgemmDirectKernel(GemmParams p, View<double> a, View<double> b) {
  if (p.guard != nullptr && *p.guard != 0) return;
  const int i = blockIdx.x * 32 + threadIdx.x % 32;
  const int j = blockIdx.y * 8 + threadIdx.x / 32;
  if (!InPart(p, i, j)) return;
  const bool crossing = p.part != kAll && InCrossingTile(p.part, p.m, p.n, i, j);
  int kb = 0, ke = p.k;
  if (p.tri != kTriNone) TriRange(p, i, j, &kb, &ke);
  double cv = 0.0;
  for (int pc = 0; pc < p.k; pc += 256) {
    const int lo = max(pc, kb), hi = min(min(p.k, pc + 256), ke);
    if (lo >= hi && pc != 0) continue;  // the reference skips the micro-tile
    double acc = 0.0;
    for (int q = lo; q < hi; ++q) acc = fma(a.data[i * a.rs + q * a.cs],
                                            b.data[q * b.rs + j * b.cs], acc);
    const double r = p.alpha * acc;
    if (pc != 0 || p.beta == 1.0) {
      if (pc == 0) cv = p.c[i + j * p.ldc];
      cv = r + cv;
    } else if (p.beta == 0.0) {
      cv = r;
    } else {
      const double cin = p.c[i + j * p.ldc];
      if (crossing) {
        const double bc = p.beta * cin;
        cv = r + bc;
      } else {
        cv = fma(cin, p.beta, r);
      }
    }
  }
  p.c[i + j * p.ldc] = cv;
}

// As DgemmDirectKernel for k > 256: each 256-wide chunk's FMA chain is
// independent, so tpe threads (a power of two >= the chunk count) compute
// one element's chunks in parallel and the first of them merges the chunk
// sums in order.
__global__ void __launch_bounds__(256)
    DgemmDirectChunkKernel(GemmParams p, View<double> a, View<double> b, int tpe) {
  if (p.guard != nullptr && *p.guard != 0) return;
  __shared__ double part[256];
  const int epb = 256 / tpe;
  const int e = threadIdx.x / tpe, ch = threadIdx.x % tpe;
  const long long elem = static_cast<long long>(blockIdx.x) * epb + e;
  const int i = static_cast<int>(elem % p.m), j = static_cast<int>(elem / p.m);
  const int nc = (p.k + 255) / 256;
  const bool valid = elem < static_cast<long long>(p.m) * p.n;
  int kb = 0, ke = p.k;
  if (valid && p.tri != kTriNone) TriRange(p, i, j, &kb, &ke);
  double acc = 0.0;
  if (valid && ch < nc) {
    const int hi = min(min(p.k, ch * 256 + 256), ke);
    for (int q = max(ch * 256, kb); q < hi; ++q)
      acc = fma(a.data[i * a.rs + q * a.cs], b.data[q * b.rs + j * b.cs], acc);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  if (!valid || ch != 0 || !InPart(p, i, j)) return;
  const bool crossing = p.part != kAll && InCrossingTile(p.part, p.m, p.n, i, j);
  double cv = 0.0;
  for (int c = 0; c < nc; ++c) {
    // A chunk outside the element's k range: the reference skips the tile.
    if (c != 0 && max(c * 256, kb) >= min(min(p.k, c * 256 + 256), ke)) continue;
    const double r = p.alpha * part[threadIdx.x + c];
    if (c != 0 || p.beta == 1.0) {
      if (c == 0) cv = p.c[i + j * p.ldc];
      cv = r + cv;
    } else if (p.beta == 0.0) {
      cv = r;
    } else {
      const double cin = p.c[i + j * p.ldc];
      if (crossing) {
        const double bc = p.beta * cin;
        cv = r + bc;
      } else {
        cv = fma(cin, p.beta, r);
      }
    }
  }
  p.c[i + j * p.ldc] = cv;
}

// Copies op(X) (rows x cols, strided view) into a dense column-major buffer
// with leading dimension ld, through a 32 x 32 shared tile so that both the
// read (along X's contiguous dimension) and the write are coalesced.
template <typename T>
__global__ void CanonicalCopyKernel(View<T> x, int rows, int cols, T* dst,
                                    long long ld) {
  __shared__ T tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  const bool trans = x.rs != 1;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    // Untransposed: threadIdx.x runs along i (contiguous); else along j.
    const int i = trans ? i0 + r : i0 + threadIdx.x;
    const int j = trans ? j0 + threadIdx.x : j0 + r;
    if (i < rows && j < cols) {
      const T v = x.data[i * x.rs + j * x.cs];
      if (trans) tile[threadIdx.x][r] = v; else tile[r][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + r;
    if (i < rows && j < cols) dst[i + j * ld] = tile[r][threadIdx.x];
  }
}

template <typename T>
__global__ void ScaleKernel(int m, int n, T beta, T* c, long long ldc,
                            int part, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  const long long total = static_cast<long long>(m) * n;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) +
                       threadIdx.x;
       idx < total; idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(idx % m), j = static_cast<int>(idx / m);
    if (part == kLower && i < j) continue;
    if (part == kUpper && i > j) continue;
    T* cij = c + i + j * ldc;
    *cij = (beta == T(0)) ? T(0) : *cij * beta;
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                                   void*, const cuuint64_t*, const cuuint64_t*,
                                   const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);
EncodeTiledFn Encoder() {
  static EncodeTiledFn fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr,
                                cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      fprintf(stderr, "hwyblas_b200: cuTensorMapEncodeTiled unavailable\n");
      return static_cast<EncodeTiledFn>(nullptr);
    }
    return reinterpret_cast<EncodeTiledFn>(ptr);
  }();
  return fn;
}

}  // namespace

// 2-D tensor map over a column-major matrix (inner dimension `rows`).
bool MakeTensorMap2d(CUtensorMap* map, CUtensorMapDataType dtype, int elem,
                     const void* base, long long rows, long long cols,
                     long long ld, int box_rows, int box_cols,
                     CUtensorMapSwizzle swizzle) {
  const EncodeTiledFn enc = Encoder();
  if (enc == nullptr) return false;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(rows),
                              static_cast<cuuint64_t>(cols)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * elem)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_rows),
                             static_cast<cuuint32_t>(box_cols)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      enc(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    fprintf(stderr, "hwyblas_b200: cuTensorMapEncodeTiled failed (%d)\n",
            static_cast<int>(r));
    return false;
  }
  return true;
}

// Whether a column-major operand can be read by TMA in place: 16-byte
// aligned base and leading dimension.
static bool TmaReady(const void* p, long long ld, int elem) {
  return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && ((ld * elem) % 16 == 0);
}

template <typename T>
const T* Canonical(View<T> x, int rows, int cols, int slot, long long* ld_out) {
  if (!x.trans() && TmaReady(x.data, x.ld(), sizeof(T))) {
    *ld_out = x.ld();
    return x.data;
  }
  const long long ld = (rows + 15) / 16 * 16;
  T* dst = static_cast<T*>(Workspace(slot, sizeof(T) * ld * cols));
  const dim3 grid((rows + 31) / 32, (cols + 31) / 32);
  CanonicalCopyKernel<T><<<grid, dim3(32, 8), 0, Ctx().stream>>>(x, rows, cols,
                                                                  dst, ld);
  CountLaunch();
  LaunchFailed("canonical copy");
  *ld_out = ld;
  return dst;
}
template const double* Canonical(View<double>, int, int, int, long long*);
template const float* Canonical(View<float>, int, int, int, long long*);

// Bytes of the per-chunk partial sums a DMMA GEMM of m x n x k takes when it
// splits over its KC chunks (few tiles, a long k), 0 when it runs unsplit.
size_t DgemmSplitBytes(int m, int n, int k) {
  const long long tiles =
      static_cast<long long>((m + kBM - 1) / kBM) * ((n + kBN - 1) / kBN);
  const int nchunks = (k + 255) / 256;
  const size_t pbytes = sizeof(double) * static_cast<size_t>(nchunks) * m * n;
  return (nchunks >= 2 && tiles * 2 <= Ctx().num_sms && pbytes <= (size_t(1) << 31)) ? pbytes
                                                                                     : 0;
}

void Dgemm(int m, int n, int k, double alpha, View<double> a, View<double> b,
           double beta, double* c, int ldc, Part part, Tri tri) {
  Context& ctx = Ctx();
  if (static_cast<long long>(m) * n * k <= (1LL << 22) || m < 32 || n < 32) {
    GemmParams p;
    p.m = m;
    p.n = n;
    p.k = k;
    p.alpha = alpha;
    p.beta = beta;
    p.c = c;
    p.ldc = ldc;
    p.part = part;
    p.tri = tri;
    p.timeout_flag = ctx.dev_status;
    p.guard = ctx.guard;
    const int nc = (k + 255) / 256;
    if (nc == 1) {
      const dim3 grid((m + 31) / 32, (n + 7) / 8);
      DgemmDirectKernel<<<grid, 256, 0, ctx.stream>>>(p, a, b);
      CountLaunch();
      LaunchFailed("dgemm direct");
      return;
    }
    if (nc <= 256) {
      int tpe = 1;
      while (tpe < nc) tpe *= 2;
      const long long elems = static_cast<long long>(m) * n;
      const long long blocks = (elems + (256 / tpe) - 1) / (256 / tpe);
      DgemmDirectChunkKernel<<<static_cast<unsigned>(blocks), 256, 0, ctx.stream>>>(
          p, a, b, tpe);
      CountLaunch();
      LaunchFailed("dgemm direct chunks");
      return;
    }
  }
  if (k <= kSkK && tri == kTriNone && TmaReady(a.data, a.ld(), 8) &&
      TmaReady(b.data, b.ld(), 8) && TmaReady(c, ldc, 8)) {
    static bool sk_configured = false;
    if (!sk_configured) {
      const auto set = [](const void* f) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSkSmemBytes);
      };
      set(reinterpret_cast<const void*>(DgemmShortKKernel<false, false, false>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<false, true, false>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<true, false, false>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<true, true, false>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<false, false, true>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<false, true, true>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<true, false, true>));
      set(reinterpret_cast<const void*>(DgemmShortKKernel<true, true, true>));
      sk_configured = true;
    }
    GemmParams p;
    p.m = m;
    p.n = n;
    p.k = k;
    p.alpha = alpha;
    p.beta = beta;
    p.c = c;
    p.ldc = ldc;
    p.part = part;
    p.tri = tri;
    p.partial = nullptr;
    p.nchunks = 1;
    p.timeout_flag = ctx.dev_status;
    p.guard = ctx.guard;
    const long long tiles =
        static_cast<long long>((m + kSkM - 1) / kSkM) * ((n + kSkN - 1) / kSkN);
    const int sms = ctx.sm_cap > 0 ? std::min(ctx.sm_cap, ctx.num_sms) : ctx.num_sms;
    const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, kSkPerSm * sms));
    cudaEvent_t t0 = KernelTimerStart(kFamilyDmmaGemm, ctx.stream);
    const auto launch = [&](auto kernel) {
      kernel<<<grid, kSkThreads, kSkSmemBytes, ctx.stream>>>(p, a.data, a.ld(), b.data, b.ld());
    };
    const bool ta = a.trans(), tb = b.trans();
    if (part == kAll) {
      if (!ta && !tb) launch(DgemmShortKKernel<false, false, false>);
      else if (!ta) launch(DgemmShortKKernel<false, true, false>);
      else if (!tb) launch(DgemmShortKKernel<true, false, false>);
      else launch(DgemmShortKKernel<true, true, false>);
    } else {
      if (!ta && !tb) launch(DgemmShortKKernel<false, false, true>);
      else if (!ta) launch(DgemmShortKKernel<false, true, true>);
      else if (!tb) launch(DgemmShortKKernel<true, false, true>);
      else launch(DgemmShortKKernel<true, true, true>);
    }
    KernelTimerStop(t0, ctx.stream);
    CountLaunch();
    LaunchFailed("dgemm short k");
    return;
  }
  long long lda, ldb;
  const double* ca = Canonical(a, m, k, kWsPackA, &lda);
  const double* cb = Canonical(b, k, n, kWsPackB, &ldb);
  CUtensorMap ma, mb;
  if (!MakeTensorMap2d(&ma, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, ca, m, k, lda,
                       16, kBK, CU_TENSOR_MAP_SWIZZLE_128B) ||
      !MakeTensorMap2d(&mb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, cb, k, n, ldb,
                       kBK, kBN, CU_TENSOR_MAP_SWIZZLE_128B)) {
    Failed(cudaErrorInvalidValue, "dgemm tensor map");
    return;
  }
  GemmParams p;
  p.m = m;
  p.n = n;
  p.k = k;
  p.alpha = alpha;
  p.beta = beta;
  p.c = c;
  p.ldc = ldc;
  p.part = part;
  p.tri = tri;
  p.partial = nullptr;
  p.nchunks = 1;
  p.timeout_flag = ctx.dev_status;
  p.guard = ctx.guard;
  const long long tiles =
      static_cast<long long>((m + kBM - 1) / kBM) * ((n + kBN - 1) / kBN);
  static bool configured = false;
  if (!configured) {
    const auto set = [](const void* f) {
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    };
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<0, false>));
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<1, false>));
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<2, false>));
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<0, true>));
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<1, true>));
    set(reinterpret_cast<const void*>(DgemmDmmaKernel<2, true>));
    configured = true;
  }
  const int tri_kind =
      tri == kTriNone ? 0 : (tri == kTriALower || tri == kTriAUpper) ? 1 : 2;
  // Few tiles and a long k (a narrow product: TRTRI's and GETRI's block
  // columns): each tile's KC chunks become separate work items, so that the
  // chunks of one tile run on different SMs, and a second kernel merges them
  // in order. Every chain and merge is the unsplit kernel's.
  const int nchunks = (k + 255) / 256;
  const size_t pbytes = DgemmSplitBytes(m, n, k);
  if (pbytes > 0) {
    double* partial = static_cast<double*>(Workspace(kWsSplitK, pbytes));
    if (partial != nullptr) {
      p.partial = partial;
      p.nchunks = nchunks;
      const int sms = ctx.sm_cap > 0 ? std::min(ctx.sm_cap, ctx.num_sms) : ctx.num_sms;
      const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles * nchunks, sms));
      cudaEvent_t t0 = KernelTimerStart(kFamilyDmmaGemm, ctx.stream);
      if (tri_kind == 0) {
        DgemmDmmaKernel<0, true><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
      } else if (tri_kind == 1) {
        DgemmDmmaKernel<1, true><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
      } else {
        DgemmDmmaKernel<2, true><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
      }
      KernelTimerStop(t0, ctx.stream);
      const long long total = static_cast<long long>(m) * n;
      const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 16));
      DgemmSplitMergeKernel<<<blocks, 256, 0, ctx.stream>>>(p);
      CountLaunch(2);
      LaunchFailed("dgemm split");
      return;
    }
  }
  // Persistent grid: one CTA per SM (the accumulators and the prefetched C
  // take 128 of each thread's registers). Measured against a variant whose
  // producer is lane 0 of warp 0 (8 warps): dgemm n = 8192 32.9 vs 27.5
  // TFLOP/s, getrf n = 16384 418 vs 440 ms.
  const int sms = ctx.sm_cap > 0 ? std::min(ctx.sm_cap, ctx.num_sms) : ctx.num_sms;
  const unsigned grid = static_cast<unsigned>(std::min<long long>(tiles, sms));
  cudaEvent_t t0 = KernelTimerStart(kFamilyDmmaGemm, ctx.stream);
  if (tri_kind == 0) {
    DgemmDmmaKernel<0, false><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
  } else if (tri_kind == 1) {
    DgemmDmmaKernel<1, false><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
  } else {
    DgemmDmmaKernel<2, false><<<grid, kThreads, kSmemBytes, ctx.stream>>>(ma, mb, p);
  }
  KernelTimerStop(t0, ctx.stream);
  CountLaunch();
  LaunchFailed("dgemm");
}

template <typename T>
void ScaleMatrix(int m, int n, T beta, T* c, int ldc, Part part) {
  if (m <= 0 || n <= 0) return;
  const long long total = static_cast<long long>(m) * n;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 8));
  ScaleKernel<T><<<blocks, 256, 0, Ctx().stream>>>(m, n, beta, c, ldc, part,
                                                   Ctx().guard);
  CountLaunch();
  LaunchFailed("scale");
}
template void ScaleMatrix<double>(int, int, double, double*, int, Part);
template void ScaleMatrix<float>(int, int, float, float*, int, Part);

}  // namespace hb
