// Pivot search, row interchanges and the leaf factorizations of the LU and
// Cholesky drivers, with the reference's exact operation order:
//   IAMAX      src/level1.cc:383-402, src/level1-inl.h:343-423
//   LASWP      src/lapack/getrf.cc:28-81
//   GetrfLeaf  src/lapack/factor_kernels.cc:79-183
//   PotrfLeaf  src/lapack/factor_kernels.cc:187-221
// "lanes" is the vector length (in elements) of the reference's SIMD target:
// AXPY columns shorter than one vector are updated as y + (alpha*x) (two
// roundings), longer ones as fma(x, alpha, y) (factor_kernels.cc:79-118).
#include <cooperative_groups.h>

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstdlib>

#include <mutex>

#include "../../include/hwyblas_b200.h"
#include "device.cuh"
#include "internal.h"
#include "ref_order.cuh"

namespace hb {

int RefLanesDouble() {
  static int lanes = [] {
    const char* e = getenv("HWYBLAS_REF_LANES");
    const int v = e ? atoi(e) : 8;
    return v == 4 ? 4 : 8;
  }();
  return lanes;
}

namespace {

// ---------------------------------------------------------------------------
// IAMAX: per-block candidates, then the last block to finish reduces them.
template <typename T>
__global__ void IamaxKernel(int n, const T* x, long long incx, T* part_v,
                            int* part_i, unsigned int* ticket, int* out) {
  T bv = T(-1);
  int bi = 0x7fffffff;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
       i < n; i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const T v = fabs(x[i * incx]);
    if (v > bv) {  // strict: NaN never wins; each thread visits i ascending
      bv = v;
      bi = static_cast<int>(i);
    }
  }
  __shared__ T sv[32];
  __shared__ int si[32];
  for (int off = 16; off > 0; off >>= 1) {
    const T ov = __shfl_down_sync(0xffffffffu, bv, off);
    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
    if (Better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
  }
  if (threadIdx.x % 32 == 0) { sv[threadIdx.x / 32] = bv; si[threadIdx.x / 32] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x / 32); ++w)
      if (Better(sv[w], si[w], bv, bi)) { bv = sv[w]; bi = si[w]; }
    part_v[blockIdx.x] = bv;
    part_i[blockIdx.x] = bi;
    __threadfence();
    const unsigned int done = atomicAdd(ticket, 1u);
    if (done == gridDim.x - 1) {
      __threadfence();
      T gv = T(-1);
      int gi = 0x7fffffff;
      for (unsigned int b = 0; b < gridDim.x; ++b) {
        const T v = *(volatile T*)&part_v[b];
        const int i = *(volatile int*)&part_i[b];
        if (Better(v, i, gv, gi)) { gv = v; gi = i; }
      }
      // The reference returns index 0 when x[0] is NaN (and x[0] is the
      // first candidate otherwise).
      if (isnan(fabs(x[0])) || gi == 0x7fffffff) gi = 0;
      *out = gi + 1;
      *ticket = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// LASWP: one thread per column applies the interchanges in order.
template <typename T>
__global__ void LaswpKernel(int n, T* a, long long lda, int i1, int i2,
                            int inc, int ix0, int incx, const int* ipiv,
                            const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  T* ac = a + col * lda;
  int ix = ix0;
  for (int i = i1; inc > 0 ? i <= i2 : i >= i2; i += inc) {
    const int ip = ipiv[ix - 1];
    if (ip != i) {
      const T t = ac[i - 1];
      ac[i - 1] = ac[ip - 1];
      ac[ip - 1] = t;
    }
    ix += incx;
  }
}

// LASWP for incx = 1 and at most kSwapMax interchanges: the interchanges
// only move data among the rows k1..k2 and their partners, so their net
// effect is one permutation of at most 2 kSwapMax rows. Thread 0 of every
// block replays the interchanges on a table of (row, row whose data it holds)
// in shared memory - rows k1..k2 at fixed slots, partners outside found
// through a small hash - and then each warp permutes whole columns: its lanes
// read the table's source rows of a column into registers and write them to
// the destination rows (the values moved, and so the result, are the same).
constexpr int kSwapMax = 512;
constexpr int kSwapTable = 2 * kSwapMax;
constexpr int kSwapHash = 2048;  // power of two, > kSwapMax
constexpr int kLaswpCols = 64;   // columns per block
template <typename T>
__global__ void __launch_bounds__(256)
    LaswpPermKernel(int n, T* a, long long lda, int k1, int k2,
                    const int* ipiv, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ int pos[kSwapTable], src[kSwapTable];
  __shared__ int hkey[kSwapHash], hfirst[kSwapHash], spiv[kSwapMax], sslot[kSwapMax];
  __shared__ int wsum[8];
  __shared__ int cnt;
  const int nb = k2 - k1 + 1;
  for (int t = threadIdx.x; t < kSwapHash; t += blockDim.x) {
    hkey[t] = -1;
    hfirst[t] = 0x7fffffff;
  }
  __syncthreads();
  // (1) Partners outside k1..k2 enter a hash (row -> first swap that names
  // it); rows inside have fixed slots.
  const int t0 = threadIdx.x;  // nb <= kSwapMax = 2 * blockDim.x: two swaps a thread
  for (int t = t0; t < nb; t += blockDim.x) {
    const int p = ipiv[k1 - 1 + t];
    spiv[t] = p;
    pos[t] = k1 + t;
    src[t] = k1 + t;
    if (p != k1 + t && (p < k1 || p > k2)) {
      int hh = static_cast<int>((static_cast<unsigned>(p) * 40503u) & (kSwapHash - 1));
      while (true) {
        const int prev = atomicCAS(&hkey[hh], -1, p);
        if (prev == -1 || prev == p) break;
        hh = (hh + 1) & (kSwapHash - 1);
      }
      atomicMin(&hfirst[hh], t);
    }
  }
  __syncthreads();
  // (2) The first swap naming each outside row gets the next extra slot, in
  // swap order: a block-wide prefix count of the first occurrences.
  int flag[2] = {0, 0}, hs[2] = {-1, -1};
  for (int r = 0; r < 2; ++r) {
    const int t = t0 + r * blockDim.x;
    if (t >= nb) continue;
    const int pp = spiv[t];
    if (pp == k1 + t || (pp >= k1 && pp <= k2)) continue;
    int hh = static_cast<int>((static_cast<unsigned>(pp) * 40503u) & (kSwapHash - 1));
    while (hkey[hh] != pp) hh = (hh + 1) & (kSwapHash - 1);
    hs[r] = hh;
    flag[r] = hfirst[hh] == t ? 1 : 0;
  }
  // Exclusive scan over t = 0..nb-1 of flag (t = t0 + r*blockDim.x).
  int base = 0;
  for (int r = 0; r < 2; ++r) {
    int v = flag[r];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    int incl = v;
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += o;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) {
      if (w < warp) before += wsum[w];
      total += wsum[w];
    }
    __syncthreads();
    const int t = t0 + r * blockDim.x;
    if (flag[r]) {
      const int slot = nb + base + before + incl - v;
      pos[slot] = spiv[t];
      src[slot] = spiv[t];
      hfirst[hs[r]] = -(slot + 1);  // from now on: the row's slot
    }
    base += total;
  }
  __syncthreads();
  for (int r = 0; r < 2; ++r) {
    const int t = t0 + r * blockDim.x;
    if (t >= nb) continue;
    const int pp = spiv[t];
    sslot[t] = (pp >= k1 && pp <= k2) ? pp - k1 : (hs[r] >= 0 ? -hfirst[hs[r]] - 1 : t);
  }
  if (threadIdx.x == 0) cnt = nb + base;
  // Factorizations' pivots name rows at or below their own (slot >= step);
  // dlaswp callers may pass any.
  int ordered = 1;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int t = t0 + r * blockDim.x;
    if (t < nb && sslot[t] < t) ordered = 0;
  }
  if (!__syncthreads_and(ordered)) {
    // (3) The interchanges in order, on the source table.
    if (threadIdx.x == 0) {
      for (int t = 0; t < nb; ++t) {
        const int sp = sslot[t];
        if (sp == t) continue;
        const int a0 = src[t];
        src[t] = src[sp];
        src[sp] = a0;
      }
    }
  } else {
  // (3) The interchanges' net effect, without replaying them one by one.
  // Interchange u swaps slots u and s_u = sslot[u] (s_u >= u). Slot u's
  // content just before step u is that before step into(u), the last earlier
  // step whose s_v is u, or its own row if none; after step u, slot u holds
  // what s_u held, i.e. the content before step prev(u), the last earlier
  // step with the same s_v, or s_u's own row; an extra slot ends with the
  // content before the last step naming it. The "content before" chains
  // point to earlier steps and resolve by pointer jumping.
  {
    int into[2] = {-1, -1}, prev[2] = {-1, -1}, later[2] = {0, 0}, su[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) su[r] = t0 + r * blockDim.x < nb ? sslot[t0 + r * blockDim.x] : -1;
    for (int v = 0; v < nb; ++v) {
      const int sv = sslot[v];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int u = t0 + r * blockDim.x;
        if (v < u) {
          if (sv == u) into[r] = v;
          if (sv == su[r]) prev[r] = v;
        } else if (v > u && sv == su[r]) {
          later[r] = 1;
        }
      }
    }
    int* ptr = hkey;    // the hash is no longer needed: [2][kSwapMax] each
    int* val = hfirst;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int u = t0 + r * blockDim.x;
      if (u < nb) {
        ptr[u] = into[r];
        val[u] = pos[u];
      }
    }
    __syncthreads();
    for (int round = 0, cur = 0; round < 11; ++round, cur ^= 1) {
      const int* pc = ptr + cur * kSwapMax;
      const int* vc = val + cur * kSwapMax;
      int* pn = ptr + (cur ^ 1) * kSwapMax;
      int* vn = val + (cur ^ 1) * kSwapMax;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int u = t0 + r * blockDim.x;
        if (u >= nb) continue;
        const int q = pc[u];
        if (q >= 0 && pc[q] < 0) {
          pn[u] = -1;
          vn[u] = vc[q];
        } else {
          pn[u] = q >= 0 ? pc[q] : -1;
          vn[u] = vc[u];
        }
      }
      __syncthreads();
    }
    const int* vf = val + (11 & 1) * kSwapMax;  // after 11 rounds: buffer 1
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int u = t0 + r * blockDim.x;
      if (u >= nb) continue;
      src[u] = prev[r] >= 0 ? vf[prev[r]] : pos[su[r]];
      if (su[r] >= nb && !later[r]) src[su[r]] = vf[u];
    }
  }
  }
  __syncthreads();
  const int c = cnt;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int col_end = min(n, (blockIdx.x + 1) * kLaswpCols);
  for (int col = blockIdx.x * kLaswpCols + warp; col < col_end; col += blockDim.x / 32) {
    T* ac = a + static_cast<long long>(col) * lda;
    T v[kSwapTable / 32];
#pragma unroll
    for (int r = 0; r < kSwapTable / 32; ++r) {
      const int e = lane + 32 * r;
      if (e < c) v[r] = ac[src[e] - 1];
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kSwapTable / 32; ++r) {
      const int e = lane + 32 * r;
      if (e < c) ac[pos[e] - 1] = v[r];
    }
    __syncwarp();
  }
}

__global__ void AdjustPivotsKernel(int* ipiv, int begin, int end, int delta) {
  const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < end) ipiv[i] += delta;
}

// ---------------------------------------------------------------------------
// LU leaf, pivot columns: the m x w panel (w <= 16) is split by rows over P
// co-resident CTAs (cooperative launch), each holding its rows in shared
// memory. Per column j: every CTA publishes its best candidate (|a|, row,
// row contents), one grid barrier, then every CTA picks the same pivot and
// applies the swap, the scaling and the rank-1 update to its own rows.
constexpr int kLeafThreads = 512;
constexpr int kLeafMaxRows = 1024;  // rows per CTA
constexpr int kLeafMaxP = 64;       // CTAs per panel (m <= 65536)
constexpr int kLeafMaxCluster = 16; // CTAs of the cluster variant (m <= 16384)
// On the look-ahead stream, beside the capped trailing GEMM, a cluster of at
// most this many CTAs still finds its SMs in one GPC; larger panels take
// the cooperative variant.
constexpr int kLeafSideCluster = 8;
constexpr int kLeafW = 16;

// Polls of the cooperative leaf's candidate exchange before a CTA gives up
// (sets the timeout flag and returns). hwyblas_set_leaf_wait_limit lowers it
// so that a test can make the wait run out; 0 there restores this default.
__device__ uint32_t g_leaf_poll_limit = kMaxPolls;

template <typename T>
struct LeafArgs {
  int m, w, lanes;
  T* a;
  long long lda;
  int* ipiv;
  int* info;
  int info_base;
  T* xchg;                // [2][P][2 kLeafW + 2] candidate slots
  unsigned int* tags;     // [2][P] slot tags, zeroed before launch
  int* timeout_flag;
};

// kCluster: the P CTAs form one thread-block cluster and exchange their
// candidates through distributed shared memory (each publishes into its own
// shared slot, one cluster barrier, then every CTA reads the P slots), which
// replaces the global-memory slots and polling of the cooperative variant.
template <typename T, bool kCluster, int W>
__global__ void __launch_bounds__(kLeafThreads)
    GetrfLeafPanelKernel(LeafArgs<T> p) {
  extern __shared__ __align__(16) uint8_t leaf_smem[];
  T* sp = reinterpret_cast<T*>(leaf_smem);  // column-major [w][R]
  __shared__ T s_piv[W], s_rowj[W];
  __shared__ T s_cand[(kCluster ? kLeafMaxCluster : kLeafMaxP) * (2 * W + 2)];
  __shared__ T s_slot[2 * (2 * W + 2)];  // kCluster: own slot per parity
  __shared__ T s_wv[kLeafThreads / 32];
  __shared__ int s_wi[kLeafThreads / 32];
  __shared__ int s_p, s_abort;
  const int P = gridDim.x, cta = blockIdx.x;
  const int rows_per = (p.m + P - 1) / P;
  const int r0 = cta * rows_per, r1 = min(p.m, r0 + rows_per);
  const int R = rows_per;
  const int w = p.w;
  const int slot_len = 2 * W + 2;
  T* cand = p.xchg;  // [2][P][slot_len]
  unsigned int* tags = p.tags;

  if (threadIdx.x == 0) s_abort = 0;
  for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
    // All of a row's loads in flight before its shared-memory stores.
    T v[W];
#pragma unroll
    for (int c = 0; c < W; ++c)
      if (c < w) v[c] = p.a[(r0 + lr) + c * p.lda];
#pragma unroll
    for (int c = 0; c < W; ++c)
      if (c < w) sp[c * R + lr] = v[c];
  }
  // kCluster: every CTA of the cluster is running before any remote access.
  if constexpr (kCluster) cooperative_groups::this_cluster().sync();
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // (a) local candidate over rows >= j.
    T bv = T(-1);
    int bi = 0x7fffffff;
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
      const int gi = r0 + lr;
      if (gi < j) continue;
      const T v = fabs(sp[j * R + lr]);
      if (v > bv) { bv = v; bi = gi; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const T ov = __shfl_down_sync(0xffffffffu, bv, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (Better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    if (threadIdx.x % 32 == 0) { s_wv[threadIdx.x / 32] = bv; s_wi[threadIdx.x / 32] = bi; }
    __syncthreads();
    if (threadIdx.x < 32) {
      // The order of the reduction is immaterial: Better is a total order.
      bv = threadIdx.x < kLeafThreads / 32 ? s_wv[threadIdx.x] : T(-1);
      bi = threadIdx.x < kLeafThreads / 32 ? s_wi[threadIdx.x] : 0x7fffffff;
      for (int off = 16; off > 0; off >>= 1) {
        const T ov = __shfl_down_sync(0xffffffffu, bv, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (Better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
      }
      __syncwarp();
      if (threadIdx.x == 0) {
        s_p = bi;
        s_wv[0] = bv;
      }
    }
    __syncthreads();
    // (b) exchange the candidates. A CTA holding the whole panel keeps them in
    // shared memory. Otherwise every CTA writes its slot for this step's
    // parity (|a|, row, row contents, and row j if it owns it), fences and
    // release-stores the step number as the slot's tag; each CTA polls the P
    // tags (one thread per slot, bounded) and copies all slots in one parallel
    // round trip. A CTA can only overwrite a parity after every CTA has
    // published the next step, i.e. after all have read this one.
    const int ci = s_p;
    if (kCluster && P > 1) {
      // Publish into the own slot of this parity; after the cluster barrier
      // every CTA copies the P slots. A slot parity is rewritten two columns
      // later, after the next barrier, when every CTA has read it.
      cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
      T* mine = s_slot + par * slot_len;
      if (threadIdx.x == 0) {
        mine[0] = s_wv[0];
        mine[1] = static_cast<T>(ci == 0x7fffffff ? -1 : ci);
      }
      if (threadIdx.x < w) {
        mine[2 + threadIdx.x] =
            (ci != 0x7fffffff) ? sp[threadIdx.x * R + (ci - r0)] : T(0);
        if (j >= r0 && j < r1)
          mine[2 + W + threadIdx.x] = sp[threadIdx.x * R + (j - r0)];
      }
      cluster.sync();
      for (int idx = threadIdx.x; idx < P * slot_len; idx += blockDim.x) {
        const int q = idx / slot_len, e = idx - q * slot_len;
        const T* peer = cluster.map_shared_rank(s_slot, q);
        s_cand[idx] = peer[par * slot_len + e];
      }
      __syncthreads();
      if (threadIdx.x < w)
        s_rowj[threadIdx.x] = s_cand[(j / rows_per) * slot_len + 2 + W + threadIdx.x];
    } else if (P == 1) {
      if (threadIdx.x == 0) {
        s_cand[0] = s_wv[0];
        s_cand[1] = static_cast<T>(ci == 0x7fffffff ? -1 : ci);
      }
      if (threadIdx.x < w) {
        s_cand[2 + threadIdx.x] =
            (ci != 0x7fffffff) ? sp[threadIdx.x * R + ci] : T(0);
        s_rowj[threadIdx.x] = sp[threadIdx.x * R + j];
      }
      __syncthreads();
    } else {
      T* slot = cand + (par * P + cta) * slot_len;
      if (threadIdx.x == 0) {
        slot[0] = s_wv[0];
        slot[1] = static_cast<T>(ci == 0x7fffffff ? -1 : ci);
      }
      if (threadIdx.x < w) {
        slot[2 + threadIdx.x] =
            (ci != 0x7fffffff) ? sp[threadIdx.x * R + (ci - r0)] : T(0);
        if (j >= r0 && j < r1)
          slot[2 + W + threadIdx.x] = sp[threadIdx.x * R + (j - r0)];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(tags + par * P + cta),
                     "r"(static_cast<unsigned>(j + 1))
                     : "memory");
      }
      if (threadIdx.x < P) {
        uint32_t polls = 0;
        while (true) {
          unsigned v;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                       : "=r"(v)
                       : "l"(tags + par * P + threadIdx.x)
                       : "memory");
          if (v >= static_cast<unsigned>(j + 1)) break;
          if (++polls >= g_leaf_poll_limit) {
            atomicExch(p.timeout_flag, 1);
            s_abort = 1;
            break;
          }
        }
      }
      __syncthreads();
      if (s_abort) return;
      for (int idx = threadIdx.x; idx < P * slot_len; idx += blockDim.x)
        s_cand[idx] = *(volatile const T*)&cand[par * P * slot_len + idx];
      __syncthreads();
      if (threadIdx.x < w)
        s_rowj[threadIdx.x] = s_cand[(j / rows_per) * slot_len + 2 + W + threadIdx.x];
    }
    // (c) the global pivot: the reference's IAMAX over rows j..m-1; warp 0
    // picks the winner among the candidates and fills the pivot row.
    if (threadIdx.x < 32) {
      __syncwarp();  // s_rowj was written by lanes of this warp
      T gv = T(-1);
      int gi = 0x7fffffff;
      int wq = -1;
      for (int q = threadIdx.x; q < P; q += 32) {
        const T fi = s_cand[q * slot_len + 1];
        if (fi < T(0)) continue;
        const T v = s_cand[q * slot_len];
        const int i = static_cast<int>(fi);
        if (Better(v, i, gv, gi)) { gv = v; gi = i; wq = q; }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const T ov = __shfl_down_sync(0xffffffffu, gv, off);
        const int oi = __shfl_down_sync(0xffffffffu, gi, off);
        const int oq = __shfl_down_sync(0xffffffffu, wq, off);
        if (Better(ov, oi, gv, gi)) { gv = ov; gi = oi; wq = oq; }
      }
      gi = __shfl_sync(0xffffffffu, gi, 0);
      wq = __shfl_sync(0xffffffffu, wq, 0);
      const T ajj = s_rowj[j];
      if (isnan(fabs(ajj)) || gi == 0x7fffffff) gi = j;
      if (threadIdx.x == 0) s_p = gi;
      // The winner's slot holds row gi (row j's own values if gi == j).
      if (threadIdx.x < w)
        s_piv[threadIdx.x] = (gi == j) ? s_rowj[threadIdx.x]
                                       : s_cand[wq * slot_len + 2 + threadIdx.x];
    }
    __syncthreads();
    const int piv = s_p;
    const T pivot = s_piv[j];
    if (cta == 0 && threadIdx.x == 0) {
      p.ipiv[j] = piv + 1;
      if (pivot == T(0) && *p.info == 0) *p.info = p.info_base + j + 1;
    }
    // (d) interchange rows j and piv across the leaf's columns.
    if (pivot != T(0) && piv != j && threadIdx.x < w) {
      if (piv >= r0 && piv < r1) sp[threadIdx.x * R + (piv - r0)] = s_rowj[threadIdx.x];
      if (j >= r0 && j < r1) sp[threadIdx.x * R + (j - r0)] = s_piv[threadIdx.x];
    }
    __syncthreads();
    // (e) column j below the diagonal: * (1/pivot), or / pivot if tiny (not
    // for a zero pivot); (f) rank-1 update of columns j+1..w-1 (AXPY with
    // alpha = -a(j, k)). A thread scales and updates its own rows, so the
    // next barrier is the next column's first one.
    const bool scale = pivot != T(0);
    const bool tiny = !(fabs(pivot) >= Sfmin<T>());
    const T rinv = T(1) / pivot;
    const int len = p.m - j - 1;
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x) {
      if (r0 + lr <= j) continue;
      T x = sp[j * R + lr];
      if (scale) {
        x = tiny ? x / pivot : x * rinv;
        sp[j * R + lr] = x;
      }
      for (int k = j + 1; k < w; ++k)
        sp[k * R + lr] = Axpy(sp[k * R + lr], -s_piv[k], x, len, p.lanes);
    }
  }
  __syncthreads();
  // kCluster: no CTA exits while a peer may still read its slot.
  if constexpr (kCluster) cooperative_groups::this_cluster().sync();
  for (int c = 0; c < w; ++c)
    for (int lr = threadIdx.x; lr < r1 - r0; lr += blockDim.x)
      p.a[(r0 + lr) + c * p.lda] = sp[c * R + lr];
}

// LU leaf, trailing columns (n > m, m <= 16). In the reference, step j swaps
// rows j and p_j of every column and then updates rows i > j of column k as
// x_i += (-x_j) * l_ij. Later swaps only exchange rows > j, in the L columns
// and in column k alike, so each multiplier stays on the row it updates: the
// same arithmetic is all swaps first, then the updates with the final L.
// Columns are independent: one thread per column.
template <typename T>
__global__ void GetrfLeafTrailingKernel(int m, int w, int n, T* a,
                                        long long lda, const int* ipiv,
                                        int lanes) {
  const int k = w + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  T* col = a + k * lda;
  for (int j = 0; j < w; ++j) {
    // A zero pivot has p == j (its column is all zeros), so no swap.
    const int p = ipiv[j] - 1;
    if (p != j) {
      const T t = col[j];
      col[j] = col[p];
      col[p] = t;
    }
  }
  for (int j = 0; j < w; ++j) {
    const T alpha = -col[j];
    const int len = m - j - 1;
    for (int i = j + 1; i < m; ++i) col[i] = Axpy(col[i], alpha, a[i + j * lda], len, lanes);
  }
}

// ---------------------------------------------------------------------------
// Cholesky leaf (n <= 64) in one CTA, the block in shared memory.
template <typename T>
__global__ void __launch_bounds__(256)
    PotrfLeafKernel(int upper, int n, T* a, long long lda, int* info,
                    int info_base, int lanes, const int* guard) {
  if (guard != nullptr && *guard != 0) return;
  __shared__ T s[64][65];  // s[i][j] = A(i, j)
  __shared__ T row[64];
  __shared__ int stop;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    const bool ref = upper ? (i <= j) : (i >= j);
    s[i][j] = ref ? a[i + j * lda] : T(0);
  }
  if (threadIdx.x == 0) stop = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x == 0) {
      const T ajj = s[j][j];
      if (ajj <= T(0) || isnan(ajj)) {
        stop = 1;
        if (*info == 0) *info = info_base + j + 1;
      } else {
        const T r = sqrt(ajj);
        s[j][j] = r;
        row[j] = T(1) / r;  // rinv
      }
    }
    __syncthreads();
    if (stop) break;
    const T rinv = row[j];
    __syncthreads();
    if (upper) {
      for (int k = j + 1 + threadIdx.x; k < n; k += blockDim.x) {
        s[j][k] = s[j][k] * rinv;
        row[k] = s[j][k];
      }
      __syncthreads();
      // Column k, rows j+1..k: y += (-U(j,k)) * row, length k - j.
      for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, k = idx / n;
        if (k <= j || i <= j || i > k) continue;
        s[i][k] = Axpy(s[i][k], -s[j][k], row[i], k - j, lanes);
      }
    } else {
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) s[i][j] = s[i][j] * rinv;
      __syncthreads();
      // Column k, rows k..n-1: y += (-L(k,j)) * L(k:n, j), length n - k.
      for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, k = idx / n;
        if (k <= j || i < k) continue;
        s[i][k] = Axpy(s[i][k], -s[k][j], s[i][j], n - k, lanes);
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int i = idx % n, j = idx / n;
    const bool ref = upper ? (i <= j) : (i >= j);
    if (ref) a[i + j * lda] = s[i][j];
  }
}

}  // namespace

template <typename T>
void Iamax(int n, const T* x, int incx, int* out) {
  Context& ctx = Ctx();
  const int blocks = static_cast<int>(std::min<long long>((n + 1023) / 1024, 296));
  T* pv = static_cast<T*>(Workspace(kWsLeaf, 296 * (sizeof(T) + sizeof(int))));
  int* pi = reinterpret_cast<int*>(pv + 296);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(ctx.dev_status + 8);
  IamaxKernel<T><<<std::max(blocks, 1), 1024, 0, ctx.stream>>>(n, x, incx, pv,
                                                                pi, ticket, out);
  CountLaunch();
  LaunchFailed("iamax");
}
template void Iamax<double>(int, const double*, int, int*);
template void Iamax<float>(int, const float*, int, int*);

template <typename T>
void Laswp(int n, T* a, int lda, int k1, int k2, const int* ipiv, int incx) {
  if (n <= 0 || incx == 0) return;
  int i1, i2, inc, ix0;
  if (incx > 0) {
    ix0 = k1; i1 = k1; i2 = k2; inc = 1;
  } else {
    ix0 = k1 + (k1 - k2) * incx; i1 = k2; i2 = k1; inc = -1;
  }
  if (inc > 0 ? i1 > i2 : i1 < i2) return;
  if (incx == 1) {
    // Consecutive runs of at most kSwapMax interchanges, in order: the same
    // sequence of interchanges as one pass over k1..k2.
    for (int c1 = k1; c1 <= k2; c1 += kSwapMax) {
      const int c2 = std::min(k2, c1 + kSwapMax - 1);
      LaswpPermKernel<T><<<(n + kLaswpCols - 1) / kLaswpCols, 256, 0, Ctx().stream>>>(
          n, a, lda, c1, c2, ipiv, Ctx().guard);
      CountLaunch();
    }
    LaunchFailed("laswp");
    return;
  }
  LaswpKernel<T><<<(n + 127) / 128, 128, 0, Ctx().stream>>>(
      n, a, lda, i1, i2, inc, ix0, incx, ipiv, Ctx().guard);
  CountLaunch();
  LaunchFailed("laswp");
}
template void Laswp<double>(int, double*, int, int, int, const int*, int);
template void Laswp<float>(int, float*, int, int, int, const int*, int);
template void Laswp<ZPair<double>>(int, ZPair<double>*, int, int, int, const int*, int);
template void Laswp<ZPair<float>>(int, ZPair<float>*, int, int, int, const int*, int);

void AdjustPivots(int* ipiv, int begin, int end, int delta) {
  if (end <= begin || delta == 0) return;
  AdjustPivotsKernel<<<(end - begin + 255) / 256, 256, 0, Ctx().stream>>>(
      ipiv, begin, end, delta);
  CountLaunch();
  LaunchFailed("adjust pivots");
}

// Rows per CTA of the 32-column leaf: its 32 columns and the static slots
// stay within the 227 KB of shared memory a CTA can have.
constexpr int kWideLeafRows = 832;

template <typename T>
void GetrfLeaf(int m, int n, T* a, int lda, int* ipiv, int* info, int info_base,
               int leaf_w) {
  Context& ctx = Ctx();
  const int w = std::min(m, n);
  const int lanes = sizeof(T) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  const bool wide = leaf_w == 32 && w > kLeafW;
  const int max_rows = wide ? kWideLeafRows : kLeafMaxRows;
  const int P = (m + max_rows - 1) / max_rows;
  const int R = (m + P - 1) / P;
  if (P > kLeafMaxP || (wide && P > kLeafMaxCluster)) {
    fprintf(stderr, "hwyblas_b200: LU panel of %d rows exceeds the leaf's limit\n", m);
    Failed(cudaErrorInvalidValue, "getrf leaf size");
    return;
  }
  const size_t smem = static_cast<size_t>(w) * R * sizeof(T);
  const int smem_max = kLeafW * kLeafMaxRows * static_cast<int>(sizeof(T));
  const int smem_wide = 32 * kWideLeafRows * static_cast<int>(sizeof(T));
  static int max_cluster = 0, max_cluster_wide = 0;
  static bool configured = false;
  auto cluster_limit = [](const void* fn, int smem_bytes) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kLeafMaxCluster);
    cfg.blockDim = dim3(kLeafThreads);
    cfg.dynamicSmemBytes = smem_bytes;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kLeafMaxCluster;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int size = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&size, fn, &cfg) != cudaSuccess) {
      cudaGetLastError();
      size = 0;
    }
    return std::min(size, kLeafMaxCluster);
  };
  if (!configured) {
    cudaFuncSetAttribute(GetrfLeafPanelKernel<T, false, kLeafW>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(GetrfLeafPanelKernel<T, true, kLeafW>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(GetrfLeafPanelKernel<T, true, kLeafW>,
                         cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(GetrfLeafPanelKernel<T, true, 32>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_wide);
    cudaFuncSetAttribute(GetrfLeafPanelKernel<T, true, 32>,
                         cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    max_cluster = cluster_limit(
        reinterpret_cast<const void*>(GetrfLeafPanelKernel<T, true, kLeafW>), smem_max);
    max_cluster_wide = cluster_limit(
        reinterpret_cast<const void*>(GetrfLeafPanelKernel<T, true, 32>), smem_wide);
    configured = true;
  }
  if (wide && P > max_cluster_wide) {
    Failed(cudaErrorInvalidValue, "getrf wide leaf cluster");
    return;
  }
  LeafArgs<T> args;
  args.m = m;
  args.w = w;
  args.lanes = lanes;
  args.a = a;
  args.lda = lda;
  args.ipiv = ipiv;
  args.info = info;
  args.info_base = info_base;
  const size_t slot_bytes = sizeof(T) * 2 * P * (2 * kLeafW + 2);
  args.xchg = static_cast<T*>(
      Workspace(kWsLeaf, slot_bytes + sizeof(unsigned int) * 2 * kLeafMaxP));
  args.tags = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(args.xchg) +
                                              slot_bytes);
  args.timeout_flag = ctx.dev_status;
  cudaEvent_t t0 = KernelTimerStart(kFamilyLuLeaf, ctx.stream);
  if (wide || (P > 1 && P <= max_cluster && (!ctx.side_leaf || P <= kLeafSideCluster))) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P);
    cfg.blockDim = dim3(kLeafThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx.stream;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = P;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    if (wide) {
      Failed(cudaLaunchKernelEx(&cfg, GetrfLeafPanelKernel<T, true, 32>, args),
             "getrf wide leaf (cluster)");
    } else {
      Failed(cudaLaunchKernelEx(&cfg, GetrfLeafPanelKernel<T, true, kLeafW>, args),
             "getrf leaf (cluster)");
    }
  } else if (P > 1) {
    cudaMemsetAsync(args.tags, 0, sizeof(unsigned int) * 2 * P, ctx.stream);
    void* kargs[] = {&args};
    Failed(cudaLaunchCooperativeKernel(
               reinterpret_cast<void*>(GetrfLeafPanelKernel<T, false, kLeafW>), P,
               kLeafThreads, kargs, smem, ctx.stream),
           "getrf leaf (cooperative)");
  } else {
    GetrfLeafPanelKernel<T, false, kLeafW><<<1, kLeafThreads, smem, ctx.stream>>>(args);
  }
  KernelTimerStop(t0, ctx.stream);
  CountLaunch();
  LaunchFailed("getrf leaf");
  if (n > w) {
    GetrfLeafTrailingKernel<T><<<(n - w + 127) / 128, 128, 0, ctx.stream>>>(
        m, w, n, a, lda, ipiv, lanes);
    CountLaunch();
    LaunchFailed("getrf leaf trailing");
  }
}
template void GetrfLeaf<double>(int, int, double*, int, int*, int*, int, int);
template void GetrfLeaf<float>(int, int, float*, int, int*, int*, int, int);

unsigned int SetLeafWaitLimit(unsigned int polls) {
  unsigned int prev = kMaxPolls;
  cudaMemcpyFromSymbol(&prev, g_leaf_poll_limit, sizeof(prev));
  const unsigned int v = polls == 0 ? kMaxPolls : polls;
  Failed(cudaMemcpyToSymbol(g_leaf_poll_limit, &v, sizeof(v)), "leaf wait limit");
  return prev;
}

template <typename T>
void PotrfLeaf(bool upper, int n, T* a, int lda, int* info, int info_base) {
  const int lanes = sizeof(T) == 8 ? RefLanesDouble() : 2 * RefLanesDouble();
  PotrfLeafKernel<T><<<1, 256, 0, Ctx().stream>>>(upper ? 1 : 0, n, a, lda, info, info_base,
                                                  lanes, Ctx().guard);
  CountLaunch();
  LaunchFailed("potrf leaf");
}
template void PotrfLeaf<double>(bool, int, double*, int, int*, int);
template void PotrfLeaf<float>(bool, int, float*, int, int*, int);

// ---------------------------------------------------------------------------
// IDAMAX that allocates nothing (hwyblas_idamax_noalloc).
//
// For callers that must not allocate device memory during a call: a
// cudaMalloc or cudaFree synchronizes the whole device, which stalls work the
// caller keeps in flight on other streams, and a caller that has handed all
// free device memory to its own pool has none left to give. This variant
// runs IamaxKernel with its per-block partial results and its completion
// ticket in a fixed scratch array that is part of the loaded module, takes
// the caller's stream, and leaves the 1-based index in device memory.
//
// Scratch: one block per kNoAllocSegment elements, the partial (value,
// index) of at most kNoAllocMaxBlocks blocks, so n <= 1024 * 16384 =
// 16,777,216 (larger n is rejected). The ticket word must be zero when a call
// starts: set-up zeroes the array, and the kernel's last block resets the
// ticket before it returns. All calls on one device share the array, so two
// calls that overlap in time (different streams without ordering, or two host
// threads) race on it and give wrong results.
namespace {
constexpr int kNoAllocSegment = 16384;
constexpr int kNoAllocMaxBlocks = 1024;
constexpr size_t kNoAllocValueBytes = kNoAllocMaxBlocks * sizeof(double);
constexpr size_t kNoAllocIndexBytes = kNoAllocMaxBlocks * sizeof(int);
constexpr size_t kNoAllocScratchBytes = 16384;  // values, indices, ticket
static_assert(kNoAllocValueBytes + kNoAllocIndexBytes + 256 <= kNoAllocScratchBytes,
              "no-alloc scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// The scratch address on the current device, looked up on every call (the
// lookup allocates nothing). Set-up zeroes the array, ordered on `stream`
// before the launch, the first time a device's address is seen and again
// whenever it changes: a context torn down and created again (for instance
// after cudaDeviceReset) loads the module afresh, possibly elsewhere, with a
// ticket that is not known to be zero.
cudaError_t NoAllocScratch(int device, cudaStream_t stream, void** out) {
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_ptr[device] != ptr) {
    e = cudaMemsetAsync(ptr, 0, kNoAllocScratchBytes, stream);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = ptr;
  }
  *out = ptr;
  return cudaSuccess;
}

// Whether a kernel on `device` may read or write p.
bool DeviceAccessible(const void* p, int device) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (attr.type == cudaMemoryTypeManaged) return true;
  if (attr.type == cudaMemoryTypeDevice) return attr.device == device;
  if (attr.type == cudaMemoryTypeHost) return attr.devicePointer != nullptr;
  return false;
}
}  // namespace

}  // namespace hb

extern "C" HWYBLAS_API int hwyblas_idamax_noalloc(int n, const double* x, int incx,
                                                  int* result, void* stream) {
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (static_cast<long long>(n) >
      static_cast<long long>(hb::kNoAllocMaxBlocks) * hb::kNoAllocSegment) {
    fprintf(stderr,
            "hwyblas_idamax_noalloc: n = %d exceeds the maximum of %d elements "
            "that its fixed scratch holds\n",
            n, hb::kNoAllocMaxBlocks * hb::kNoAllocSegment);
    hb::ReportError("IDAMAX_NOALLOC", 1);
    return -1;
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (device < 0 || device >= hb::kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  if (!hb::DeviceAccessible(result, device)) {
    hb::ReportError("IDAMAX_NOALLOC", 4);
    return -4;
  }
  if (n < 1 || incx <= 0) {  // the reference returns 0 (src/level1.cc:383-402)
    e = cudaMemsetAsync(result, 0, sizeof(int), s);
    return static_cast<int>(e);
  }
  const long long span = static_cast<long long>(n - 1) * incx + 1;
  if (!hb::DeviceAccessible(x, device) ||
      !hb::DeviceAccessible(x + (span - 1), device)) {
    hb::ReportError("IDAMAX_NOALLOC", 2);
    return -2;
  }
  void* scratch = nullptr;
  e = hb::NoAllocScratch(device, s, &scratch);
  if (e != cudaSuccess) return static_cast<int>(e);
  unsigned char* base = static_cast<unsigned char*>(scratch);
  double* values = reinterpret_cast<double*>(base);
  int* indices = reinterpret_cast<int*>(base + hb::kNoAllocValueBytes);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(
      base + hb::kNoAllocValueBytes + hb::kNoAllocIndexBytes);
  const int blocks = (n + hb::kNoAllocSegment - 1) / hb::kNoAllocSegment;
  hb::IamaxKernel<double><<<blocks, 1024, 0, s>>>(n, x, incx, values, indices,
                                                  ticket, result);
  hb::CountLaunch();
  return static_cast<int>(cudaGetLastError());
}
