// Near field of 16-column mixed passes on the 5th-generation tensor cores
// (tcgen05), instantiated once per kernel functor by the kernel tables
// (kernel_table.cuh).  Same arithmetic contract as k_p2p_mma (batched_k.cuh):
// FP32 entries from leaf-anchored coordinates with the FP64 fallback for
// close pairs, entries and charges split into TF32 high / low parts and
// multiplied as hi*hi + hi*lo + lo*hi, FP32 sums per source leaf added in
// FP64 -- but the products run as tcgen05.mma.kind::tf32 issued by one thread,
// with the accumulators in tensor memory, instead of warp-level mma.sync.
//
// Mapping: one CTA of 256 threads per pair of horizontally adjacent sibling
// leaves (quadtree boxes 2c and 2c + 1): the MMA's 128 rows are the two
// leaves' targets (64 rows each, so leaves of at most 64 points), and its K
// dimension runs over the union of the two leaves' 3 x 3 neighbourhoods (at
// most 12 source leaves, 32 sources per stage).  A row's entries for a source
// leaf outside its own neighbourhood are zero.  Per stage the 256 threads
// write the entries (A, 128 x 32, high and low parts) and the charges (B,
// 16 RHS x 32 sources, high and low parts) into shared memory in the K-major
// canonical layout without swizzle (8-row x 16-byte core matrices, K-adjacent
// cores 128 B apart, row groups 1 KB apart); thread 0 issues 4 K-steps x 3
// products into the source leaf's accumulator and commits them to the
// stage's mbarrier.  Two stages alternate; two 16-column accumulators
// alternate by source leaf, so the FP32 sum of leaf m is read (tcgen05.ld)
// into FP64 registers while leaf m + 1 accumulates.  Every mbarrier wait is
// bounded: on a timeout the CTA sets *err, stops issuing, waits (bounded) for
// its MMAs, frees its tensor memory and returns.
#pragma once
#include <stdint.h>

#include "batched_k.cuh"
#include "tcgen05.cuh"

namespace afmm {

namespace p2p_tc_detail {

using batched_detail::fallback_r2_b;
using batched_detail::split_tf32_mask;

constexpr int kThreads = 256;
constexpr int kRows = 128;      // M: 64 targets of each of the two leaves
constexpr int kLeafMax = 64;    // points per leaf this kernel takes
constexpr int kChunk = 32;      // sources per stage (K)
constexpr int kUnionMax = 12;   // source leaves of the two neighbourhoods
constexpr int kChunksMax = kUnionMax * (kLeafMax / kChunk);
constexpr uint32_t kBytesA = kRows * kChunk * 4;  // one A matrix (high or low): 16 KB
constexpr uint32_t kBytesB = 16 * kChunk * 4;     // one B matrix: 2 KB
constexpr uint32_t kStage = 2 * kBytesA + 2 * kBytesB;
constexpr uint32_t kCoreK = 128;                  // bytes between K-adjacent core matrices
constexpr uint32_t kCoreRows = (kChunk / 4) * 128;  // bytes between 8-row groups (1 KB)
constexpr size_t kSmem = 2 * (size_t)kStage + (size_t)kUnionMax * kLeafMax * sizeof(float2) + 1024;
constexpr uint32_t kTmemCols = 32;  // two 16-column FP32 accumulators

using namespace tc;

template <class K>
__global__ void __launch_bounds__(kThreads, 2) k_p2p_tc(NearView nv, KernelParams kp, const uint2* __restrict__ qhl,
                                                        double* __restrict__ ys, int L, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_nu, s_nch, s_fail;
  __shared__ int s_usrc[kUnionMax], s_ucnt[kUnionMax], s_uok[kUnionMax];
  __shared__ float s_uthr[kUnionMax][2];
  __shared__ float2 s_udel[kUnionMax];
  __shared__ unsigned char s_chleaf[kChunksMax], s_choff[kChunksMax], s_chfirst[kChunksMax];
  const int tid = threadIdx.x, warp = tid >> 5;
  const long b1 = nv.leaf0 + 2L * blockIdx.x, b2 = b1 + 1;  // leaf0 is even
  const int n1 = nv.leaf_cnt[b1], n2 = nv.leaf_cnt[b2];
  const int s01 = nv.leaf_start[b1], s02 = nv.leaf_start[b2];
  const double2 a1 = nv.anchor[b1];
  if (tid == 0) {
    // union of the two 3 x 3 neighbourhoods (the leaves share their row of cells)
    int x1, y1, x2, y2;
    cell_of(b1, L, x1, y1);
    cell_of(b2, L, x2, y2);
    const int side = 1 << L, xl = min(x1, x2);
    const float sp1 = nv.span[b1], sp2 = nv.span[b2];
    int nu = 0, nch = 0;
    for (int cy = y1 - 1; cy <= y1 + 1; ++cy)
      for (int cx = xl - 1; cx <= xl + 2; ++cx) {
        if (cx < 0 || cy < 0 || cx >= side || cy >= side) continue;
        const long u = box_of(cx, cy, L);
        // empty leaves take no slot: union slots with chunks stay consecutive,
        // which the alternation of the two accumulators relies on
        if (nv.leaf_cnt[u] == 0) continue;
        const int ok = (abs(cx - x1) <= 1 ? 1 : 0) | (abs(cx - x2) <= 1 ? 2 : 0);
        const double2 au = nv.anchor[u];
        s_usrc[nu] = nv.leaf_start[u];
        s_ucnt[nu] = nv.leaf_cnt[u];
        s_uok[nu] = ok;
        s_udel[nu] = make_float2((float)(a1.x - au.x), (float)(a1.y - au.y));
        s_uthr[nu][0] = fmaxf(fallback_r2_b<K>(sp1, nv.span[u]), 1.0e-30f);
        s_uthr[nu][1] = fmaxf(fallback_r2_b<K>(sp2, nv.span[u]), 1.0e-30f);
        for (int off = 0; off < nv.leaf_cnt[u]; off += kChunk) {
          s_chleaf[nch] = (unsigned char)nu;
          s_choff[nch] = (unsigned char)off;
          s_chfirst[nch] = off == 0;
          ++nch;
        }
        ++nu;
      }
    s_nu = nu;
    s_nch = nch;
    s_fail = 0;
    mbar_init(smem_addr(&s_mbar[0]), 1);
    mbar_init(smem_addr(&s_mbar[1]), 1);
    mbar_init_fence();
  }
  __syncwarp();
  if (warp == 0) tmem_alloc(&s_tmem, kTmemCols);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  const int nu = s_nu, nch = s_nch;
  // sources of every union leaf in leaf b1's frame
  float2* sx = (float2*)(smem + 2 * (size_t)kStage);
  for (int u = 0; u < nu; ++u)
    for (int t = tid; t < s_ucnt[u]; t += kThreads) {
      float2 p = nv.rel[s_usrc[u] + t];
      p.x -= s_udel[u].x;
      p.y -= s_udel[u].y;
      sx[u * kLeafMax + t] = p;
    }
  // this thread's row (target) and half of each stage's sources
  const int row = tid & (kRows - 1), half = tid >> 7;
  const int leafbit = row < kLeafMax ? 1 : 2;
  const int ti = row < kLeafMax ? row : row - kLeafMax;
  const bool rowok = ti < (row < kLeafMax ? n1 : n2);
  const int pi = row < kLeafMax ? s01 + ti : s02 + ti;
  float2 xr = make_float2(0.0f, 0.0f);
  if (rowok) {
    xr = nv.rel[pi];
    if (row >= kLeafMax) {
      const double2 a2 = nv.anchor[b2];
      xr.x -= (float)(a1.x - a2.x);
      xr.y -= (float)(a1.y - a2.y);
    }
  }
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  double acc[16];
#pragma unroll
  for (int n = 0; n < 16; ++n) acc[n] = 0.0;
  // FP32 sums of a finished source leaf into the FP64 sums (warps 0-3 own
  // the accumulator lanes: warp w reads lanes 32w .. 32w + 31 = rows)
  auto read_leaf = [&](int m) {
    if (warp < 4) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(16 * (m & 1)), v);
#pragma unroll
      for (int n = 0; n < 16; ++n) acc[n] += (double)v[n];
    }
  };
  __syncthreads();
  int issued = -1;  // last chunk whose MMAs were committed
  for (int i = 0; i < nch; ++i) {
    const int st = i & 1;
    unsigned char* sA = smem + (size_t)st * kStage;  // A high, A low, B high, B low
    const int m = s_chleaf[i], off = s_choff[i];
    if (i >= 2) {
      const bool ok = mbar_wait(smem_addr(&s_mbar[st]), (uint32_t)((i - 2) >> 1) & 1u);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) s_fail = 1;
        break;
      }
      fence_after();
      // the leaf two back is complete (its last chunk is at most i - 2):
      // take its sums before this leaf's first product overwrites them
      if (s_chfirst[i] && m >= 2) read_leaf(m - 2);
    }
    // entries of this thread's row for its 16 sources of the stage
    {
      const int cnt = s_ucnt[m], src = s_usrc[m];
      const bool live = rowok && (s_uok[m] & leafbit);
      const float thr = s_uthr[m][leafbit - 1];
      const float2* xs = sx + m * kLeafMax;
      uint32_t hi[16], lo[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int o = off + half * 16 + j;
        float kv = 0.0f;
        if (live && o < cnt) {
          const float2 q = xs[o];
          const float dx = xr.x - q.x, dy = xr.y - q.y;
          const float r2 = fmaf(dx, dx, dy * dy);
          kv = K::eval32_pos(r2, a32, p32);
          if (r2 < thr) {  // close pair (the diagonal among them): FP64 from the exact coordinates
            const int qi = src + o;
            if (pi == qi) {
              kv = (float)K::at_zero(kp);
            } else {
              const double2 pa = nv.pts[pi], pc = nv.pts[qi];
              kv = (float)K::eval_exact(r2_exact(pa.x, pa.y, pc.x, pc.y), kp);
            }
          }
        }
        split_tf32_mask(kv, hi[j], lo[j]);
      }
      unsigned char* rowA = sA + (size_t)(row >> 3) * kCoreRows + (size_t)(row & 7) * 16;
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const size_t o = (size_t)(half * 4 + g) * kCoreK;
        *reinterpret_cast<uint4*>(rowA + o) = make_uint4(hi[4 * g], hi[4 * g + 1], hi[4 * g + 2], hi[4 * g + 3]);
        *reinterpret_cast<uint4*>(rowA + kBytesA + o) =
            make_uint4(lo[4 * g], lo[4 * g + 1], lo[4 * g + 2], lo[4 * g + 3]);
      }
    }
    // charges: thread -> (high or low part, column n, 4 sources)
    {
      const int hl = tid >> 7, n = (tid >> 3) & 15, kg = tid & 7;
      const int cnt = s_ucnt[m], src = s_usrc[m];
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = off + kg * 4 + j;
        uint32_t x = 0u;
        if (o < cnt) {
          const uint2 v = qhl[(long)(src + o) * 16 + n];
          x = hl ? v.y : v.x;
        }
        w[j] = x;
      }
      unsigned char* b = sA + 2 * kBytesA + (size_t)hl * kBytesB + (size_t)(n >> 3) * kCoreRows +
                         (size_t)kg * kCoreK + (size_t)(n & 7) * 16;
      *reinterpret_cast<uint4*>(b) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const uint32_t aH = smem_addr(sA), aL = aH + kBytesA, bH = aH + 2 * kBytesA, bL = bH + kBytesB;
      const uint32_t d = tmem + (uint32_t)(16 * (m & 1));
#pragma unroll
      for (int kk = 0; kk < kChunk / 8; ++kk) {
        const uint32_t ko = (uint32_t)kk * 2 * kCoreK;  // 8 sources = two K-adjacent core matrices
        const uint64_t dah = smem_desc(aH + ko, kCoreK, kCoreRows), dal = smem_desc(aL + ko, kCoreK, kCoreRows);
        const uint64_t dbh = smem_desc(bH + ko, kCoreK, kCoreRows), dbl = smem_desc(bL + ko, kCoreK, kCoreRows);
        mma_tf32(d, dah, dbh, kIdescTf32M128N16, (s_chfirst[i] && kk == 0) ? 0u : 1u);
        mma_tf32(d, dah, dbl, kIdescTf32M128N16, 1u);
        mma_tf32(d, dal, dbh, kIdescTf32M128N16, 1u);
      }
      mma_commit(smem_addr(&s_mbar[st]));
    }
    issued = i;
  }
  // drain: the commits of the last two chunks (not waited for in the loop)
  // arrive, then the last one or two leaves' sums
  bool ok = true;
  if (issued >= 1) ok = mbar_wait(smem_addr(&s_mbar[(issued - 1) & 1]), (uint32_t)((issued - 1) >> 1) & 1u);
  if (issued >= 0) ok = mbar_wait(smem_addr(&s_mbar[issued & 1]), (uint32_t)(issued >> 1) & 1u) && ok;
  const bool fail = __syncthreads_or(!ok) || s_fail;
  fence_after();
  if (!fail && nch > 0) {
    const int mlast = s_chleaf[nch - 1];
    if (mlast >= 1) read_leaf(mlast - 1);
    read_leaf(mlast);
    if (warp < 4 && rowok) {
      double2* o = reinterpret_cast<double2*>(ys + (long)pi * 16);
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        double2 v = o[n];
        v.x += acc[2 * n];
        v.y += acc[2 * n + 1];
        o[n] = v;
      }
    }
  }
  if (fail && tid == 0) *(volatile int*)err = 1;  // host-mapped flag
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// Launches k_p2p_tc over all leaf pairs (leaves of at most 64 points).
template <class K>
void p2p_tc_batched16(const NearView& nv, const KernelParams& kp, const uint2* qhl, double* ys, int L, int* err,
                      cudaStream_t s) {
  if (nv.nmax > kLeafMax || (nv.nleaf & 1) || (nv.leaf0 & 1))
    throw Error{AFMM_BAD_ARG, "tcgen05 near field takes leaves of <= 64 points in sibling pairs"};
  allow_smem(k_p2p_tc<K>, kSmem);
  k_p2p_tc<K><<<(int)(nv.nleaf / 2), kThreads, kSmem, s>>>(nv, kp, qhl, ys, L, err);
  AFMM_LAUNCH_CHECK();
}

}  // namespace p2p_tc_detail

}  // namespace afmm
