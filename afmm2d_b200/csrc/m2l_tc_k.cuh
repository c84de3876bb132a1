// M2L of 16-column mixed passes on the 5th-generation tensor cores
// (tcgen05) from the 32-bit fixed-point blocks (m2l_q / m2l_dec, the same
// stored copy the FP64-tile kernels decode).  Arithmetic: every entry
// decoded to FP32, entries and charges split into TF32 high / low parts and
// multiplied as hi*hi + hi*lo + lo*hi (tcgen05.mma.kind::tf32 issued by one
// thread), FP32 sums per source box in tensor memory added in FP64 -- the
// contract of the mixed near field, applied to the far field.
//
// Mapping: one CTA of 256 threads per row tile of a parent box: the rows of
// the parent's four children (quadtree boxes 4P .. 4P + 3), concatenated in
// child order and cut into balanced tiles of at most 128 rows (the MMA's M).
// The K dimension runs over the union of the tile's children's interaction
// lists -- boxes among the 6 x 6 children of the parent's 3 x 3
// neighbourhood -- source box by source box, 32 skeleton columns per stage.
// A row's entries for a source outside its own box's list are zero.  The
// stored block (child c, slot s) is column-major r_c x r_s, so 32 columns of
// it are one contiguous piece: those pieces are streamed into L2 two stages
// ahead (cp.async.bulk.prefetch.L2), and each thread reads its row's 16
// entries of the stage (a warp's lanes read consecutive rows: 128-byte
// lines).  Stages, accumulators, waits and the error path are those of the
// tcgen05 near field (p2p_tc_k.cuh): two shared-memory stages, two 16-column
// accumulators alternating by source box, every mbarrier wait bounded (~1 s;
// on a timeout the CTA sets *err, stops issuing, waits for its MMAs, frees
// its tensor memory and returns).
//
// Accuracy: the far field's sums cancel and the L2P weights amplify their
// rounding, so FP32 products and sums are not enough on deep trees (measured
// 6.2e-5 of the FP64 path on the 4,194,304-point mixture at TOL 6, max over
// 16 columns, and 6.6e-6 on 1,048,576 uniform points at TOL 10, against
// 5.1e-7 / 4.3e-8 for the FP64 tiles).  It is an explicit choice (tuning value m2l_tc), never the
// autotuner's.
#pragma once
#include <stdint.h>

#include "batched_common.cuh"
#include "fmm.cuh"
#include "tcgen05.cuh"

namespace afmm {

namespace m2l_tc_detail {

using namespace tc;

constexpr int kThreads = 256;
constexpr int kRows = 128;   // M: rows of one tile
constexpr int kChunk = 32;   // source columns per stage (K)
constexpr int kGrid = 36;    // 6 x 6 cells around the parent
constexpr uint32_t kBytesA = kRows * kChunk * 4;  // one A matrix (high or low): 16 KB
constexpr uint32_t kBytesB = 16 * kChunk * 4;     // one B matrix: 2 KB
constexpr uint32_t kStage = 2 * kBytesA + 2 * kBytesB;
constexpr uint32_t kCoreK = 128;                    // bytes between K-adjacent core matrices
constexpr uint32_t kCoreRows = (kChunk / 4) * 128;  // bytes between 8-row groups (1 KB)
constexpr size_t kSmem = 2 * (size_t)kStage;
constexpr uint32_t kTmemCols = 32;  // two 16-column FP32 accumulators

// A 32-bit fixed-point entry (u - 2^31) 2^k in FP32, with scale = 2^(k + 31)
// the block's largest magnitude rounded up to a power of two (0 for an
// all-zero block, NaN for a block holding a non-finite entry): the integer
// rounded to 24 bits, times 2^-31, times the scale, both exact.
__device__ __forceinline__ float decode_q32_f(uint32_t u, float scale) {
  return ((float)(int)(u ^ 0x80000000u) * __int_as_float(0x30000000)) * scale;
}

// Prefetches [begin, end) into L2 in 4 KB pieces spread over 8 lanes
// (`part` = 0..7); start rounded down, end up to 16 bytes (the block arrays
// carry that much padding).
__device__ __forceinline__ void prefetch_piece8(const void* begin, const void* end, int part) {
  const uintptr_t a = (uintptr_t)begin & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)end + 15) & ~(uintptr_t)15;
  for (uintptr_t p = a + (uintptr_t)part * 4096; p < e; p += 8 * 4096) {
    const uintptr_t left = e - p;
    prefetch_l2_bulk(p, (uint32_t)(left < 4096 ? left : 4096));
  }
}

__global__ void __launch_bounds__(kThreads, 2) k_m2l_tc(LevelSet ls, const double* const* __restrict__ qhat_lv,
                                                        double* const* __restrict__ yhat_lv, int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail, s_nu, s_j, s_t0, s_t1;
  __shared__ long s_parent;
  __shared__ int s_crank[4], s_cskel[4], s_crow0[5];
  __shared__ int s_slot[4][kGrid];        // slot of grid cell g in child c's list (-1: none)
  __shared__ long long s_pos[4][kGrid];   // first entry of block (c, slot) in m2l_q
  __shared__ float s_scale[4][kGrid];     // its decode scale 2^(k + 31)
  __shared__ int s_urank[kGrid], s_uskel[kGrid];  // rank and first skeleton row of the cell's box
  __shared__ int s_ulist[kGrid];          // union of the tile's lists (grid cells, in order)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    const long t = blockIdx.x;
    int j = 0;
    while (j + 1 < ls.nlev && t >= ls.pt0[j + 1]) ++j;
    const LevelView& v = ls.lv[j];
    const long tl = t - ls.pt0[j];
    const long P = v.ptile_par[tl];
    int row0 = 0;
    for (int c = 0; c < 4; ++c) {
      const int r = v.rank[4 * P + c];
      s_crank[c] = r;
      s_cskel[c] = v.skel_off[4 * P + c];
      s_crow0[c] = row0;
      row0 += r;
    }
    s_crow0[4] = row0;
    s_t0 = v.ptile_row[tl];
    s_t1 = (tl + 1 < v.nptiles && v.ptile_par[tl + 1] == P) ? v.ptile_row[tl + 1] : row0;
    s_j = j;
    s_parent = P;
    s_fail = 0;
    mbar_init(smem_addr(&s_mbar[0]), 1);
    mbar_init(smem_addr(&s_mbar[1]), 1);
    mbar_init_fence();
  }
  for (int i = tid; i < 4 * kGrid; i += kThreads) (&s_slot[0][0])[i] = -1;
  if (warp == 0) tmem_alloc(&s_tmem, kTmemCols);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  const int j = s_j;
  const LevelView& v = ls.lv[j];
  const int level = ls.src[j] + 2;
  const long P = s_parent;
  // each child's list (warp c): slot offsets in the stored order (slots
  // 0..39, a block of r_c x r_s entries per slot whose source has rank > 0)
  // and the grid cell of each source
  if (warp < 4) {
    const int c = warp;
    const long b = 4 * P + c;
    const int r = s_crank[c];
    int px, py;
    cell_of(P, level - 1, px, py);
    const int ox = 2 * px - 2, oy = 2 * py - 2;
    const int srcA = v.il[b * 40 + lane];
    const int srcB = lane < 8 ? v.il[b * 40 + 32 + lane] : -1;
    const int rcA = (srcA >= 0 && r > 0) ? v.rank[srcA] : 0;
    const int rcB = (srcB >= 0 && r > 0) ? v.rank[srcB] : 0;
    const long long nA = (long long)r * rcA, nB = (long long)r * rcB;
    long long sA = nA, sB = nB;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long ta = __shfl_up_sync(0xffffffffu, sA, o), tb = __shfl_up_sync(0xffffffffu, sB, o);
      if (lane >= o) {
        sA += ta;
        sB += tb;
      }
    }
    const long long totA = __shfl_sync(0xffffffffu, sA, 31);
    const long long base = v.m2l_off[b];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int src = h ? srcB : srcA, rc = h ? rcB : rcA, slot = h ? 32 + lane : lane;
      if (rc == 0) continue;
      const long long off = h ? base + totA + sB - nB : base + sA - nA;
      int ux, uy;
      cell_of(src, level, ux, uy);
      const int gx = ux - ox, gy = uy - oy;
      if (gx < 0 || gy < 0 || gx >= 6 || gy >= 6) {  // not a child of the parent's neighbours
        s_fail = 1;
        continue;
      }
      const int g = gy * 6 + gx;
      s_slot[c][g] = slot;
      s_pos[c][g] = off;
      s_scale[c][g] = (float)(v.m2l_dec[b * 40 + slot].x * 2147483648.0);
      s_urank[g] = rc;  // the same values from every child listing the cell
      s_uskel[g] = v.skel_off[src];
    }
  }
  __syncthreads();
  if (tid == 0) {
    int nu = 0;
    for (int g = 0; g < kGrid; ++g) {
      bool any = false;
      for (int c = 0; c < 4; ++c)
        any |= s_crow0[c] < s_t1 && s_crow0[c + 1] > s_t0 && s_slot[c][g] >= 0;
      if (any) s_ulist[nu++] = g;
    }
    s_nu = nu;
  }
  __syncthreads();
  const int nu = s_nu;
  // this thread's row of the tile and half of each stage's 32 columns
  const int row = tid & (kRows - 1), half = tid >> 7;
  const int crow = s_t0 + row;
  const bool rowok = crow < s_t1;
  int c = 0;
  while (c < 3 && crow >= s_crow0[c + 1]) ++c;
  const int ii = crow - s_crow0[c];
  const int rrow = s_crank[c];
  const uint32_t* __restrict__ mq = v.m2l_q;
  const double* __restrict__ qh = qhat_lv[ls.src[j]];
  double* __restrict__ yh = yhat_lv[ls.src[j]];
  double acc[16];
#pragma unroll
  for (int n = 0; n < 16; ++n) acc[n] = 0.0;
  auto read_src = [&](int m) {
    if (warp < 4) {
      float x[16];
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(16 * (m & 1)), x);
#pragma unroll
      for (int n = 0; n < 16; ++n) acc[n] += (double)x[n];
    }
  };
  // L2 prefetch of a stage's block pieces (warp 4: lanes 8c .. 8c + 7 for child c)
  auto prefetch_stage = [&](int m, int off) {
    if (warp == 4 && m < nu) {
      const int pc = lane >> 3, g = s_ulist[m];
      const int sl = s_slot[pc][g];
      if (sl >= 0 && s_crow0[pc] < s_t1 && s_crow0[pc + 1] > s_t0) {
        const int rp = s_crank[pc], cnt = min(kChunk, s_urank[g] - off);
        const uint32_t* a = mq + s_pos[pc][g] + (long long)off * rp;
        prefetch_piece8(a, a + (long long)cnt * rp, lane & 7);
      }
    }
  };
  // stages 0 and 1 now; stage i + 2 while stage i is written
  int pm = 0, poff = 0;
  for (int k = 0; k < 2 && pm < nu; ++k) {
    prefetch_stage(pm, poff);
    poff += kChunk;
    if (poff >= s_urank[s_ulist[pm]]) {
      poff = 0;
      ++pm;
    }
  }
  int i = 0, issued = -1;
  bool stop = false;
  for (int m = 0; m < nu && !stop; ++m) {
    const int g = s_ulist[m];
    const int ru = s_urank[g], sku = s_uskel[g];
    const int slot = rowok ? s_slot[c][g] : -1;
    const long long bpos = slot >= 0 ? s_pos[c][g] : 0;
    const float scale = slot >= 0 ? s_scale[c][g] : 0.0f;
    for (int off = 0; off < ru; off += kChunk, ++i) {
      const int st = i & 1;
      unsigned char* sA = smem + (size_t)st * kStage;  // A high, A low, B high, B low
      const int cnt = min(kChunk, ru - off);
      // this stage's loads first: they overlap the wait for stage i - 2
      uint32_t raw[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int k = off + half * 16 + q;
        raw[q] = (slot >= 0 && k < ru) ? mq[bpos + (long long)k * rrow + ii] : 0x80000000u;
      }
      const int kr = tid >> 3, n2 = (tid & 7) * 2;
      double2 qv = make_double2(0.0, 0.0);
      if (kr < cnt) qv = *reinterpret_cast<const double2*>(qh + (long)(sku + off + kr) * 16 + n2);
      prefetch_stage(pm, poff);
      if (pm < nu) {
        poff += kChunk;
        if (poff >= s_urank[s_ulist[pm]]) {
          poff = 0;
          ++pm;
        }
      }
      if (i >= 2) {
        const bool ok = mbar_wait(smem_addr(&s_mbar[st]), (uint32_t)((i - 2) >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
          if (tid == 0) s_fail = 1;
          stop = true;
          break;
        }
        fence_after();
        // source m - 2 is complete (its last stage is at most i - 2): take
        // its sums before source m's first product overwrites them
        if (off == 0 && m >= 2) read_src(m - 2);
      }
      // entries of this thread's row, TF32 high and low parts
      {
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int k = off + half * 16 + q;
          const float e = (slot >= 0 && k < ru) ? decode_q32_f(raw[q], scale) : 0.0f;
          split_tf32(e, hi[q], lo[q]);
        }
        unsigned char* rowA = sA + (size_t)(row >> 3) * kCoreRows + (size_t)(row & 7) * 16;
#pragma unroll
        for (int g4 = 0; g4 < 4; ++g4) {
          const size_t o = (size_t)(half * 4 + g4) * kCoreK;
          *reinterpret_cast<uint4*>(rowA + o) = make_uint4(hi[4 * g4], hi[4 * g4 + 1], hi[4 * g4 + 2], hi[4 * g4 + 3]);
          *reinterpret_cast<uint4*>(rowA + kBytesA + o) =
              make_uint4(lo[4 * g4], lo[4 * g4 + 1], lo[4 * g4 + 2], lo[4 * g4 + 3]);
        }
      }
      // charges of source row kr, columns n2 and n2 + 1
      {
        uint32_t h0, l0, h1, l1;
        split_tf32((float)qv.x, h0, l0);
        split_tf32((float)qv.y, h1, l1);
        unsigned char* bB = sA + 2 * kBytesA + (size_t)(kr >> 2) * kCoreK + (size_t)(kr & 3) * 4;
        const int na = n2, nb = n2 + 1;
        *reinterpret_cast<uint32_t*>(bB + (size_t)(na >> 3) * kCoreRows + (size_t)(na & 7) * 16) = h0;
        *reinterpret_cast<uint32_t*>(bB + (size_t)(nb >> 3) * kCoreRows + (size_t)(nb & 7) * 16) = h1;
        *reinterpret_cast<uint32_t*>(bB + kBytesB + (size_t)(na >> 3) * kCoreRows + (size_t)(na & 7) * 16) = l0;
        *reinterpret_cast<uint32_t*>(bB + kBytesB + (size_t)(nb >> 3) * kCoreRows + (size_t)(nb & 7) * 16) = l1;
      }
      fence_async_smem();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        const uint32_t aH = smem_addr(sA), aL = aH + kBytesA, bH = aH + 2 * kBytesA, bL = bH + kBytesB;
        const uint32_t d = tmem + (uint32_t)(16 * (m & 1));
        const int nks = (cnt + 7) >> 3;  // K-steps of 8 columns holding data
        for (int kk = 0; kk < nks; ++kk) {
          const uint32_t ko = (uint32_t)kk * 2 * kCoreK;  // 8 columns = two K-adjacent core matrices
          const uint64_t dah = smem_desc(aH + ko, kCoreK, kCoreRows), dal = smem_desc(aL + ko, kCoreK, kCoreRows);
          const uint64_t dbh = smem_desc(bH + ko, kCoreK, kCoreRows), dbl = smem_desc(bL + ko, kCoreK, kCoreRows);
          mma_tf32(d, dah, dbh, kIdescTf32M128N16, (off == 0 && kk == 0) ? 0u : 1u);
          mma_tf32(d, dah, dbl, kIdescTf32M128N16, 1u);
          mma_tf32(d, dal, dbh, kIdescTf32M128N16, 1u);
        }
        mma_commit(smem_addr(&s_mbar[st]));
      }
      issued = i;
    }
  }
  // drain: the commits of the last two stages (not waited for in the loop)
  // arrive, then the last one or two sources' sums
  bool ok = true;
  if (issued >= 1) ok = mbar_wait(smem_addr(&s_mbar[(issued - 1) & 1]), (uint32_t)((issued - 1) >> 1) & 1u);
  if (issued >= 0) ok = mbar_wait(smem_addr(&s_mbar[issued & 1]), (uint32_t)(issued >> 1) & 1u) && ok;
  const bool fail = __syncthreads_or(!ok) || s_fail;
  fence_after();
  if (!fail) {
    if (nu >= 2) read_src(nu - 2);
    if (nu >= 1) read_src(nu - 1);
    if (warp < 4 && rowok) {
      double2* o = reinterpret_cast<double2*>(yh + (long)(s_cskel[c] + ii) * 16);
#pragma unroll
      for (int n = 0; n < 8; ++n) o[n] = make_double2(acc[2 * n], acc[2 * n + 1]);
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

}  // namespace m2l_tc_detail

}  // namespace afmm
