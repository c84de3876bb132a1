// Batched mixed-precision matvec: RC right-hand sides per pass (RC = 4, 8 or
// 16), each operator entry read or evaluated once and applied to all of them.
//
// Layout: point-major blocks, value (i, c) at i*RC + c, for the sorted charges
// and potentials and for the outgoing / incoming vectors of every level, so a
// warp's lanes (consecutive rows of one box) read the same RC-vector of a
// source with one broadcast load.
//  * M2M / L2L: FP64 L2P (row-major / column-major), one thread per output
//    row with RC FP64 accumulators.
//  * M2L: the stored blocks (one HBM read for all RC columns; the 32-bit
//    fixed-point copy in mixed precision, the FP64 blocks otherwise), or
//    entries evaluated on the fly in FP64 from the skeleton coordinates when
//    no blocks are stored, multiplied with the RC-column charge blocks on the
//    FP64 tensor cores (8 rows x 4 sources tiles).
//  * Near field: entries in FP32 from leaf-relative coordinates with the FP64
//    fallback for close pairs (as in the single-RHS mixed path), multiplied
//    on the TF32 tensor cores in a three-term high/low split (16 targets x 8
//    sources tiles), tile sums per source leaf accumulated in FP64.
// With RC = 4 the same products run on the FMA pipes.
#include <algorithm>

#include "batched_common.cuh"
#include "kernel_table.cuh"
#include "m2l_i8_k.cuh"
#include "m2l_tc_k.cuh"
#include "mixed.cuh"

namespace afmm {

namespace {

// Gather through a shared-memory transpose: a block takes kTileJ consecutive
// points, reads each column of q as one contiguous run, and writes each
// point's sorted row qs[iperm[j]][0:RC] (one 128-byte line for RC = 16),
// and also as interleaved TF32 high / low parts (the tensor-core near
// field's charges) unless the pass is FP64 throughout.
constexpr int kTileJ = 128;

template <int RC>
__global__ void __launch_bounds__(256) k_gather_b(const double* __restrict__ q, int64_t ldq, int ncols,
                                                  const int32_t* __restrict__ iperm, int N, double* qs, uint2* qhl,
                                                  int fp64_only) {
  __shared__ double tile[RC][kTileJ + 1];
  const long j0 = (long)blockIdx.x * kTileJ;
  for (int idx = threadIdx.x; idx < RC * kTileJ; idx += blockDim.x) {
    const int c = idx / kTileJ, jj = idx % kTileJ;
    const long j = j0 + jj;
    tile[c][jj] = (c < ncols && j < N) ? q[(long)c * ldq + j] : 0.0;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < (RC / 2) * kTileJ; idx += blockDim.x) {
    const int jj = idx / (RC / 2), cp = idx % (RC / 2);
    const long j = j0 + jj;
    if (j >= N) continue;
    const double v0 = tile[2 * cp][jj], v1 = tile[2 * cp + 1][jj];
    const long d = (long)iperm[j] * RC + 2 * cp;
    *reinterpret_cast<double2*>(qs + d) = make_double2(v0, v1);
    if (fp64_only) continue;
    uint4 hl;
    split_tf32((float)v0, hl.x, hl.y);
    split_tf32((float)v1, hl.z, hl.w);
    *reinterpret_cast<uint4*>(qhl + d) = hl;
  }
}

// Scatter through a shared-memory transpose: a block takes kTileJ consecutive
// points, reads their sorted rows ys[iperm[j]][0:RC], and writes each column
// of y as one contiguous run.
// With ys_near, the near field's potentials are added to the far field's
// (the one addition the near-field kernels would have made into ys).
template <int RC>
__global__ void __launch_bounds__(256) k_scatter_b(const double* __restrict__ ys, const double* __restrict__ ys_near,
                                                   const int32_t* __restrict__ iperm, int N, int ncols, double* y,
                                                   int64_t ldy) {
  __shared__ double tile[RC][kTileJ + 1];
  const long j0 = (long)blockIdx.x * kTileJ;
  for (int idx = threadIdx.x; idx < (RC / 2) * kTileJ; idx += blockDim.x) {
    const int jj = idx / (RC / 2), cp = idx % (RC / 2);
    const long j = j0 + jj;
    if (j >= N) continue;
    const long o = (long)iperm[j] * RC + 2 * cp;
    double2 v = *reinterpret_cast<const double2*>(ys + o);
    if (ys_near) {
      const double2 w = *reinterpret_cast<const double2*>(ys_near + o);
      v.x += w.x;
      v.y += w.y;
    }
    tile[2 * cp][jj] = v.x;
    tile[2 * cp + 1][jj] = v.y;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < RC * kTileJ; idx += blockDim.x) {
    const int c = idx / kTileJ, jj = idx % kTileJ;
    const long j = j0 + jj;
    if (c < ncols && j < N) y[(long)c * ldy + j] = tile[c][jj];
  }
}

// ------------------------------------------------------- tensor-core tiles
// FP64 tensor-core product of one warp's row chunk: for NT tiles of 8 rows,
// c[u] += A[rows of tile u][0:K] * B[0:K][0:RC], A column-major with leading
// dimension lda (A points at the lane's row of tile 0: base + first row +
// trow), B point-major (k, col) at k*RC + col.  Each 4-column step issues all
// of its A and B loads before its MMAs; for lda >= 32 the warp's A loads are
// five contiguous runs of up to 40 rows.
template <int RC, int NT>
__device__ __forceinline__ void mma_rows(double (&c)[NT][RC / 8][2], const double* __restrict__ A, int lda, int K,
                                         const double* __restrict__ B, const bool (&rowok)[NT], int trow, int tsrc) {
#pragma unroll 4
  for (int k0 = 0; k0 < K; k0 += 4) {
    const int k = k0 + tsrc;
    const bool vk = k < K;
    const double* Ak = A + (long)k * lda;
    double a[NT], bq[RC / 8];
#pragma unroll
    for (int u = 0; u < NT; ++u) a[u] = (vk && rowok[u]) ? Ak[u * 8] : 0.0;
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) bq[t] = vk ? B[(long)k * RC + t * 8 + trow] : 0.0;
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) mma_f64_8x8x4(c[u][t][0], c[u][t][1], a[u], bq[t]);
  }
}

// mma_rows with the 32-bit fixed-point M2L entries of one block (decode
// constants `dec`, decode_q32): each 4-column step loads its A entries as
// 32-bit words (half the bytes of FP64) and decodes them exactly before the
// FP64 products.
template <int RC, int NT>
__device__ __forceinline__ void mma_rows_q32(double (&c)[NT][RC / 8][2], const uint32_t* __restrict__ A, int lda,
                                             int K, double2 dec, const double* __restrict__ B,
                                             const bool (&rowok)[NT], int trow, int tsrc) {
#pragma unroll 4
  for (int k0 = 0; k0 < K; k0 += 4) {
    const int k = k0 + tsrc;
    const bool vk = k < K;
    const uint32_t* Ak = A + (long)k * lda;
    uint32_t ua[NT];
    double bq[RC / 8];
#pragma unroll
    for (int u = 0; u < NT; ++u) ua[u] = (vk && rowok[u]) ? Ak[u * 8] : 0x80000000u;  // 2^31 decodes to 0
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) bq[t] = vk ? B[(long)k * RC + t * 8 + trow] : 0.0;
#pragma unroll
    for (int u = 0; u < NT; ++u) {
      const double a = decode_q32(ua[u], dec);
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) mma_f64_8x8x4(c[u][t][0], c[u][t][1], a, bq[t]);
    }
  }
}

template <int RC, int NT>
__device__ __forceinline__ void zero_tiles(double (&c)[NT][RC / 8][2]) {
#pragma unroll
  for (int u = 0; u < NT; ++u)
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) c[u][t][0] = c[u][t][1] = 0.0;
}

// Writes (or adds) the chunk's rows: out points at row 0 of the chunk.
template <int RC, int NT, bool ADD>
__device__ __forceinline__ void store_tiles(const double (&c)[NT][RC / 8][2], double* __restrict__ out,
                                            const bool (&rowok)[NT], int trow, int tsrc) {
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    if (rowok[u]) {
      double2* o = reinterpret_cast<double2*>(out + (long)(u * 8 + trow) * RC + 2 * tsrc);
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) {
        double2 w = make_double2(c[u][t][0], c[u][t][1]);
        if (ADD) {
          const double2 cur = o[t * 4];
          w.x += cur.x;
          w.y += cur.y;
        }
        o[t * 4] = w;
      }
    }
  }
}

// M2L from the stored FP64 blocks (the same blocks the FP64 path applies)
// with FP64 tensor-core tiles: one warp per chunk of up to kChunkRows skeleton
// rows of one box, i.e. NT <= 5 tiles of 8 rows that share every B fragment.
// The 40 slots' rank and skeleton offset are fetched once per warp and
// broadcast by shuffles; the box's contiguous block region is streamed into
// L2 ahead of the loads.
template <int RC, int NT, bool Q32>
__device__ __forceinline__ void m2l_stored_chunk(const LevelView& v, const double* __restrict__ qh,
                                                 double* __restrict__ yb, int b, int r0, int lane, uint32_t ahead) {
  const int r = v.rank[b];
  const int i0 = r0 - v.skel_off[b];
  const int nrow = min(8 * NT, r - i0);
  const int trow = lane >> 2, tsrc = lane & 3;
  // slot table: lane l holds slot l (and slot 32 + l for l < 8)
  const int sa = v.il[(long)b * 40 + lane];
  const int sb = lane < 8 ? v.il[(long)b * 40 + 32 + lane] : -1;
  const int ra = sa >= 0 ? v.rank[sa] : 0, rb = sb >= 0 ? v.rank[sb] : 0;
  const int oa = sa >= 0 ? v.skel_off[sa] : 0, ob = sb >= 0 ? v.skel_off[sb] : 0;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + trow < nrow;
  long pos = v.m2l_off[b];  // first entry of the current slot's block
  const long stop = v.m2l_off[b + 1];
  L2Stream pf(Q32 ? (const void*)(v.m2l_q + pos) : (const void*)(v.m2l + pos),
              Q32 ? (const void*)(v.m2l_q + stop) : (const void*)(v.m2l + stop), ahead);
  double c[NT][RC / 8][2];
  zero_tiles<RC, NT>(c);
  for (int s = 0; s < 40; ++s) {
    const int rc = __shfl_sync(0xffffffffu, s < 32 ? ra : rb, s & 31);
    if (rc == 0) continue;  // empty slot or rank-0 box: no block stored
    const int sc = __shfl_sync(0xffffffffu, s < 32 ? oa : ob, s & 31);
    if (Q32) {
      pf.advance(v.m2l_q + pos, lane);
      mma_rows_q32<RC, NT>(c, v.m2l_q + pos + i0 + trow, r, rc, v.m2l_dec[(long)b * 40 + s], qh + (long)sc * RC,
                           rowok, trow, tsrc);
    } else {
      pf.advance(v.m2l + pos, lane);
      mma_rows<RC, NT>(c, v.m2l + pos + i0 + trow, r, rc, qh + (long)sc * RC, rowok, trow, tsrc);
    }
    pos += (long)r * rc;
  }
  store_tiles<RC, NT, false>(c, yb + (long)r0 * RC, rowok, trow, tsrc);
}

// m2l_stored_chunk for 16 columns in transposed form on m16n8k4 tiles:
// yhat^T (16 columns x rows) += qhat_c^T (16 x r_c) M^T (r_c x rows), so the
// 16 right-hand sides fill the tile's M dimension without padding and the
// chunk's rows (NT tiles of 8) are the N dimension; half the MMA
// instructions of the 8x8x4 form for the same products.  Same block reads,
// same per-box L2 streaming.
template <int NT, bool Q32>
__device__ __forceinline__ void m2l_stored_chunk_t16(const LevelView& v, const double* __restrict__ qh,
                                                     double* __restrict__ yb, int b, int r0, int lane,
                                                     uint32_t ahead) {
  constexpr int RC = 16;
  const int r = v.rank[b];
  const int i0 = r0 - v.skel_off[b];
  const int nrow = min(8 * NT, r - i0);
  const int g = lane >> 2, t = lane & 3;
  const int sa = v.il[(long)b * 40 + lane];
  const int sb = lane < 8 ? v.il[(long)b * 40 + 32 + lane] : -1;
  const int ra = sa >= 0 ? v.rank[sa] : 0, rb = sb >= 0 ? v.rank[sb] : 0;
  const int oa = sa >= 0 ? v.skel_off[sa] : 0, ob = sb >= 0 ? v.skel_off[sb] : 0;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + g < nrow;
  long pos = v.m2l_off[b];
  const long stop = v.m2l_off[b + 1];
  L2Stream pf(Q32 ? (const void*)(v.m2l_q + pos) : (const void*)(v.m2l + pos),
              Q32 ? (const void*)(v.m2l_q + stop) : (const void*)(v.m2l + stop), ahead);
  double c[NT][4];
#pragma unroll
  for (int u = 0; u < NT; ++u) c[u][0] = c[u][1] = c[u][2] = c[u][3] = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int rc = __shfl_sync(0xffffffffu, s < 32 ? ra : rb, s & 31);
    if (rc == 0) continue;
    const int sc = __shfl_sync(0xffffffffu, s < 32 ? oa : ob, s & 31);
    const double* qb = qh + (long)sc * RC + g;
    double2 dec = make_double2(0.0, 0.0);
    if (Q32) {
      dec = v.m2l_dec[(long)b * 40 + s];
      pf.advance(v.m2l_q + pos, lane);
    } else {
      pf.advance(v.m2l + pos, lane);
    }
    const double* M = v.m2l + pos + i0 + g;
    const uint32_t* MQ = v.m2l_q + pos + i0 + g;
#pragma unroll 4
    for (int k0 = 0; k0 < rc; k0 += 4) {
      const int k = k0 + t;
      const bool vk = k < rc;
      const double a0 = vk ? qb[(long)k * RC] : 0.0;
      const double a1 = vk ? qb[(long)k * RC + 8] : 0.0;
      double bm[NT];
      if (Q32) {
        uint32_t uq[NT];
#pragma unroll
        for (int u = 0; u < NT; ++u) uq[u] = (vk && rowok[u]) ? MQ[(long)k * r + u * 8] : 0x80000000u;
#pragma unroll
        for (int u = 0; u < NT; ++u) bm[u] = decode_q32(uq[u], dec);
      } else {
#pragma unroll
        for (int u = 0; u < NT; ++u) bm[u] = (vk && rowok[u]) ? M[(long)k * r + u * 8] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < NT; ++u) mma_f64_16x8x4(c[u], a0, a1, bm[u]);
    }
    pos += (long)r * rc;
  }
  // D^T[col][row]: lane holds columns g, g + 8 of rows 2t, 2t + 1 of each tile
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    const int row = u * 8 + 2 * t;
    double* o = yb + (long)(r0 + row) * RC + g;
    if (row < nrow) {
      o[0] = c[u][0];
      o[8] = c[u][2];
    }
    if (row + 1 < nrow) {
      o[RC] = c[u][1];
      o[RC + 8] = c[u][3];
    }
  }
}

// M2M on FP64 tensor-core tiles: qhat rows of box b = L2P_b^T src_b, one warp
// per chunk of up to kChunkRows skeleton rows (the row-major L2P copy is the
// column-major A with lda = rank).
template <int RC, int NT>
__device__ __forceinline__ void m2m_chunk(const LevelView& v, const double* __restrict__ src_all, int leaf,
                                          double* __restrict__ qhat, int b, int r0, int lane) {
  const int r = v.rank[b];
  const int i0 = r0 - v.skel_off[b];
  const int nrow = min(8 * NT, r - i0);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int trow = lane >> 2, tsrc = lane & 3;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + trow < nrow;
  const double* src = src_all + (long)(leaf ? v.leaf_start[b] : v.node_off[b]) * RC;
  // the box's L2P block and source rows are read once, in order: bring
  // them into L2 up front
  prefetch_l2_region(v.l2p_rm + v.l2p_off[b], v.l2p_rm + v.l2p_off[b + 1], lane);
  prefetch_l2_region(src, src + (long)n * RC, lane);
  double c[NT][RC / 8][2];
  zero_tiles<RC, NT>(c);
  mma_rows<RC, NT>(c, v.l2p_rm + v.l2p_off[b] + i0 + trow, r, n, src, rowok, trow, tsrc);
  store_tiles<RC, NT, false>(c, qhat + (long)r0 * RC, rowok, trow, tsrc);
}

// L2L on FP64 tensor-core tiles: node rows of box b get L2P_b yhat_b, added
// to the child's incoming potential, or written as the leaf potential; one
// warp per chunk of up to kChunkRows node rows.
template <int RC, int NT>
__device__ __forceinline__ void l2l_chunk(const LevelView& v, const double* __restrict__ yhat,
                                          double* __restrict__ child_yhat, double* __restrict__ ys, int leaf, int b,
                                          int g0, int lane) {
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int i0 = g0 - v.node_off[b];
  const int nrow = min(8 * NT, n - i0);
  const int trow = lane >> 2, tsrc = lane & 3;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + trow < nrow;
  prefetch_l2_region(v.l2p + v.l2p_off[b] + (long)i0, v.l2p + v.l2p_off[b + 1], lane);
  double c[NT][RC / 8][2];
  zero_tiles<RC, NT>(c);
  mma_rows<RC, NT>(c, v.l2p + v.l2p_off[b] + i0 + trow, n, r, yhat + (long)v.skel_off[b] * RC, rowok, trow, tsrc);
  if (leaf)
    store_tiles<RC, NT, false>(c, ys + (long)(v.leaf_start[b] + i0) * RC, rowok, trow, tsrc);
  else
    store_tiles<RC, NT, true>(c, child_yhat + (long)g0 * RC, rowok, trow, tsrc);
}

// Number of 8-row tiles of a chunk: rows up to the next chunk's first row
// (the chunk tables cut boxes into equal chunks of at most kChunkRows rows).
__device__ __forceinline__ int chunk_tiles(const int32_t* chunk_first, long g, long nchunks, int box_end) {
  const int next = g + 1 < nchunks ? min(box_end, chunk_first[g + 1]) : box_end;
  return (next - chunk_first[g] + 7) >> 3;
}

#define AFMM_NT_SWITCH(nt, CALL) \
  switch (nt) {                  \
    case 1: CALL(1); break;      \
    case 2: CALL(2); break;      \
    case 3: CALL(3); break;      \
    case 4: CALL(4); break;      \
    default: CALL(5); break;     \
  }

template <int RC>
__global__ void __launch_bounds__(128) k_m2m_mma(LevelView v, const double* __restrict__ src_all, int leaf,
                                                 double* __restrict__ qhat) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= v.ncgroups) return;  // whole warps only
  const int b = v.cgrp_box[g];
  const int r0 = v.cgrp_row[g];
#define AFMM_M2M(NT) m2m_chunk<RC, NT>(v, src_all, leaf, qhat, b, r0, lane)
  AFMM_NT_SWITCH(chunk_tiles(v.cgrp_row, g, v.ncgroups, v.skel_off[b] + v.rank[b]), AFMM_M2M)
#undef AFMM_M2M
}

template <int RC>
__global__ void __launch_bounds__(128) k_l2l_mma(LevelView v, const double* __restrict__ yhat,
                                                 double* __restrict__ child_yhat, double* __restrict__ ys, int leaf) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= v.nncgroups) return;  // whole warps only
  const int b = v.ncgrp_box[g];
  const int g0 = v.ncgrp_row[g];
#define AFMM_L2L(NT) l2l_chunk<RC, NT>(v, yhat, child_yhat, ys, leaf, b, g0, lane)
  AFMM_NT_SWITCH(chunk_tiles(v.ncgrp_row, g, v.nncgroups, v.node_off[b + 1]), AFMM_L2L)
#undef AFMM_L2L
}

// Sweeps of the levels with few boxes, split along K: a CTA of S warps per
// chunk, warp w multiplying the w-th share of the chunk's K range (node rows
// for M2M, the box's rank for L2L); the partial tiles meet in shared memory
// and are added in warp order, so the result does not depend on scheduling.
// The upper levels have a handful of boxes whose K loops are the longest of
// the tree: one warp per chunk would leave most SMs idle.

// Warps per chunk for a level of `chunks` chunks (0: one warp per chunk, the
// unsplit kernels).  M2M's K (the children's ranks) is several times L2L's
// (the box's own rank), so M2M splits more levels.
inline int split_warps(long chunks, bool m2m) {
  if (chunks < 2048) return 8;
  if (m2m && chunks < 8192) return 8;
  if (m2m && chunks < 32768) return 2;
  return 0;
}

// Shared doubles of the partial tiles of a CTA (the largest chunk, 5 tiles):
// [warp][tile][column tile][fragment][lane].
template <int RC, int S>
constexpr int split_part_doubles() {
  return S * 5 * (RC / 8) * 2 * 32;
}

template <int RC, int NT, int S, bool ADD>
__device__ __forceinline__ void split_reduce_store(double (&c)[NT][RC / 8][2], double* __restrict__ part,
                                                   double* __restrict__ out, const bool (&rowok)[NT], int trow,
                                                   int tsrc, int w, int lane) {
  constexpr int kTile = (RC / 8) * 2 * 32;
#pragma unroll
  for (int u = 0; u < NT; ++u)
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) {
      part[(w * NT + u) * kTile + (t * 2) * 32 + lane] = c[u][t][0];
      part[(w * NT + u) * kTile + (t * 2 + 1) * 32 + lane] = c[u][t][1];
    }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) {
        double s0 = part[u * kTile + (t * 2) * 32 + lane], s1 = part[u * kTile + (t * 2 + 1) * 32 + lane];
        for (int x = 1; x < S; ++x) {
          s0 += part[(x * NT + u) * kTile + (t * 2) * 32 + lane];
          s1 += part[(x * NT + u) * kTile + (t * 2 + 1) * 32 + lane];
        }
        c[u][t][0] = s0;
        c[u][t][1] = s1;
      }
    store_tiles<RC, NT, ADD>(c, out, rowok, trow, tsrc);
  }
}

// K share [kb, ke) of warp w of S out of K, in multiples of 4.
template <int S>
__device__ __forceinline__ void split_range(int K, int w, int& kb, int& ke) {
  const int per = ((K + 4 * S - 1) / (4 * S)) * 4;
  kb = min(K, w * per);
  ke = min(K, kb + per);
}

template <int RC, int NT, int S>
__device__ __forceinline__ void m2m_chunk_split(const LevelView& v, const double* __restrict__ src_all, int leaf,
                                                double* __restrict__ qhat, int b, int r0, int w, int lane,
                                                double* part) {
  const int r = v.rank[b];
  const int i0 = r0 - v.skel_off[b];
  const int nrow = min(8 * NT, r - i0);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int trow = lane >> 2, tsrc = lane & 3;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + trow < nrow;
  int kb, ke;
  split_range<S>(n, w, kb, ke);
  const double* src = src_all + (long)(leaf ? v.leaf_start[b] : v.node_off[b]) * RC;
  const double* A = v.l2p_rm + v.l2p_off[b] + (long)kb * r;
  prefetch_l2_region(A, A + (long)(ke - kb) * r, lane);
  prefetch_l2_region(src + (long)kb * RC, src + (long)ke * RC, lane);
  double c[NT][RC / 8][2];
  zero_tiles<RC, NT>(c);
  mma_rows<RC, NT>(c, A + i0 + trow, r, ke - kb, src + (long)kb * RC, rowok, trow, tsrc);
  split_reduce_store<RC, NT, S, false>(c, part, qhat + (long)r0 * RC, rowok, trow, tsrc, w, lane);
}

template <int RC, int NT, int S>
__device__ __forceinline__ void l2l_chunk_split(const LevelView& v, const double* __restrict__ yhat,
                                                double* __restrict__ child_yhat, double* __restrict__ ys, int leaf,
                                                int b, int g0, int w, int lane, double* part) {
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int i0 = g0 - v.node_off[b];
  const int nrow = min(8 * NT, n - i0);
  const int trow = lane >> 2, tsrc = lane & 3;
  bool rowok[NT];
#pragma unroll
  for (int u = 0; u < NT; ++u) rowok[u] = u * 8 + trow < nrow;
  int kb, ke;
  split_range<S>(r, w, kb, ke);
  const double* A = v.l2p + v.l2p_off[b] + (long)kb * n;
  prefetch_l2_region(A + i0, A + (long)(ke - kb) * n, lane);
  double c[NT][RC / 8][2];
  zero_tiles<RC, NT>(c);
  mma_rows<RC, NT>(c, A + i0 + trow, n, ke - kb, yhat + (long)(v.skel_off[b] + kb) * RC, rowok, trow, tsrc);
  if (leaf)
    split_reduce_store<RC, NT, S, false>(c, part, ys + (long)(v.leaf_start[b] + i0) * RC, rowok, trow, tsrc, w,
                                         lane);
  else
    split_reduce_store<RC, NT, S, true>(c, part, child_yhat + (long)g0 * RC, rowok, trow, tsrc, w, lane);
}

template <int RC, int S>
__global__ void __launch_bounds__(32 * S) k_m2m_mma_split(LevelView v, const double* __restrict__ src_all, int leaf,
                                                          double* __restrict__ qhat) {
  __shared__ double part[split_part_doubles<RC, S>()];
  const long g = blockIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = v.cgrp_box[g];
  const int r0 = v.cgrp_row[g];
#define AFMM_M2M(NT) m2m_chunk_split<RC, NT, S>(v, src_all, leaf, qhat, b, r0, w, lane, part)
  AFMM_NT_SWITCH(chunk_tiles(v.cgrp_row, g, v.ncgroups, v.skel_off[b] + v.rank[b]), AFMM_M2M)
#undef AFMM_M2M
}

template <int RC, int S>
__global__ void __launch_bounds__(32 * S) k_l2l_mma_split(LevelView v, const double* __restrict__ yhat,
                                                          double* __restrict__ child_yhat, double* __restrict__ ys,
                                                          int leaf) {
  __shared__ double part[split_part_doubles<RC, S>()];
  const long g = blockIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = v.ncgrp_box[g];
  const int g0 = v.ncgrp_row[g];
#define AFMM_L2L(NT) l2l_chunk_split<RC, NT, S>(v, yhat, child_yhat, ys, leaf, b, g0, w, lane, part)
  AFMM_NT_SWITCH(chunk_tiles(v.ncgrp_row, g, v.nncgroups, v.node_off[b + 1]), AFMM_L2L)
#undef AFMM_L2L
}

template <int RC, bool Q32>
__global__ void __launch_bounds__(128) k_m2l_stored_mma(LevelSet ls, const double* const* __restrict__ qhat_lv,
                                                        double* const* __restrict__ yhat_lv) {
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= ls.cgrp0[ls.nlev]) return;  // whole warps only
  int j = 0;
  while (j + 1 < ls.nlev && gw >= ls.cgrp0[j + 1]) ++j;
  const LevelView& v = ls.lv[j];
  const long g = gw - ls.cgrp0[j];
  const int b = v.cgrp_box[g];
  const int r0 = v.cgrp_row[g];
#define AFMM_M2L(NT) m2l_stored_chunk<RC, NT, Q32>(v, qhat_lv[ls.src[j]], yhat_lv[ls.src[j]], b, r0, lane, ls.pf_ahead)
  AFMM_NT_SWITCH(chunk_tiles(v.cgrp_row, g, v.ncgroups, v.skel_off[b] + v.rank[b]), AFMM_M2L)
#undef AFMM_M2L
}

template <bool Q32>
__global__ void __launch_bounds__(128) k_m2l_stored_mma_t16(LevelSet ls, const double* const* __restrict__ qhat_lv,
                                                            double* const* __restrict__ yhat_lv) {
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= ls.cgrp0[ls.nlev]) return;  // whole warps only
  int j = 0;
  while (j + 1 < ls.nlev && gw >= ls.cgrp0[j + 1]) ++j;
  const LevelView& v = ls.lv[j];
  const long g = gw - ls.cgrp0[j];
  const int b = v.cgrp_box[g];
  const int r0 = v.cgrp_row[g];
#define AFMM_M2L(NT) m2l_stored_chunk_t16<NT, Q32>(v, qhat_lv[ls.src[j]], yhat_lv[ls.src[j]], b, r0, lane, ls.pf_ahead)
  AFMM_NT_SWITCH(chunk_tiles(v.cgrp_row, g, v.ncgroups, v.skel_off[b] + v.rank[b]), AFMM_M2L)
#undef AFMM_M2L
}

inline int nbk(long n, int t) { return (int)((n + t - 1) / t); }

// Streaming multiprocessors of the current device.
inline int sm_count() {
  int dev = 0, n = 0;
  AFMM_CUDA(cudaGetDevice(&dev));
  AFMM_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

template <int RC>
struct Pass {
  static_assert(RC == 8 || RC == 16, "passes of 8 or 16 columns (tensor-core tiles)");
  // M2L of every level: the stored blocks (fixed point in mixed precision,
  // FP64 otherwise; kernel-independent), or the entries on the fly (the
  // kernel's table)
  // (the levels of the tuning mask, in mixed precision, on the fly as well)
  static int m2l(const MatvecPlan& p, const double* const* qh, double* const* yh, int fp64, int* err,
                 cudaStream_t s) {
    if (p.levels.row0[p.levels.nlev] == 0) return 0;  // every box of ACA rank 0: no far field
    const bool q32 = !fp64 && p.levels.lv[0].m2l_q != nullptr;
    const bool stored = q32 || p.levels.lv[0].m2l != nullptr;
    const uint32_t otf = !stored ? 0xffffffffu : (fp64 ? 0u : p.tune.otf_batched);
    LevelSet st = level_subset(p.levels_m2l, otf, false);  // a shard's boxes at the sharded levels
    const LevelSet fly = level_subset(p.levels, otf, true);
    st.pf_ahead = p.tune.pf_batched;
    int n = 0;
    if (st.nlev > 0 && st.cgrp0[st.nlev] > 0) {
      // stored blocks: one HBM read of the blocks serves all RC columns
      // (mixed precision: the 32-bit fixed-point copy, half the bytes)
      const long warps = st.cgrp0[st.nlev];
      if (RC == 16 && q32 && p.tune.m2l_tc == 2 && err && st.lv[0].m2l_s != nullptr) {
        // exact integer products on tcgen05: the charges' byte planes of this
        // pass, then persistent CTAs over the 128-row tiles
        using namespace m2l_i8_detail;
        const long nb = st.b0[st.nlev];
        k_qhat_slice<<<nbk(nb * 32, 128), 128, 0, s>>>(st, qh);
        AFMM_LAUNCH_CHECK();
        ++n;
        allow_smem(k_m2l_i8, kSmem);
        const long items = st.t0[st.nlev];
        const int grid = (int)std::min<long>(items, 2L * sm_count());
        if (grid > 0) k_m2l_i8<<<grid, kThreads, kSmem, s>>>(st, yh, err);
      } else if (RC == 16 && q32 && p.tune.m2l_tc == 1 && err) {
        // tcgen05 TF32 tiles, one CTA per row tile of a parent's children
        allow_smem(m2l_tc_detail::k_m2l_tc, m2l_tc_detail::kSmem);
        m2l_tc_detail::k_m2l_tc<<<(int)st.pt0[st.nlev], m2l_tc_detail::kThreads, m2l_tc_detail::kSmem, s>>>(st, qh, yh,
                                                                                                          err);
      } else if (RC == 16 && p.tune.m2l_t16) {
        if (q32) k_m2l_stored_mma_t16<true><<<nbk(warps * 32, 128), 128, 0, s>>>(st, qh, yh);
        else k_m2l_stored_mma_t16<false><<<nbk(warps * 32, 128), 128, 0, s>>>(st, qh, yh);
      } else if (q32) {
        k_m2l_stored_mma<RC, true><<<nbk(warps * 32, 128), 128, 0, s>>>(st, qh, yh);
      } else {
        k_m2l_stored_mma<RC, false><<<nbk(warps * 32, 128), 128, 0, s>>>(st, qh, yh);
      }
      AFMM_LAUNCH_CHECK();
      ++n;
    }
    if (fly.nlev > 0 && fly.row0[fly.nlev] > 0) {
      kernel_table(p.kp.id).m2l_otf_mma[RC == 16](fly, p.kp, qh, yh, s);
      ++n;
    }
    return n;
  }

  // Near field of the pass: the mixed 16-column form on tcgen05 tiles when
  // tuned so (leaves of at most 64 points), else mma.sync tiles (TF32x3 in
  // mixed precision, FP64 in FP64-batched passes).
  // (adds into ys_out)
  static void p2p(const MatvecPlan& p, BatchState& bs, const NearView& nv, int fp64, cudaStream_t s,
                  double* ys_out = nullptr) {
    const KernelTable& kt = kernel_table(p.kp.id);
    double* ys = ys_out ? ys_out : bs.ys;
    if (RC == 16 && !fp64 && p.tune.p2p_tc && nv.nmax <= 64 && bs.err_dev) {
      kt.p2p_tc16(nv, p.kp, bs.qhl, ys, p.L, bs.err_dev, s);
    } else if (fp64) {
      kt.p2p_dmma[RC == 16](nv, p.kp, bs.qs, ys, s);
    } else {
      kt.p2p_mma[RC == 16](nv, p.kp, bs.qhl, ys, s);
    }
  }

  static void run(const MatvecPlan& p, BatchState& bs, const NearView& nv, const double* q, int64_t ldq, double* y,
                  int64_t ldy, int ncols, int fp64, cudaStream_t s, StageTimer* tm, int64_t* launches) {
    const int N = p.N;
    if (p.shard_count > 1) {  // points outside the shard's leaves come out as zeros
      AFMM_CUDA(cudaMemsetAsync(bs.ys, 0, sizeof(double) * (size_t)N * RC, s));
    }
    if (tm) tm->mark(s, "gather");
    k_gather_b<RC><<<nbk(N, kTileJ), 256, 0, s>>>(q, ldq, ncols, p.iperm, N, bs.qs, bs.qhl, fp64);
    AFMM_LAUNCH_CHECK();
    ++*launches;
    // the near field does not depend on the far field: it runs on its own
    // lower-priority stream into ys_near, filling what the far-field
    // kernels leave of the GPU (after the far field when profiling serially)
    const bool overlap = bs.s_near != nullptr && !(tm && tm->serial);
    if (overlap) {
      AFMM_CUDA(cudaEventRecord(bs.ev_q, s));
      AFMM_CUDA(cudaStreamWaitEvent(bs.s_near, bs.ev_q, 0));
      AFMM_CUDA(cudaMemsetAsync(bs.ys_near, 0, sizeof(double) * (size_t)N * RC, bs.s_near));
      const int sp = tm ? tm->span_begin(bs.s_near, "p2p_kernel") : -1;  // the kernel's own duration
      p2p(p, bs, nv, fp64, bs.s_near, bs.ys_near);
      if (tm) tm->span_end(bs.s_near, sp);
      AFMM_CUDA(cudaEventRecord(bs.ev_near, bs.s_near));
      ++*launches;
    }
    if (tm) tm->mark(s, "m2m");
    for (int j = p.L; j >= 2; --j) {
      const LevelView& v = p.lv[j];
      if (v.nrows == 0) continue;
      const double* src = j == p.L ? bs.qs : bs.qhat[j + 1];
      const int sw = split_warps(v.ncgroups, true);
      if (sw == 8)
        k_m2m_mma_split<RC, 8><<<(int)v.ncgroups, 256, 0, s>>>(v, src, j == p.L, bs.qhat[j]);
      else if (sw == 2)
        k_m2m_mma_split<RC, 2><<<(int)v.ncgroups, 64, 0, s>>>(v, src, j == p.L, bs.qhat[j]);
      else
        k_m2m_mma<RC><<<nbk(v.ncgroups * 32, 128), 128, 0, s>>>(v, src, j == p.L, bs.qhat[j]);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "m2l");
    *launches += m2l(p, bs.d_qhat_lv, bs.d_yhat_lv, fp64, bs.err_dev, s);
    if (tm) tm->mark(s, "l2l");
    for (int j = 2; j <= p.L; ++j) {
      const LevelView& v = p.lv_down[j];  // a shard's subtrees at the sharded levels
      if (v.nnodes == 0) continue;
      // the split follows the whole level, so a shard's rows get the same bits
      if (split_warps(p.lv[j].nncgroups, false) == 8)
        k_l2l_mma_split<RC, 8><<<(int)v.nncgroups, 256, 0, s>>>(v, bs.yhat[j], j < p.L ? bs.yhat[j + 1] : nullptr,
                                                                bs.ys, j == p.L);
      else
        k_l2l_mma<RC><<<nbk(v.nncgroups * 32, 128), 128, 0, s>>>(v, bs.yhat[j], j < p.L ? bs.yhat[j + 1] : nullptr,
                                                                bs.ys, j == p.L);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    // (overlapped: the "p2p" stage is the wait for the near field's end)
    if (tm) tm->mark(s, "p2p");
    if (overlap) {
      AFMM_CUDA(cudaStreamWaitEvent(s, bs.ev_near, 0));
    } else {
      p2p(p, bs, nv, fp64, s);
      ++*launches;
    }
    if (tm) tm->mark(s, "scatter");
    k_scatter_b<RC><<<nbk(N, kTileJ), 256, 0, s>>>(bs.ys, overlap ? bs.ys_near : nullptr, p.iperm, N, ncols, y, ldy);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
};

}  // namespace

int p2p_batched(const MatvecPlan& p, MixedState& ms, BatchState& bs, int rc, int fp64, cudaStream_t s) {
  NearView nv = p.near;
  nv.anchor = ms.leaf_anchor;
  nv.rel = ms.rel;
  nv.span = ms.leaf_span;
  if (rc == 16) Pass<16>::p2p(p, bs, nv, fp64, s);
  else Pass<8>::p2p(p, bs, nv, fp64, s);
  return 1;
}

void m2l_slice(const LevelView& v, cudaStream_t s) {
  if (v.nbox == 0) return;
  m2l_i8_detail::k_m2l_slice<<<(int)v.nbox, 256, 0, s>>>(v);
  AFMM_LAUNCH_CHECK();
}

int m2l_batched(const MatvecPlan& p, BatchState& bs, int rc, int fp64, cudaStream_t s) {
  if (rc == 16) return Pass<16>::m2l(p, bs.d_qhat_lv, bs.d_yhat_lv, fp64, bs.err_dev, s);
  return Pass<8>::m2l(p, bs.d_qhat_lv, bs.d_yhat_lv, fp64, bs.err_dev, s);
}

void batch_reserve(const MatvecPlan& p, BatchState& bs, DevArena& arena, cudaStream_t s) {
  if (bs.ready) return;
  const int RC = kBatchMax;
  bs.qs = arena.alloc<double>((size_t)p.N * RC);
  bs.qhl = arena.alloc<uint2>((size_t)p.N * RC);  // TF32 parts of the mixed near field
  bs.ys = arena.alloc<double>((size_t)p.N * RC);
  std::vector<const double*> hq(kMaxLevels, nullptr);
  std::vector<double*> hy(kMaxLevels, nullptr);
  for (int j = 2; j <= p.L; ++j) {
    bs.qhat[j] = arena.alloc<double>((size_t)std::max<long>(p.lv[j].nrows, 1) * RC);
    bs.yhat[j] = arena.alloc<double>((size_t)std::max<long>(p.lv[j].nrows, 1) * RC);
  }
  for (int t = 0; t < p.levels.nlev; ++t) {
    hq[t] = bs.qhat[t + 2];
    hy[t] = bs.yhat[t + 2];
  }
  bs.ys_near = arena.alloc<double>((size_t)p.N * RC);
  int least = 0, greatest = 0;  // the near field's stream at the lowest priority
  AFMM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  AFMM_CUDA(cudaStreamCreateWithPriority(&bs.s_near, cudaStreamNonBlocking, least));
  AFMM_CUDA(cudaEventCreateWithFlags(&bs.ev_q, cudaEventDisableTiming));
  AFMM_CUDA(cudaEventCreateWithFlags(&bs.ev_near, cudaEventDisableTiming));
  AFMM_CUDA(cudaHostAlloc((void**)&bs.err_host, sizeof(int), cudaHostAllocMapped));
  *bs.err_host = 0;
  AFMM_CUDA(cudaHostGetDevicePointer((void**)&bs.err_dev, bs.err_host, 0));
  bs.d_qhat_lv = arena.alloc<const double*>(kMaxLevels);
  bs.d_yhat_lv = arena.alloc<double*>(kMaxLevels);
  AFMM_CUDA(cudaMemcpyAsync((void*)bs.d_qhat_lv, hq.data(), sizeof(double*) * kMaxLevels, cudaMemcpyHostToDevice, s));
  AFMM_CUDA(cudaMemcpyAsync((void*)bs.d_yhat_lv, hy.data(), sizeof(double*) * kMaxLevels, cudaMemcpyHostToDevice, s));
  AFMM_CUDA(cudaStreamSynchronize(s));
  bs.ready = true;
}

void matvec_batched(const MatvecPlan& p, MixedState& ms, BatchState& bs, const double* q, int64_t ldq, double* y,
                    int64_t ldy, int nrhs, int fp64, cudaStream_t s, StageTimer* tm, int64_t* launches) {
  if (!ms.ready || !bs.ready) throw Error{AFMM_BAD_ARG, "batched operators are not set up"};
  NearView nv = p.near_own;
  nv.anchor = ms.leaf_anchor;
  nv.rel = ms.rel;
  nv.span = ms.leaf_span;
  for (int c0 = 0; c0 < nrhs;) {
    const int left = nrhs - c0;
    // passes of 8 or 16 columns (tensor-core tiles; unused columns are zero):
    // a pass of 8 costs less than a 4-column FMA pass would (measured at the
    // 4,194,304-point mixture: 6.7 against 10.9 ms)
    const int rc = left > 8 ? 16 : 8;
    const int nc = std::min(left, rc);
    const double* qc = q + (long)c0 * ldq;
    double* yc = y + (long)c0 * ldy;
    if (rc == 16) Pass<16>::run(p, bs, nv, qc, ldq, yc, ldy, nc, fp64, s, tm, launches);
    else Pass<8>::run(p, bs, nv, qc, ldq, yc, ldy, nc, fp64, s, tm, launches);
    c0 += nc;
  }
}

}  // namespace afmm
