// K2 (interaction lists), K5 (M2L blocks) and the FP64 matvec sweeps
// K6-K10 (gather, M2M, M2L, L2L, near field, scatter).
#include <algorithm>

#include "afmm_internal.cuh"
#include "fmm.cuh"
#include "kernel_table.cuh"

namespace afmm {

// ----------------------------------------------------------------- lists
// Closed form of the reference's parent-to-child recurrence
// (src/AFMM2DTree.cpp:65-967).  Box k at level j sits at grid cell (ix, iy)
// whose bits are the base-4 digits of k read as child offsets
// 0:(0,0) 1:(1,0) 2:(1,1) 3:(0,1) (src/AFMM2DTree.cpp:978-986).  Slot s of
// ring m (m = 1 neighbours N0..N7, 2 inner I0..I15, 3 outer O0..O23) is the
// cell at the s-th offset counter-clockwise around the ring starting at
// (-m,-m).  It is set when the cell is inside the domain and, for ring 3,
// when its parent neighbours the box's parent (the recurrence only visits the
// children of the parent's neighbours).
__device__ __forceinline__ void ring_offset(int m, int s, int& dx, int& dy) {
  const int side = 2 * m, seg = s / side, t = s % side;
  if (seg == 0) { dx = -m + t; dy = -m; }
  else if (seg == 1) { dx = m; dy = -m + t; }
  else if (seg == 2) { dx = m - t; dy = m; }
  else { dx = -m; dy = m - t; }
}

// One thread per (box, slot of the 48 ring slots).
__global__ void k_lists(int j, long nbox, int32_t* nbr, int32_t* il) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbox * 48) return;
  long k = t / 48;
  int s = (int)(t % 48);
  int m = s < 8 ? 1 : (s < 24 ? 2 : 3);
  int ss = s < 8 ? s : (s < 24 ? s - 8 : s - 24);
  int ix, iy, dx, dy;
  cell_of(k, j, ix, iy);
  ring_offset(m, ss, dx, dy);
  const int side = 1 << j;
  int cx = ix + dx, cy = iy + dy;
  bool ok = cx >= 0 && cy >= 0 && cx < side && cy < side;
  if (ok && m == 3) ok = abs((cx >> 1) - (ix >> 1)) <= 1 && abs((cy >> 1) - (iy >> 1)) <= 1;
  int32_t v = ok ? (int32_t)box_of(cx, cy, j) : -1;
  if (m == 1) nbr[k * 8 + ss] = v;
  else il[k * 40 + (s - 8)] = v;  // inner 0..15 then outer 0..23
}

void build_lists(int j, long nbox, int32_t* nbr, int32_t* il, cudaStream_t s) {
  long n = nbox * 48;
  k_lists<<<(int)((n + 255) / 256), 256, 0, s>>>(j, nbox, nbr, il);
  AFMM_LAUNCH_CHECK();
}

__global__ void k_fill_box_map(const int32_t* __restrict__ off, long nbox, int32_t* map) {
  long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  for (int32_t t = off[b]; t < off[b + 1]; ++t) map[t] = (int32_t)b;
}

__global__ void k_invert_perm(const int64_t* __restrict__ perm, int n, int32_t* iperm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) iperm[perm[i]] = i;
}

__global__ void k_gather_points(const double2* __restrict__ pts, const int32_t* __restrict__ ids, long n,
                                double2* out) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = pts[ids[t]];
}

void gather_points(const double2* pts, const int32_t* ids, long n, double2* out, cudaStream_t s) {
  if (n == 0) return;
  k_gather_points<<<(int)((n + 255) / 256), 256, 0, s>>>(pts, ids, n, out);
  AFMM_LAUNCH_CHECK();
}

void invert_permutation(const int64_t* perm, int n, int32_t* iperm, cudaStream_t s) {
  k_invert_perm<<<(n + 255) / 256, 256, 0, s>>>(perm, n, iperm);
  AFMM_LAUNCH_CHECK();
}

void fill_box_map(const int32_t* off, long nbox, int32_t* map, cudaStream_t s) {
  k_fill_box_map<<<(int)((nbox + 255) / 256), 256, 0, s>>>(off, nbox, map);
  AFMM_LAUNCH_CHECK();
}

// ------------------------------------------------------------ M2L blocks
// (k_m2l_assemble, fmm_k.cuh)
void m2l_assemble(const LevelView& v, const KernelParams& kp, cudaStream_t s) {
  kernel_table(kp.id).m2l_assemble(v, kp, s);
}

// 32-bit fixed-point copy of the FP64 blocks: per block a power-of-two scale
// 2^k with max|M| * 2^-k in [2^30, 2^31), entries rounded to the nearest
// multiple of 2^k (absolute error <= 2^-31 max|M|) and stored offset by 2^31
// as unsigned.  A block whose largest entry is 0 or below 2^-960 decodes to
// zeros; a block holding a non-finite entry decodes to NaN (as the FP64
// blocks would propagate it).  One CTA per box.
__global__ void __launch_bounds__(256) k_m2l_compress(LevelView v) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  __shared__ double red[8];
  __shared__ double2 s_dec;
  const double* M = v.m2l + v.m2l_off[b];
  uint32_t* Q = v.m2l_q + v.m2l_off[b];
  long off = 0;
  for (int s = 0; s < 40; ++s) {
    const int c = v.il[b * 40 + s];
    const int rc = (c >= 0 && r > 0) ? v.rank[c] : 0;
    const long n = (long)r * rc;
    if (n == 0) {
      if (threadIdx.x == 0) v.m2l_dec[b * 40 + s] = make_double2(0.0, 0.0);
      continue;
    }
    double mx = 0.0;
    bool bad = false;
    for (long e = threadIdx.x; e < n; e += blockDim.x) {
      const double x = M[off + e];
      bad |= !isfinite(x);
      mx = fmax(mx, fabs(x));
    }
    if (bad) mx = __longlong_as_double(0x7ff0000000000000ll);  // +inf
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
      int ex = 0;
      frexp(m, &ex);  // m in [2^(ex-1), 2^ex)
      const int k = ex - 31;
      if (!isfinite(m)) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        s_dec = make_double2(nan, nan);
      } else if (m == 0.0 || k < -960) {
        s_dec = make_double2(0.0, 0.0);
      } else {
        const double sc = scalbn(1.0, k);
        s_dec = make_double2(sc, -(4503601774854144.0 * sc));  // 2^52 + 2^31
      }
      v.m2l_dec[b * 40 + s] = s_dec;
    }
    __syncthreads();
    const double2 dec = s_dec;
    const bool zero = !(dec.x != 0.0) || !isfinite(dec.x);
    int ex = 0;
    if (!zero) frexp(dec.x, &ex);
    const int k = ex - 1;  // dec.x = 2^k
    for (long e = threadIdx.x; e < n; e += blockDim.x) {
      uint32_t u = 0x80000000u;
      if (!zero) {
        long long t = llrint(scalbn(M[off + e], -k)) + 0x80000000ll;
        t = t < 0 ? 0 : (t > 0xffffffffll ? 0xffffffffll : t);
        u = (uint32_t)t;
      }
      Q[off + e] = u;
    }
    off += n;
    __syncthreads();
  }
}

void m2l_compress(const LevelView& v, cudaStream_t s) {
  k_m2l_compress<<<(int)v.nbox, 256, 0, s>>>(v);
  AFMM_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- sweeps
// qs[i] = q[perm[i]]  (src/AFMM2D.cpp:49-51)
__global__ void k_gather(const double* __restrict__ q, const int64_t* __restrict__ perm, int n, double* qs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) qs[i] = q[perm[i]];
}

// y[perm[i]] = ys[i]  (src/AFMM2D.cpp:61-63)
__global__ void k_scatter(const double* __restrict__ ys, const int64_t* __restrict__ perm, int n, double* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[perm[i]] = ys[i];
}

// Row-major copy of L2P (per box, r fastest) for the M2M sweep.
template <class T>
__global__ void k_l2p_transpose(LevelView v, const T* __restrict__ cm, T* rm) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  if (r == 0) return;
  const int n = v.node_off[b + 1] - v.node_off[b];
  const long o = v.l2p_off[b];
  for (int e = threadIdx.x; e < n * r; e += blockDim.x) {
    int i = e / r, c = e - i * r;
    rm[o + e] = cm[o + (long)c * n + i];
  }
}

void l2p_transpose(const LevelView& v, const double* cm, double* rm, cudaStream_t s) {
  k_l2p_transpose<double><<<(int)v.nbox, 256, 0, s>>>(v, cm, rm);
  AFMM_LAUNCH_CHECK();
}

// Level of flat warp chunk g of a LevelSet (wgrp0: prefix of chunk counts).
__device__ __forceinline__ int level_of_wchunk(const LevelSet& ls, long g) {
  int j = 0;
  while (j + 1 < ls.nlev && g >= ls.wgrp0[j + 1]) ++j;
  return j;
}

// M2L (src/AFMM2DTree.cpp:1156-1178) for every level in one launch, one warp
// per chunk of up to 32 skeleton rows of one box, lane = row.  Each row's
// arithmetic is m2l_row's (slots in the reference's order, four partial sums
// per block), so the result has the same bits as the thread-per-row form; the
// warp's loads of one block column are contiguous, every lane of a warp
// takes the same slots, and the box's block region is streamed into L2 ahead
// of the loads.  Q32: the 32-bit fixed-point blocks (decode_q32) instead of
// the FP64 ones (the single-RHS mixed path).
template <bool Q32>
__global__ void __launch_bounds__(128) k_m2l_apply_w(LevelSet ls) {
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= ls.wgrp0[ls.nlev]) return;  // whole warps only
  const int j = level_of_wchunk(ls, gw);
  const LevelView& v = ls.lv[j];
  const long g = gw - ls.wgrp0[j];
  const int b = v.wgrp_box[g];
  const int r0 = v.wgrp_row[g];
  const int box_end = v.skel_off[b] + v.rank[b];
  const int next = g + 1 < v.nwgroups ? min(box_end, v.wgrp_row[g + 1]) : box_end;
  const int r = v.rank[b];
  const int i = r0 - v.skel_off[b] + lane;
  const bool act = lane < next - r0;
  // slot table: lane l holds slot l (and slot 32 + l for l < 8)
  const int sa = v.il[(long)b * 40 + lane];
  const int sb = lane < 8 ? v.il[(long)b * 40 + 32 + lane] : -1;
  const int ra = sa >= 0 ? v.rank[sa] : 0, rb = sb >= 0 ? v.rank[sb] : 0;
  const int oa = sa >= 0 ? v.skel_off[sa] : 0, ob = sb >= 0 ? v.skel_off[sb] : 0;
  const long base = v.m2l_off[b];
  const long stop = v.m2l_off[b + 1];
  long pos = base;  // first entry of the current slot's block
  L2Stream pf(Q32 ? (const void*)(v.m2l_q + base) : (const void*)(v.m2l + base),
              Q32 ? (const void*)(v.m2l_q + stop) : (const void*)(v.m2l + stop), ls.pf_ahead);
  double acc = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int rc = __shfl_sync(0xffffffffu, s < 32 ? ra : rb, s & 31);
    if (rc == 0) continue;  // empty slot or rank-0 box: no block stored
    const int sc = __shfl_sync(0xffffffffu, s < 32 ? oa : ob, s & 31);
    const double* qc = v.qhat + sc;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int cc = 0;
    if (Q32) {
      const double2 dec = v.m2l_dec[(long)b * 40 + s];
      pf.advance(v.m2l_q + pos, lane);
      const uint32_t* M = v.m2l_q + pos + i;
#define AFMM_ENT(c) (act ? decode_q32(M[(long)(c) * r], dec) : 0.0)
#pragma unroll 2
      for (; cc + 3 < rc; cc += 4) {
        a0 += AFMM_ENT(cc) * qc[cc];
        a1 += AFMM_ENT(cc + 1) * qc[cc + 1];
        a2 += AFMM_ENT(cc + 2) * qc[cc + 2];
        a3 += AFMM_ENT(cc + 3) * qc[cc + 3];
      }
      for (; cc < rc; ++cc) a0 += AFMM_ENT(cc) * qc[cc];
#undef AFMM_ENT
    } else {
      pf.advance(v.m2l + pos, lane);
      const double* M = v.m2l + pos + i;
#define AFMM_ENT(c) (act ? M[(long)(c) * r] : 0.0)
#pragma unroll 2
      for (; cc + 3 < rc; cc += 4) {
        a0 += AFMM_ENT(cc) * qc[cc];
        a1 += AFMM_ENT(cc + 1) * qc[cc + 1];
        a2 += AFMM_ENT(cc + 2) * qc[cc + 2];
        a3 += AFMM_ENT(cc + 3) * qc[cc + 3];
      }
      for (; cc < rc; ++cc) a0 += AFMM_ENT(cc) * qc[cc];
#undef AFMM_ENT
    }
    acc += (a0 + a1) + (a2 + a3);
    pos += (long)r * rc;
  }
  if (act) v.yhat[r0 + lane] = acc;
}

// End of warp chunk g of a chunk table (the next chunk's first row, or the
// end of the box).
__device__ __forceinline__ int wchunk_end(const int32_t* first, long g, long n, int box_end) {
  return g + 1 < n ? min(box_end, first[g + 1]) : box_end;
}

// M2M (m2m_row's arithmetic, so the same bits) with one warp per chunk of up
// to 32 skeleton rows of one box: no warp straddles two boxes, and the box's
// L2P block and source rows are brought into L2 up front.
__global__ void __launch_bounds__(128) k_m2m_w(LevelView v, const double* __restrict__ src_all, int leaf) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= v.nwgroups) return;
  const int b = v.wgrp_box[g];
  const int r0 = v.wgrp_row[g];
  const int end = wchunk_end(v.wgrp_row, g, v.nwgroups, v.skel_off[b] + v.rank[b]);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (leaf ? v.leaf_start[b] : v.node_off[b]);
  prefetch_l2_region(v.l2p_rm + v.l2p_off[b], v.l2p_rm + v.l2p_off[b + 1], lane);
  prefetch_l2_region(src, src + n, lane);
  if (r0 + lane < end) m2m_row(v, src_all, leaf, r0 + lane);
}

// L2L (l2l_row's arithmetic) with one warp per chunk of up to 32 node rows of
// one box, the box's L2P block brought into L2 up front.
__global__ void __launch_bounds__(128) k_l2l_w(LevelView v, double* __restrict__ child_yhat, double* __restrict__ ys,
                                               int leaf) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= v.nnwgroups) return;
  const int b = v.nwgrp_box[g];
  const int g0 = v.nwgrp_row[g];
  const int end = wchunk_end(v.nwgrp_row, g, v.nnwgroups, v.node_off[b + 1]);
  prefetch_l2_region(v.l2p + v.l2p_off[b] + (g0 - v.node_off[b]), v.l2p + v.l2p_off[b + 1], lane);
  if (g0 + lane < end) l2l_row(v, child_yhat, ys, leaf, g0 + lane);
}


void sweep_m2m(const MatvecPlan& p, const double* qs, cudaStream_t s, int64_t* launches) {
  for (int j = p.L; j >= 2; --j) {
    const LevelView& v = p.lv[j];
    if (v.nrows == 0) continue;
    k_m2m_w<<<(int)((v.nwgroups * 32 + 127) / 128), 128, 0, s>>>(v, j == p.L ? qs : p.lv[j + 1].qhat, j == p.L);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

void sweep_l2l(const MatvecPlan& p, double* ys, cudaStream_t s, int64_t* launches) {
  for (int j = 2; j <= p.L; ++j) {
    const LevelView& v = p.lv_down[j];  // a shard's subtrees at the sharded levels
    if (v.nnodes == 0) continue;
    k_l2l_w<<<(int)((v.nnwgroups * 32 + 127) / 128), 128, 0, s>>>(v, j < p.L ? p.lv[j + 1].yhat : nullptr, ys,
                                                                  j == p.L);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

void m2l_apply(const MatvecPlan& p, cudaStream_t s) {
  const long rows = p.levels.row0[p.levels.nlev];
  if (rows == 0) return;
  if (p.levels.lv[0].m2l == nullptr) {  // blocks not stored: entries on the fly
    m2l_apply_otf(p, p.levels, s);
    return;
  }
  LevelSet ls = p.levels_m2l;  // a shard's boxes at the sharded levels
  ls.pf_ahead = p.tune.pf_fp64;
  const long warps = ls.wgrp0[ls.nlev];
  k_m2l_apply_w<false><<<(int)((warps * 32 + 127) / 128), 128, 0, s>>>(ls);
  AFMM_LAUNCH_CHECK();
}

void m2l_apply_stored(const MatvecPlan& p, const LevelSet& levels, bool q32, cudaStream_t s) {
  LevelSet ls = levels;
  ls.pf_ahead = p.tune.pf_fp64;
  const long warps = ls.wgrp0[ls.nlev];
  if (warps == 0) return;
  if (q32 && ls.lv[0].m2l_q == nullptr) throw Error{AFMM_BAD_ARG, "no fixed-point M2L blocks stored"};
  if (!q32 && ls.lv[0].m2l == nullptr) throw Error{AFMM_BAD_ARG, "no M2L blocks stored"};
  if (q32) k_m2l_apply_w<true><<<(int)((warps * 32 + 127) / 128), 128, 0, s>>>(ls);
  else k_m2l_apply_w<false><<<(int)((warps * 32 + 127) / 128), 128, 0, s>>>(ls);
  AFMM_LAUNCH_CHECK();
}

void matvec_fp64(const MatvecPlan& p, const double* q, double* y, cudaStream_t s, StageTimer* tm, int64_t* launches) {
  const int N = p.N;
  const int gb = (N + 255) / 256;
  if (tm) tm->mark(s, "gather");
  if (p.shard_count > 1) AFMM_CUDA(cudaMemsetAsync(p.ys, 0, sizeof(double) * (size_t)N, s));
  k_gather<<<gb, 256, 0, s>>>(q, p.perm, N, p.qs);
  AFMM_LAUNCH_CHECK();
  ++*launches;
  if (tm) tm->mark(s, "m2m");
  sweep_m2m(p, p.qs, s, launches);
  if (tm) tm->mark(s, "m2l");
  m2l_apply(p, s);
  ++*launches;
  if (tm) tm->mark(s, "l2l");
  sweep_l2l(p, p.ys, s, launches);
  if (tm) tm->mark(s, "p2p");
  kernel_table(p.kp.id).p2p64(p.near_own, p.kp, p.qs, p.ys, s);
  ++*launches;
  if (tm) tm->mark(s, "scatter");
  k_scatter<<<gb, 256, 0, s>>>(p.ys, p.perm, N, y);
  AFMM_LAUNCH_CHECK();
  ++*launches;
  if (tm) tm->mark(s, "end");
}

}  // namespace afmm
