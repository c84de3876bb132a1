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

#include "mixed.cuh"

namespace afmm {

namespace {

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo with both parts TF32 (hi: 11 significant bits, lo: the next 11).
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// Gather through a shared-memory transpose: a block takes kTileJ consecutive
// points, reads each column of q as one contiguous run, and writes each
// point's sorted row qs[iperm[j]][0:RC] (one 128-byte line for RC = 16).
// With RC >= 8 the row is also written as interleaved TF32 high / low parts
// (the tensor-core near field's charges), otherwise as FP32; neither when the
// pass is FP64 throughout.
constexpr int kTileJ = 64;

template <int RC>
__global__ void __launch_bounds__(256) k_gather_b(const double* __restrict__ q, int64_t ldq, int ncols,
                                                  const int32_t* __restrict__ iperm, int N, double* qs, float* qs32,
                                                  uint2* qhl, int fp64_only) {
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
    const float f0 = (float)v0, f1 = (float)v1;
    if (RC >= 8) {
      uint4 hl;
      split_tf32(f0, hl.x, hl.y);
      split_tf32(f1, hl.z, hl.w);
      *reinterpret_cast<uint4*>(qhl + d) = hl;
    } else {
      *reinterpret_cast<float2*>(qs32 + d) = make_float2(f0, f1);
    }
  }
}

// Scatter through a shared-memory transpose: a block takes kTileJ consecutive
// points, reads their sorted rows ys[iperm[j]][0:RC], and writes each column
// of y as one contiguous run.
template <int RC>
__global__ void __launch_bounds__(256) k_scatter_b(const double* __restrict__ ys, const int32_t* __restrict__ iperm,
                                                   int N, int ncols, double* y, int64_t ldy) {
  __shared__ double tile[RC][kTileJ + 1];
  const long j0 = (long)blockIdx.x * kTileJ;
  for (int idx = threadIdx.x; idx < (RC / 2) * kTileJ; idx += blockDim.x) {
    const int jj = idx / (RC / 2), cp = idx % (RC / 2);
    const long j = j0 + jj;
    if (j >= N) continue;
    const double2 v = *reinterpret_cast<const double2*>(ys + (long)iperm[j] * RC + 2 * cp);
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

template <int RC>
__device__ __forceinline__ void load_vec(const double* __restrict__ p, double (&v)[RC]) {
  const double2* p2 = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int c = 0; c < RC / 2; ++c) {
    double2 t = p2[c];
    v[2 * c] = t.x;
    v[2 * c + 1] = t.y;
  }
}

template <int RC>
__device__ __forceinline__ void store_vec(double* p, const double (&v)[RC]) {
  double2* p2 = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int c = 0; c < RC / 2; ++c) p2[c] = make_double2(v[2 * c], v[2 * c + 1]);
}

// M2M: one thread per output row; qhat[row] = sum_i L2P[i][c] src[i].
template <int RC>
__global__ void k_m2m_b(LevelView v, const double* __restrict__ src_all, int leaf, double* qhat) {
  const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= v.nrows) return;
  const int b = v.skel_box[row];
  const int r = v.rank[b];
  const int c = (int)(row - v.skel_off[b]);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (long)(leaf ? v.leaf_start[b] : v.node_off[b]) * RC;
  const double* P = v.l2p_rm + v.l2p_off[b] + c;
  double acc[RC];
#pragma unroll
  for (int k = 0; k < RC; ++k) acc[k] = 0.0;
  for (int i = 0; i < n; ++i) {
    const double p = P[(long)i * r];
    double s[RC];
    load_vec<RC>(src + (long)i * RC, s);
#pragma unroll
    for (int k = 0; k < RC; ++k) acc[k] = fma(p, s[k], acc[k]);
  }
  store_vec<RC>(qhat + row * RC, acc);
}

// M2L on the fly (FP64 entries), one thread per skeleton row of every level.
template <class K, int RC>
__global__ void k_m2l_b(LevelSet ls, KernelParams kp, const double* const* __restrict__ qhat_lv,
                        double* const* __restrict__ yhat_lv) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ls.row0[ls.nlev]) return;
  int j = 0;
  while (j + 1 < ls.nlev && g >= ls.row0[j + 1]) ++j;
  const LevelView& v = ls.lv[j];
  const double* qh = qhat_lv[j];
  const long row = g - ls.row0[j];
  const int b = v.skel_box[row];
  const double2 xi = v.skel_xy[row];
  double acc[RC];
#pragma unroll
  for (int k = 0; k < RC; ++k) acc[k] = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int c = v.il[(long)b * 40 + s];
    if (c < 0) continue;
    const int rc = v.rank[c];
    const int sc = v.skel_off[c];
    const double2* xc = v.skel_xy + sc;
    for (int cc = 0; cc < rc; ++cc) {
      const double2 p = xc[cc];
      const double dx = xi.x - p.x, dy = xi.y - p.y;
      const double kv = K::eval(dx * dx + dy * dy, kp);
      double q[RC];
      load_vec<RC>(qh + (long)(sc + cc) * RC, q);
#pragma unroll
      for (int k = 0; k < RC; ++k) acc[k] = fma(kv, q[k], acc[k]);
    }
  }
  store_vec<RC>(yhat_lv[j] + row * RC, acc);
}

// L2L: one thread per node row; child incoming potential += L2P yhat, or the
// leaf potential = L2P yhat.
template <int RC>
__global__ void k_l2l_b(LevelView v, const double* __restrict__ yhat, double* __restrict__ child_yhat,
                        double* __restrict__ ys, int leaf) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= v.nnodes) return;
  const int b = v.node_box[g];
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int i = (int)(g - v.node_off[b]);
  const double* P = v.l2p + v.l2p_off[b] + i;
  const double* yb = yhat + (long)v.skel_off[b] * RC;
  double acc[RC];
#pragma unroll
  for (int k = 0; k < RC; ++k) acc[k] = 0.0;
  for (int c = 0; c < r; ++c) {
    const double p = P[(long)c * n];
    double yv[RC];
    load_vec<RC>(yb + (long)c * RC, yv);
#pragma unroll
    for (int k = 0; k < RC; ++k) acc[k] = fma(p, yv[k], acc[k]);
  }
  if (leaf) {
    store_vec<RC>(ys + (long)(v.leaf_start[b] + i) * RC, acc);
  } else {
    double* out = child_yhat + g * RC;
    double cur[RC];
    load_vec<RC>(out, cur);
#pragma unroll
    for (int k = 0; k < RC; ++k) cur[k] += acc[k];
    store_vec<RC>(out, cur);
  }
}

template <class K>
__device__ __forceinline__ float fallback_r2_b(float span_b, float span_c) {
  float e = (span_b + span_c) * 0.0078125f;
  float t = e * e;
  if (K::id == AFMM_KERNEL_LOG) t = fmaxf(t, 4e-10f);
  return t;
}

// Near field in FP32: one CTA per leaf, one thread per target, all source
// leaves staged in shared memory (coordinates relative to the target leaf's
// anchor folded per source leaf; charges as RC-vectors).
template <class K, int RC>
__global__ void k_p2p_b(NearView nv, KernelParams kp, const float* __restrict__ qs32, double* __restrict__ ys) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_src[9], s_cnt[9], s_off[10], s_ns;
  __shared__ float s_dx[9], s_dy[9], s_thr[9];
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  if (threadIdx.x == 0) {
    const double2 ab = nv.anchor[b];
    const float sb = nv.span[b];
    int m = 0, off = 0;
    for (int slot = 0; slot < 9; ++slot) {
      const long c = slot < 8 ? nv.nbr[b * 8 + slot] : b;
      if (c < 0) continue;
      const double2 ac = nv.anchor[c];
      s_src[m] = nv.leaf_start[c];
      s_cnt[m] = nv.leaf_cnt[c];
      s_off[m] = off;
      s_dx[m] = (float)(ab.x - ac.x);
      s_dy[m] = (float)(ab.y - ac.y);
      s_thr[m] = fallback_r2_b<K>(sb, nv.span[c]);
      off += nv.leaf_cnt[c];
      ++m;
    }
    s_off[m] = off;
    s_ns = m;
  }
  __syncthreads();
  const int ns = s_ns;
  float4* sq = (float4*)smem;                 // 9*nmax*RC/4
  float2* sx = (float2*)(sq + 9 * nv.nmax * (RC / 4));
  for (int m = 0; m < ns; ++m) {
    const float4* qsrc = reinterpret_cast<const float4*>(qs32 + (long)s_src[m] * RC);
    const int o = s_off[m], nc = s_cnt[m];
    for (int t = threadIdx.x; t < nc; t += blockDim.x) sx[o + t] = nv.rel[s_src[m] + t];
    for (int t = threadIdx.x; t < nc * (RC / 4); t += blockDim.x) sq[o * (RC / 4) + t] = qsrc[t];
  }
  __syncthreads();
  const int i = threadIdx.x;
  if (i >= n) return;
  const float2 xi = nv.rel[s0 + i];
  double acc[RC];
#pragma unroll
  for (int k = 0; k < RC; ++k) acc[k] = 0.0;
  for (int m = 0; m < ns; ++m) {
    const int o = s_off[m], nc = s_cnt[m];
    const float ox = xi.x + s_dx[m], oy = xi.y + s_dy[m], thr = s_thr[m];
    float part[RC];
#pragma unroll
    for (int k = 0; k < RC; ++k) part[k] = 0.0f;
    for (int t = 0; t < nc; ++t) {
      const float2 p = sx[o + t];
      const float dx = ox - p.x, dy = oy - p.y;
      const float R2 = fmaf(dx, dx, dy * dy);
      float kv;
      if (R2 < thr) {
        const int ps = s0 + i, qsrc = s_src[m] + t;
        if (ps == qsrc) {
          kv = (float)K::at_zero();
        } else {
          const double2 a = nv.pts[ps], c2 = nv.pts[qsrc];
          kv = (float)K::eval_exact(r2_exact(a.x, a.y, c2.x, c2.y), kp);
        }
      } else {
        kv = K::eval32(R2, a32, p32);
      }
      const float4* qv = sq + (o + t) * (RC / 4);
#pragma unroll
      for (int k4 = 0; k4 < RC / 4; ++k4) {
        const float4 w = qv[k4];
        part[4 * k4] = fmaf(kv, w.x, part[4 * k4]);
        part[4 * k4 + 1] = fmaf(kv, w.y, part[4 * k4 + 1]);
        part[4 * k4 + 2] = fmaf(kv, w.z, part[4 * k4 + 2]);
        part[4 * k4 + 3] = fmaf(kv, w.w, part[4 * k4 + 3]);
      }
    }
#pragma unroll
    for (int k = 0; k < RC; ++k) acc[k] += (double)part[k];
  }
  double* out = ys + (long)(s0 + i) * RC;
  double cur[RC];
  load_vec<RC>(out, cur);
#pragma unroll
  for (int k = 0; k < RC; ++k) cur[k] += acc[k];
  store_vec<RC>(out, cur);
}

// ------------------------------------------------------- tensor-core tiles
// FP64 MMA m8n8k4 (D = A B + C; A 8x4 row-major, B 4x8 column-major): lane l
// holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) .. 2(l%4)+1].
__device__ __forceinline__ void mma_f64_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// TF32 MMA m16n8k8: lane l = 4g + t holds A[g][t], A[g+8][t], A[g][t+4],
// A[g+8][t+4]; B[t][g], B[t+4][g]; D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1].
__device__ __forceinline__ void mma_tf32_16x8x8(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// M2L on the fly with FP64 tensor-core tiles: one warp per row group (up to 8
// skeleton rows of one box).  For every interaction-list box and every 4 of
// its skeleton points, each lane evaluates the one FP64 entry it holds in the
// A fragment (row l/4, source l%4: no entry is evaluated twice) and the warp
// multiplies the 8x4 tile with the 4 x RC block of outgoing charges.
template <class K, int RC>
__global__ void __launch_bounds__(128) k_m2l_mma(LevelSet ls, KernelParams kp, const double* const* __restrict__ qhat_lv,
                                                 double* const* __restrict__ yhat_lv) {
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= ls.grp0[ls.nlev]) return;  // whole warps only
  int j = 0;
  while (j + 1 < ls.nlev && gw >= ls.grp0[j + 1]) ++j;
  const LevelView& v = ls.lv[j];
  const double* qh = qhat_lv[j];
  const long g = gw - ls.grp0[j];
  const int b = v.grp_box[g];
  const int r0 = v.grp_row[g];
  const int nv = min(8, v.skel_off[b] + v.rank[b] - r0);
  const int trow = lane >> 2, tsrc = lane & 3;
  const bool vrow = trow < nv;
  const double2 xi = vrow ? v.skel_xy[r0 + trow] : make_double2(0.0, 0.0);
  double c[RC / 8][2];
#pragma unroll
  for (int t = 0; t < RC / 8; ++t) c[t][0] = c[t][1] = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int cb = v.il[(long)b * 40 + s];
    if (cb < 0) continue;
    const int rc = v.rank[cb];
    const int sc = v.skel_off[cb];
    for (int cc0 = 0; cc0 < rc; cc0 += 4) {
      const int cs = cc0 + tsrc;
      const bool vs = cs < rc;
      double a = 0.0;
      if (vrow && vs) {
        const double2 p = v.skel_xy[sc + cs];
        const double dx = xi.x - p.x, dy = xi.y - p.y;
        a = K::eval(dx * dx + dy * dy, kp);
      }
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) {
        const double bq = vs ? qh[(long)(sc + cs) * RC + t * 8 + trow] : 0.0;
        mma_f64_8x8x4(c[t][0], c[t][1], a, bq);
      }
    }
  }
  if (vrow) {
    double* out = yhat_lv[j] + (long)(r0 + trow) * RC;
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) {
      out[t * 8 + 2 * tsrc] = c[t][0];
      out[t * 8 + 2 * tsrc + 1] = c[t][1];
    }
  }
}

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
                                                 double* __restrict__ yb, int b, int r0, int lane) {
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
              Q32 ? (const void*)(v.m2l_q + stop) : (const void*)(v.m2l + stop));
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
#define AFMM_M2L(NT) m2l_stored_chunk<RC, NT, Q32>(v, qhat_lv[j], yhat_lv[j], b, r0, lane)
  AFMM_NT_SWITCH(chunk_tiles(v.cgrp_row, g, v.ncgroups, v.skel_off[b] + v.rank[b]), AFMM_M2L)
#undef AFMM_M2L
}

// TF32 high / low parts of an FP32 value by masking (the tensor cores read
// the top 19 bits of a TF32 operand): hi keeps 11 significant bits, lo the
// next 11 of the exact remainder; |x - hi - lo| <= 2^-21 |x|.
__device__ __forceinline__ void split_tf32_mask(float x, uint32_t& hi, uint32_t& lo) {
  hi = __float_as_uint(x) & 0xffffe000u;
  lo = __float_as_uint(x - __uint_as_float(hi)) & 0xffffe000u;
}

// Far-away stand-ins for padded source slots and absent targets: their
// entries are finite for every kernel and never below a fallback threshold;
// padded sources get zero charges and absent targets are not stored.
constexpr float kPadSrc = 1.0e15f, kPadTgt = -1.0e15f;

// Near field with TF32 tensor-core tiles in a three-term split
// (A_hi B_hi + A_hi B_lo + A_lo B_hi, ~FP32 accuracy).  One CTA per leaf, one
// warp per 32 targets (two 16 x 8 tiles sharing every charge fragment).  The
// source leaves (neighbours 0..7, then the leaf itself) are staged in shared
// memory in the target leaf's frame (each source leaf's anchor offset folded
// in FP64), padded to multiples of 8; the charges' interleaved TF32 high / low
// parts (split once per pass by the gather) come from L2, one 8-byte load per
// fragment element.  Each lane evaluates 8 FP32 entries per 8-source step; a
// warp vote sends the rare close pairs to the FP64 fallback.  The high*high
// products and the two correction products accumulate in separate FP32 tiles
// (independent MMA chains), which are added per source leaf into FP64 sums
// kept in shared memory.
template <class K, int RC>
__global__ void __launch_bounds__(128) k_p2p_mma(NearView nv, KernelParams kp, const uint2* __restrict__ qhl,
                                                 double* __restrict__ ys) {
  constexpr int NE = 2 * (RC / 8) * 4;  // FP64 sums per lane
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_src[9], s_cnt[9], s_coff[10], s_ns;
  __shared__ float s_dx[9], s_dy[9], s_thr[9];
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  if (threadIdx.x == 0) {
    const double2 ab = nv.anchor[b];
    const float sb = nv.span[b];
    int m = 0, off = 0;
    for (int slot = 0; slot < 9; ++slot) {
      const long cbx = slot < 8 ? nv.nbr[b * 8 + slot] : b;
      if (cbx < 0) continue;
      const double2 ac = nv.anchor[cbx];
      s_src[m] = nv.leaf_start[cbx];
      s_cnt[m] = nv.leaf_cnt[cbx];
      s_coff[m] = off;
      s_dx[m] = (float)(ab.x - ac.x);
      s_dy[m] = (float)(ab.y - ac.y);
      s_thr[m] = fmaxf(fallback_r2_b<K>(sb, nv.span[cbx]), 1.0e-30f);
      off += (nv.leaf_cnt[cbx] + 7) >> 3;
      ++m;
    }
    s_coff[m] = off;
    s_ns = m;
  }
  __syncthreads();
  const int ns = s_ns;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double* sacc = (double*)smem + (long)warp * NE * 32;  // lane-major: sum e of lane l at e*32 + l
  float2* sx = (float2*)((double*)smem + (long)nw * NE * 32);
  for (int m = 0; m < ns; ++m) {
    const int o = s_coff[m] * 8, nc = s_cnt[m], src = s_src[m], np = (s_coff[m + 1] - s_coff[m]) * 8;
    const float ddx = s_dx[m], ddy = s_dy[m];
    for (int t = threadIdx.x; t < np; t += blockDim.x) {
      float2 p = make_float2(kPadSrc, kPadSrc);
      if (t < nc) {
        p = nv.rel[src + t];
        p.x -= ddx;
        p.y -= ddy;
      }
      sx[o + t] = p;
    }
  }
  __syncthreads();
  const int gq = lane >> 2, tq = lane & 3;
  for (int tg = warp; tg * 32 < n; tg += nw) {
    // targets of this lane: rows gq, gq + 8 of tile 0 (k = 0, 1) and of tile 1 (k = 2, 3)
    float2 x[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int ti = tg * 32 + k * 8 + gq;
      x[k] = ti < n ? nv.rel[s0 + ti] : make_float2(kPadTgt, kPadTgt);
    }
#pragma unroll
    for (int e = 0; e < NE; ++e) sacc[e * 32 + lane] = 0.0;
    for (int m = 0; m < ns; ++m) {
      const int src = s_src[m], nc = s_cnt[m];
      const float thr = s_thr[m];
      float cm[2][RC / 8][4], cc[2][RC / 8][4];
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int t = 0; t < RC / 8; ++t)
#pragma unroll
          for (int e = 0; e < 4; ++e) cm[u][t][e] = cc[u][t][e] = 0.0f;
      for (int c = s_coff[m]; c < s_coff[m + 1]; ++c) {
        const int j0 = (c - s_coff[m]) * 8;
        const float2 ps[2] = {sx[c * 8 + tq], sx[c * 8 + tq + 4]};
        float kv[4][2];
        bool close = false;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float dx = x[k].x - ps[h].x, dy = x[k].y - ps[h].y;
            const float r2 = fmaf(dx, dx, dy * dy);
            close |= r2 < thr;
            // close pairs (R2 = 0 among them) are overwritten by the FP64 fallback below
            kv[k][h] = K::eval32_pos(r2, a32, p32);
          }
        if (__any_sync(0xffffffffu, close)) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const float dx = x[k].x - ps[h].x, dy = x[k].y - ps[h].y;
              if (fmaf(dx, dx, dy * dy) < thr) {  // both points are real (stand-ins are never close)
                const int pi = s0 + tg * 32 + k * 8 + gq, qi = src + j0 + tq + 4 * h;
                if (pi == qi) {
                  kv[k][h] = (float)K::at_zero();
                } else {
                  const double2 pa = nv.pts[pi], pc = nv.pts[qi];
                  kv[k][h] = (float)K::eval_exact(r2_exact(pa.x, pa.y, pc.x, pc.y), kp);
                }
              }
            }
        }
        // A fragments: tile u rows (gq, gq + 8) = targets 2u, 2u + 1
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          split_tf32_mask(kv[2 * u][0], ah[u][0], al[u][0]);
          split_tf32_mask(kv[2 * u + 1][0], ah[u][1], al[u][1]);
          split_tf32_mask(kv[2 * u][1], ah[u][2], al[u][2]);
          split_tf32_mask(kv[2 * u + 1][1], ah[u][3], al[u][3]);
        }
        const bool va = j0 + tq < nc, vb = j0 + tq + 4 < nc;
        const uint2* ra = qhl + (long)(src + j0 + tq) * RC + gq;
        const uint2* rb = ra + 4 * RC;
#pragma unroll
        for (int t = 0; t < RC / 8; ++t) {
          const uint2 b0 = va ? ra[t * 8] : make_uint2(0u, 0u);
          const uint2 b1 = vb ? rb[t * 8] : make_uint2(0u, 0u);
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            mma_tf32_16x8x8(cm[u][t], ah[u], b0.x, b1.x);
            mma_tf32_16x8x8(cc[u][t], ah[u], b0.y, b1.y);
            mma_tf32_16x8x8(cc[u][t], al[u], b0.x, b1.x);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int t = 0; t < RC / 8; ++t)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            sacc[((u * (RC / 8) + t) * 4 + e) * 32 + lane] += (double)cm[u][t][e] + (double)cc[u][t][e];
    }
    // D fragment of tile u: rows gq (e = 0, 1) and gq + 8 (e = 2, 3), columns 2tq, 2tq + 1
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int hr = 0; hr < 2; ++hr) {
        const int ti = tg * 32 + (2 * u + hr) * 8 + gq;
        if (ti < n) {
#pragma unroll
          for (int t = 0; t < RC / 8; ++t) {
            double2* o = reinterpret_cast<double2*>(ys + (long)(s0 + ti) * RC + t * 8 + 2 * tq);
            double2 w = *o;
            w.x += sacc[((u * (RC / 8) + t) * 4 + 2 * hr) * 32 + lane];
            w.y += sacc[((u * (RC / 8) + t) * 4 + 2 * hr + 1) * 32 + lane];
            *o = w;
          }
        }
      }
  }
}

// Stand-in coordinates of padded source slots and absent targets of the FP64
// near field (finite entries for every kernel, never stored).
constexpr double kPadSrc64 = 1.0e100, kPadTgt64 = -1.0e100;

// Near field in FP64 on the FP64 tensor cores (AFMM_PREC_FP64_BATCHED): one
// CTA per leaf, one warp per 32 targets (four 8-row tiles sharing every charge
// fragment).  Source leaves (neighbours 0..7, then the leaf itself) are staged
// in shared memory with their exact coordinates, padded to multiples of 4 with
// far stand-ins; each lane evaluates one FP64 entry per tile and 4-source step
// with the FP64 matvec form K::eval (the diagonal included, as in the FP64
// path), and the 8 x 4 entry tiles multiply the 4 x RC FP64 charge blocks
// (mma.sync m8n8k4, FP64 accumulation).
template <class K, int RC>
__global__ void __launch_bounds__(128) k_p2p_dmma(NearView nv, KernelParams kp, const double* __restrict__ qs,
                                                  double* __restrict__ ys) {
  constexpr int NTT = 4;  // 8-row target tiles per warp
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_src[9], s_cnt[9], s_coff[10], s_ns;
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  if (threadIdx.x == 0) {
    int m = 0, off = 0;
    for (int slot = 0; slot < 9; ++slot) {
      const long cbx = slot < 8 ? nv.nbr[b * 8 + slot] : b;
      if (cbx < 0) continue;
      s_src[m] = nv.leaf_start[cbx];
      s_cnt[m] = nv.leaf_cnt[cbx];
      s_coff[m] = off;
      off += (nv.leaf_cnt[cbx] + 3) >> 2;
      ++m;
    }
    s_coff[m] = off;
    s_ns = m;
  }
  __syncthreads();
  const int ns = s_ns;
  double2* sx = (double2*)smem;
  for (int m = 0; m < ns; ++m) {
    const int o = s_coff[m] * 4, nc = s_cnt[m], src = s_src[m], np = (s_coff[m + 1] - s_coff[m]) * 4;
    for (int t = threadIdx.x; t < np; t += blockDim.x)
      sx[o + t] = t < nc ? nv.pts[src + t] : make_double2(kPadSrc64, kPadSrc64);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int trow = lane >> 2, tsrc = lane & 3;
  for (int tg = warp; tg * 32 < n; tg += nw) {
    double2 x[NTT];
#pragma unroll
    for (int u = 0; u < NTT; ++u) {
      const int ti = tg * 32 + u * 8 + trow;
      x[u] = ti < n ? nv.pts[s0 + ti] : make_double2(kPadTgt64, kPadTgt64);
    }
    double c[NTT][RC / 8][2];
#pragma unroll
    for (int u = 0; u < NTT; ++u)
#pragma unroll
      for (int t = 0; t < RC / 8; ++t) c[u][t][0] = c[u][t][1] = 0.0;
    for (int m = 0; m < ns; ++m) {
      const int src = s_src[m], nc = s_cnt[m];
      for (int st = s_coff[m]; st < s_coff[m + 1]; ++st) {
        const int j = (st - s_coff[m]) * 4 + tsrc;
        const double2 p = sx[st * 4 + tsrc];
        const bool vj = j < nc;
        double bq[RC / 8];
#pragma unroll
        for (int t = 0; t < RC / 8; ++t) bq[t] = vj ? qs[(long)(src + j) * RC + t * 8 + trow] : 0.0;
#pragma unroll
        for (int u = 0; u < NTT; ++u) {
          const double dx = x[u].x - p.x, dy = x[u].y - p.y;
          const double a = K::eval(dx * dx + dy * dy, kp);
#pragma unroll
          for (int t = 0; t < RC / 8; ++t) mma_f64_8x8x4(c[u][t][0], c[u][t][1], a, bq[t]);
        }
      }
    }
    // D fragment: row trow, columns 2*tsrc, 2*tsrc + 1 of each 8-column block
#pragma unroll
    for (int u = 0; u < NTT; ++u) {
      const int ti = tg * 32 + u * 8 + trow;
      if (ti < n) {
#pragma unroll
        for (int t = 0; t < RC / 8; ++t) {
          double2* o = reinterpret_cast<double2*>(ys + (long)(s0 + ti) * RC + t * 8 + 2 * tsrc);
          double2 w = *o;
          w.x += c[u][t][0];
          w.y += c[u][t][1];
          *o = w;
        }
      }
    }
  }
}

inline int nbk(long n, int t) { return (int)((n + t - 1) / t); }

template <int RC>
struct Pass {
  template <class K>
  struct M2l {
    static void run(const LevelSet& ls, const KernelParams& kp, const double* const* qh, double* const* yh,
                    int fp64, cudaStream_t s) {
      constexpr int RM = RC >= 8 ? RC : 8;
      if (ls.row0[ls.nlev] == 0) return;  // every box of ACA rank 0: no far field
      if (RC >= 8 && !fp64 && ls.lv[0].m2l_q != nullptr) {
        // mixed precision: the 32-bit fixed-point blocks (half the bytes)
        const long warps = ls.cgrp0[ls.nlev];
        k_m2l_stored_mma<RM, true><<<nbk(warps * 32, 128), 128, 0, s>>>(ls, qh, yh);
      } else if (RC >= 8 && ls.lv[0].m2l != nullptr) {
        // stored blocks: one HBM read of the blocks serves all RC columns
        const long warps = ls.cgrp0[ls.nlev];
        k_m2l_stored_mma<RM, false><<<nbk(warps * 32, 128), 128, 0, s>>>(ls, qh, yh);
      } else if (RC >= 8) {
        const long warps = ls.grp0[ls.nlev];
        k_m2l_mma<K, RM><<<nbk(warps * 32, 128), 128, 0, s>>>(ls, kp, qh, yh);
      } else {
        const long rows = ls.row0[ls.nlev];
        k_m2l_b<K, RC><<<nbk(rows, 128), 128, 0, s>>>(ls, kp, qh, yh);
      }
      AFMM_LAUNCH_CHECK();
    }
  };
  template <class K>
  struct P2p {
    static void run(const NearView& nv, const KernelParams& kp, const float* qs32, const uint2* qhl,
                    const double* qs, double* ys, int fp64, cudaStream_t s) {
      constexpr int RM = RC >= 8 ? RC : 8;
      if (fp64) {
        if (RC < 8) throw Error{AFMM_BAD_ARG, "FP64 batched passes take 8 or 16 columns"};
        const int warps = std::min(4, (nv.nmax + 31) / 32);
        const size_t smem = (size_t)9 * ((nv.nmax + 3) / 4 * 4) * sizeof(double2);
        allow_smem(k_p2p_dmma<K, RM>, smem);
        k_p2p_dmma<K, RM><<<(int)nv.nleaf, 32 * warps, smem, s>>>(nv, kp, qs, ys);
        AFMM_LAUNCH_CHECK();
        return;
      }
      const int warps = std::min(4, (nv.nmax + 31) / 32);
      const size_t smem_mma =
          (size_t)9 * ((nv.nmax + 7) / 8 * 8) * sizeof(float2) + (size_t)warps * RM * 32 * sizeof(double);
      if (RC >= 8) {
        allow_smem(k_p2p_mma<K, RM>, smem_mma);
        k_p2p_mma<K, RM><<<(int)nv.nleaf, 32 * warps, smem_mma, s>>>(nv, kp, qhl, ys);
      } else {
        const int T = (nv.nmax + 31) / 32 * 32;
        size_t smem = (size_t)9 * nv.nmax * (sizeof(float) * RC + sizeof(float2));
        allow_smem(k_p2p_b<K, RC>, smem);
        k_p2p_b<K, RC><<<(int)nv.nleaf, T, smem, s>>>(nv, kp, qs32, ys);
      }
      AFMM_LAUNCH_CHECK();
    }
  };

  static void run(const MatvecPlan& p, BatchState& bs, const NearView& nv, const double* q, int64_t ldq, double* y,
                  int64_t ldy, int ncols, int fp64, cudaStream_t s, StageTimer* tm, int64_t* launches) {
    constexpr int RM = RC >= 8 ? RC : 8;
    const int N = p.N;
    if (tm) tm->mark(s, "gather");
    k_gather_b<RC><<<nbk(N, kTileJ), 256, 0, s>>>(q, ldq, ncols, p.iperm, N, bs.qs, bs.qs32, bs.qhl, fp64);
    AFMM_LAUNCH_CHECK();
    ++*launches;
    if (tm) tm->mark(s, "m2m");
    for (int j = p.L; j >= 2; --j) {
      const LevelView& v = p.lv[j];
      if (v.nrows == 0) continue;
      if (RC >= 8)
        k_m2m_mma<RM><<<nbk(v.ncgroups * 32, 128), 128, 0, s>>>(v, j == p.L ? bs.qs : bs.qhat[j + 1], j == p.L,
                                                               bs.qhat[j]);
      else
        k_m2m_b<RC><<<nbk(v.nrows, 128), 128, 0, s>>>(v, j == p.L ? bs.qs : bs.qhat[j + 1], j == p.L, bs.qhat[j]);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "m2l");
    dispatch_kernel<M2l>(p.kp.id, p.levels, p.kp, bs.d_qhat_lv, bs.d_yhat_lv, fp64, s);
    ++*launches;
    if (tm) tm->mark(s, "l2l");
    for (int j = 2; j <= p.L; ++j) {
      const LevelView& v = p.lv[j];
      if (v.nnodes == 0) continue;
      if (RC >= 8)
        k_l2l_mma<RM><<<nbk(v.nncgroups * 32, 128), 128, 0, s>>>(v, bs.yhat[j], j < p.L ? bs.yhat[j + 1] : nullptr,
                                                                bs.ys, j == p.L);
      else
        k_l2l_b<RC><<<nbk(v.nnodes, 128), 128, 0, s>>>(v, bs.yhat[j], j < p.L ? bs.yhat[j + 1] : nullptr, bs.ys,
                                                       j == p.L);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "p2p");
    dispatch_kernel<P2p>(p.kp.id, nv, p.kp, bs.qs32, bs.qhl, bs.qs, bs.ys, fp64, s);
    ++*launches;
    if (tm) tm->mark(s, "scatter");
    k_scatter_b<RC><<<nbk(N, kTileJ), 256, 0, s>>>(bs.ys, p.iperm, N, ncols, y, ldy);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
};

}  // namespace

void batch_reserve(const MatvecPlan& p, BatchState& bs, DevArena& arena, cudaStream_t s) {
  if (bs.ready) return;
  const int RC = kBatchMax;
  bs.qs = arena.alloc<double>((size_t)p.N * RC);
  // FP32 charges (passes of fewer than 8 columns) and TF32 parts (8 or more)
  // are never needed by the same pass: one buffer holds either
  bs.qhl = arena.alloc<uint2>((size_t)p.N * RC);
  bs.qs32 = reinterpret_cast<float*>(bs.qhl);
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
  NearView nv = p.near;
  nv.anchor = ms.leaf_anchor;
  nv.rel = ms.rel;
  nv.span = ms.leaf_span;
  for (int c0 = 0; c0 < nrhs;) {
    const int left = nrhs - c0;
    // FP64 passes take 8 or 16 columns (tensor-core tiles; unused columns are zero)
    const int rc = left > 8 ? 16 : (left > 4 || fp64 ? 8 : 4);
    const int nc = std::min(left, rc);
    const double* qc = q + (long)c0 * ldq;
    double* yc = y + (long)c0 * ldy;
    if (rc == 16) Pass<16>::run(p, bs, nv, qc, ldq, yc, ldy, nc, fp64, s, tm, launches);
    else if (rc == 8) Pass<8>::run(p, bs, nv, qc, ldq, yc, ldy, nc, fp64, s, tm, launches);
    else Pass<4>::run(p, bs, nv, qc, ldq, yc, ldy, nc, fp64, s, tm, launches);
    c0 += nc;
  }
}

}  // namespace afmm
