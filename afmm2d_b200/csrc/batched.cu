// Batched mixed-precision matvec: RC right-hand sides per pass (RC = 4, 8 or
// 16), each operator entry read or evaluated once and applied to all of them.
//
// Layout: point-major blocks, value (i, c) at i*RC + c, for the sorted charges
// and potentials and for the outgoing / incoming vectors of every level, so a
// warp's lanes (consecutive rows of one box) read the same RC-vector of a
// source with one broadcast load.
//  * M2M / L2L: FP64 L2P (row-major / column-major), one thread per output
//    row with RC FP64 accumulators.
//  * M2L: entries evaluated on the fly in FP64 from the skeleton coordinates
//    (as in the single-RHS mixed path), RC FP64 multiply-adds per entry.
//  * Near field: entries in FP32 from leaf-relative coordinates with the FP64
//    fallback for close pairs (as in the single-RHS mixed path), RC FP32
//    multiply-adds per entry, FP32 partial sums per source leaf accumulated
//    in FP64.
#include <algorithm>

#include "mixed.cuh"

namespace afmm {

namespace {

template <int RC>
__global__ void k_gather_b(const double* __restrict__ q, int64_t ldq, int ncols, const int64_t* __restrict__ perm,
                           int N, double* qs, float* qs32) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)N * RC) return;
  const int i = (int)(t / RC), c = (int)(t % RC);
  const double v = c < ncols ? q[(long)c * ldq + perm[i]] : 0.0;
  qs[t] = v;
  qs32[t] = (float)v;
}

template <int RC>
__global__ void k_scatter_b(const double* __restrict__ ys, const int64_t* __restrict__ perm, int N, int ncols,
                            double* y, int64_t ldy) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)N * RC) return;
  const int i = (int)(t / RC), c = (int)(t % RC);
  if (c < ncols) y[(long)c * ldy + perm[i]] = ys[t];
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

inline int nbk(long n, int t) { return (int)((n + t - 1) / t); }

template <int RC>
struct Pass {
  template <class K>
  struct M2l {
    static void run(const LevelSet& ls, const KernelParams& kp, const double* const* qh, double* const* yh,
                    cudaStream_t s) {
      const long rows = ls.row0[ls.nlev];
      k_m2l_b<K, RC><<<nbk(rows, 128), 128, 0, s>>>(ls, kp, qh, yh);
      AFMM_LAUNCH_CHECK();
    }
  };
  template <class K>
  struct P2p {
    static void run(const NearView& nv, const KernelParams& kp, const float* qs32, double* ys, cudaStream_t s) {
      const int T = (nv.nmax + 31) / 32 * 32;
      size_t smem = (size_t)9 * nv.nmax * (sizeof(float) * RC + sizeof(float2));
      allow_smem(k_p2p_b<K, RC>, smem);
      k_p2p_b<K, RC><<<(int)nv.nleaf, T, smem, s>>>(nv, kp, qs32, ys);
      AFMM_LAUNCH_CHECK();
    }
  };

  static void run(const MatvecPlan& p, BatchState& bs, const NearView& nv, const double* q, int64_t ldq, double* y,
                  int64_t ldy, int ncols, cudaStream_t s, StageTimer* tm, int64_t* launches) {
    const int N = p.N;
    if (tm) tm->mark(s, "gather");
    k_gather_b<RC><<<nbk((long)N * RC, 256), 256, 0, s>>>(q, ldq, ncols, p.perm, N, bs.qs, bs.qs32);
    AFMM_LAUNCH_CHECK();
    ++*launches;
    if (tm) tm->mark(s, "m2m");
    for (int j = p.L; j >= 2; --j) {
      const LevelView& v = p.lv[j];
      if (v.nrows == 0) continue;
      k_m2m_b<RC><<<nbk(v.nrows, 128), 128, 0, s>>>(v, j == p.L ? bs.qs : bs.qhat[j + 1], j == p.L, bs.qhat[j]);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "m2l");
    dispatch_kernel<M2l>(p.kp.id, p.levels, p.kp, bs.d_qhat_lv, bs.d_yhat_lv, s);
    ++*launches;
    if (tm) tm->mark(s, "l2l");
    for (int j = 2; j <= p.L; ++j) {
      const LevelView& v = p.lv[j];
      if (v.nnodes == 0) continue;
      k_l2l_b<RC><<<nbk(v.nnodes, 128), 128, 0, s>>>(v, bs.yhat[j], j < p.L ? bs.yhat[j + 1] : nullptr, bs.ys,
                                                     j == p.L);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "p2p");
    dispatch_kernel<P2p>(p.kp.id, nv, p.kp, bs.qs32, bs.ys, s);
    ++*launches;
    if (tm) tm->mark(s, "scatter");
    k_scatter_b<RC><<<nbk((long)N * RC, 256), 256, 0, s>>>(bs.ys, p.perm, N, ncols, y, ldy);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
};

}  // namespace

void batch_reserve(const MatvecPlan& p, BatchState& bs, DevArena& arena, cudaStream_t s) {
  if (bs.ready) return;
  const int RC = kBatchMax;
  bs.qs = arena.alloc<double>((size_t)p.N * RC);
  bs.qs32 = arena.alloc<float>((size_t)p.N * RC);
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
                    int64_t ldy, int nrhs, cudaStream_t s, StageTimer* tm, int64_t* launches) {
  if (!ms.ready || !bs.ready) throw Error{AFMM_BAD_ARG, "batched operators are not set up"};
  NearView nv = p.near;
  nv.anchor = ms.leaf_anchor;
  nv.rel = ms.rel;
  nv.span = ms.leaf_span;
  for (int c0 = 0; c0 < nrhs;) {
    const int left = nrhs - c0;
    const int rc = left > 8 ? 16 : (left > 4 ? 8 : 4);
    const int nc = std::min(left, rc);
    const double* qc = q + (long)c0 * ldq;
    double* yc = y + (long)c0 * ldy;
    if (rc == 16) Pass<16>::run(p, bs, nv, qc, ldq, yc, ldy, nc, s, tm, launches);
    else if (rc == 8) Pass<8>::run(p, bs, nv, qc, ldq, yc, ldy, nc, s, tm, launches);
    else Pass<4>::run(p, bs, nv, qc, ldq, yc, ldy, nc, s, tm, launches);
    c0 += nc;
  }
}

}  // namespace afmm
