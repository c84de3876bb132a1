// Mixed-precision matvec: FP32 apply with FP64 where it matters.
//
// Same sweeps as the FP64 path (src/AFMM2DTree.cpp:1129-1213), with
//  * L2P stored in FP32 (both layouts) and applied with FP64 accumulation to
//    FP64 outgoing / incoming vectors (those vectors are small);
//  * M2L evaluated on the fly from skeleton coordinates instead of reading
//    stored blocks: K(R_b, R_c) entries are the kernel between skeleton points
//    (src/AFMM2DTree.cpp:1080);
//  * near field evaluated on the fly in FP32.
// Precision safeguards:
//  * coordinates are kept relative to a per-box anchor point in FP32, and the
//    anchor difference of a box pair is formed in FP64 before rounding, so dx
//    keeps ~2^-24 relative precision however clustered the points are;
//  * pairs closer than 2^-7 of the two boxes' extents (where the FP32 relative
//    coordinates lose more than ~2^-17 relative precision), and for the log
//    kernel every pair with R2 near its 1e-10 diagonal convention, are
//    re-evaluated in FP64 from the exact coordinates;
//  * M2L: the outgoing charges are split into FP32 high and low parts, the
//    products with the high part are summed with Kahan compensation per
//    interaction-list box, and the per-box sums are accumulated in FP64;
//  * near field: FP32 partial sums per source leaf, accumulated in FP64;
//    outputs are FP64.
#include <algorithm>

#include "mixed.cuh"

namespace afmm {

namespace {

// Per box: anchor = first skeleton point; rel = skeleton - anchor (FP32);
// span = max |rel| component.
__global__ void k_anchor_level(long nbox, const int32_t* __restrict__ rank, const int32_t* __restrict__ skel_off,
                               const double2* __restrict__ skel_xy, double2* anchor, float2* rel, float* span) {
  const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  const int r = rank[b], so = skel_off[b];
  double2 a = r > 0 ? skel_xy[so] : make_double2(0.0, 0.0);
  float sp = 0.0f;
  for (int l = 0; l < r; ++l) {
    double2 p = skel_xy[so + l];
    float2 d = make_float2((float)(p.x - a.x), (float)(p.y - a.y));
    rel[so + l] = d;
    sp = fmaxf(sp, fmaxf(fabsf(d.x), fabsf(d.y)));
  }
  anchor[b] = a;
  span[b] = sp;
}

// Leaves: anchor = first point of the leaf; rel for every sorted point.
__global__ void k_anchor_leaf(long nleaf, const int32_t* __restrict__ start, const int32_t* __restrict__ cnt,
                              const double2* __restrict__ pts, double2* anchor, float2* rel, float* span) {
  const long b = blockIdx.x;
  const int s0 = start[b], n = cnt[b];
  const double2 a = pts[s0];
  float sp = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 p = pts[s0 + i];
    float2 d = make_float2((float)(p.x - a.x), (float)(p.y - a.y));
    rel[s0 + i] = d;
    sp = fmaxf(sp, fmaxf(fabsf(d.x), fabsf(d.y)));
  }
  for (int o = 16; o > 0; o >>= 1) sp = fmaxf(sp, __shfl_down_sync(0xffffffffu, sp, o));
  __shared__ float ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sp;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.0f;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmaxf(m, ws[w]);
    anchor[b] = a;
    span[b] = m;
  }
}

__global__ void k_to_f32(const double* __restrict__ src, long n, float* dst) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

// qs[i] = q[perm[i]] in FP64 and FP32
__global__ void k_gather_mixed(const double* __restrict__ q, const int64_t* __restrict__ perm, int N, double* qs,
                               float* qs32) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double v = q[perm[i]];
  qs[i] = v;
  qs32[i] = (float)v;
}

__global__ void k_scatter64(const double* __restrict__ ys, const int64_t* __restrict__ perm, int N, int nrhs,
                            double* y, int64_t ldy) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)N * nrhs) return;
  int c = (int)(t / N), i = (int)(t - (long)c * N);
  y[(long)c * ldy + perm[i]] = ys[t];
}

// M2M with FP32 L2P (row-major) and FP64 accumulation: one CTA per box, rows
// split across warps, lanes over outputs.  Writes qhat (FP64) and its FP32
// high/low split.
__global__ void __launch_bounds__(SW_T) k_m2m_mixed(LevelView v, const double* __restrict__ src_all, int leaf) {
  extern __shared__ double part[];  // SW_WARPS x r
  const long b = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = v.rank[b];
  if (r == 0) return;
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (leaf ? v.leaf_start[b] : v.node_off[b]);
  const float* P = v.l2p32_rm + v.l2p_off[b];
  const int i0 = (int)((long)n * warp / SW_WARPS), i1 = (int)((long)n * (warp + 1) / SW_WARPS);
  for (int c0 = 0; c0 < r; c0 += 32) {
    const int c = c0 + lane;
    if (c < r) {
      double s = 0.0;
#pragma unroll 4
      for (int i = i0; i < i1; ++i) s += (double)P[(long)i * r + c] * src[i];
      part[warp * r + c] = s;
    }
  }
  __syncthreads();
  const int so = v.skel_off[b];
  for (int c = threadIdx.x; c < r; c += SW_T) {
    double s = 0.0;
    for (int w = 0; w < SW_WARPS; ++w) s += part[w * r + c];
    v.qhat[so + c] = s;
    float hi = (float)s;
    v.qhat32[so + c] = hi;
    v.qlo32[so + c] = (float)(s - (double)hi);
  }
}

// Threshold below which a pair is re-evaluated in FP64.
template <class K>
__device__ __forceinline__ float fallback_r2(float span_b, float span_c) {
  float e = (span_b + span_c) * 0.0078125f;  // 2^-7 of the combined extent
  float t = e * e;
  if (K::id == AFMM_KERNEL_LOG) t = fmaxf(t, 4e-10f);
  return t;
}

// M2L on the fly for every level: one CTA per box (upper levels first), warp
// w takes the valid interaction-list slots w, w + SW_WARPS, ...; lanes run
// over the box's skeleton rows; partial sums are added in warp order.
template <class K>
__global__ void __launch_bounds__(SW_T) k_m2l32(LevelSet ls, KernelParams kp) {
  extern __shared__ double part[];  // SW_WARPS x r
  __shared__ int s_slot[40], s_nvalid;
  long gb = blockIdx.x;
  int j = 0;
  while (j < ls.nlev && gb >= ls.lv[j].nbox) gb -= ls.lv[j++].nbox;
  if (j >= ls.nlev) return;
  const LevelView& v = ls.lv[j];
  const long b = gb;
  const int r = v.rank[b];
  if (r == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    int m = 0;
    for (int s = 0; s < 40; ++s) {
      int c = v.il[b * 40 + s];
      if (c >= 0 && v.rank[c] > 0) s_slot[m++] = c;
    }
    s_nvalid = m;
  }
  __syncthreads();
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  const double2 ab = v.anchor[b];
  const float sb = v.span[b];
  const int so = v.skel_off[b];
  for (int i0 = 0; i0 < r; i0 += 32) {
    const int i = i0 + lane;
    double acc = 0.0;
    if (i < r) {
      const float2 xi = v.skel_rel[so + i];
      for (int t = warp; t < s_nvalid; t += SW_WARPS) {
        const int c = s_slot[t];
        const int rc = v.rank[c];
        const int sc = v.skel_off[c];
        const double2 ac = v.anchor[c];
        const float ox = xi.x + (float)(ab.x - ac.x), oy = xi.y + (float)(ab.y - ac.y);
        const float thr = fallback_r2<K>(sb, v.span[c]);
        float sum = 0.0f, comp = 0.0f, lo = 0.0f;
#pragma unroll 4
        for (int cc = 0; cc < rc; ++cc) {
          const float2 xc = v.skel_rel[sc + cc];
          const float dx = ox - xc.x, dy = oy - xc.y;
          const float R2 = fmaf(dx, dx, dy * dy);
          float kv;
          if (R2 < thr) {
            const double2 p = v.skel_xy[so + i], q = v.skel_xy[sc + cc];
            kv = (float)K::eval_exact(r2_exact(p.x, p.y, q.x, q.y), kp);
          } else {
            kv = K::eval32(R2, a32, p32);
          }
          // Kahan-compensated sum of kv * qhi; plain sum of kv * qlo
          const float yk = fmaf(kv, v.qhat32[sc + cc], -comp);
          const float tk = sum + yk;
          comp = (tk - sum) - yk;
          sum = tk;
          lo = fmaf(kv, v.qlo32[sc + cc], lo);
        }
        acc += (double)sum - (double)comp + (double)lo;
      }
      part[warp * r + i] = acc;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < r; i += SW_T) {
    double s = 0.0;
    for (int w = 0; w < SW_WARPS; ++w) s += part[w * r + i];
    v.yhat[so + i] = s;
  }
}

template <class K>
struct M2l32Run {
  static void run(const LevelSet& ls, const KernelParams& kp, long boxes, int rmax, cudaStream_t s) {
    k_m2l32<K><<<(int)boxes, SW_T, sizeof(double) * SW_WARPS * std::max(rmax, 1), s>>>(ls, kp);
    AFMM_LAUNCH_CHECK();
  }
};

// L2L with FP32 L2P (column-major) and FP64 accumulation: one CTA per box,
// threads over rows.
__global__ void __launch_bounds__(SW_T) k_l2l_mixed(LevelView v, double* __restrict__ child_yhat,
                                                    double* __restrict__ ys, int leaf) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const float* P = v.l2p32 + v.l2p_off[b];
  const double* yb = v.yhat + v.skel_off[b];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double t = 0.0;
#pragma unroll 8
    for (int c = 0; c < r; ++c) t += (double)P[(long)c * n + i] * yb[c];
    if (leaf) ys[v.leaf_start[b] + i] = t;
    else child_yhat[v.node_off[b] + i] += t;
  }
}

// Near field in FP32 from leaf-relative coordinates: CTA per leaf, threads
// over targets, source leaves (neighbours 0..7, then self) staged in
// shared memory.
template <class K>
__global__ void k_p2p32(NearView nv, KernelParams kp, const float* __restrict__ qs32, double* __restrict__ ys) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* sx = (float2*)smem;
  float* sq = (float*)(sx + nv.nmax);
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const int T = blockDim.x;
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  const double2 ab = nv.anchor[b];
  const float sb = nv.span[b];
  constexpr int MAXT = 4;
  float2 xi[MAXT];
  double pot[MAXT];
#pragma unroll
  for (int u = 0; u < MAXT; ++u) {
    int i = threadIdx.x + u * T;
    xi[u] = i < n ? nv.rel[s0 + i] : make_float2(0.f, 0.f);
    pot[u] = i < n ? ys[s0 + i] : 0.0;
  }
  for (int slot = 0; slot < 9; ++slot) {
    const long c = slot < 8 ? nv.nbr[b * 8 + slot] : b;
    if (c < 0) continue;
    const int nc = nv.leaf_cnt[c];
    const int c0 = nv.leaf_start[c];
    const double2 ac = nv.anchor[c];
    const float dxa = (float)(ab.x - ac.x), dya = (float)(ab.y - ac.y);
    const float thr = fallback_r2<K>(sb, nv.span[c]);
    __syncthreads();
    for (int t = threadIdx.x; t < nc; t += T) {
      sx[t] = nv.rel[c0 + t];
      sq[t] = qs32[c0 + t];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < MAXT; ++u) {
      const int i = threadIdx.x + u * T;
      if (i < n) {
        float acc = 0.0f;
        const float ox = xi[u].x + dxa, oy = xi[u].y + dya;
#pragma unroll 4
        for (int t = 0; t < nc; ++t) {
          const float dx = ox - sx[t].x, dy = oy - sx[t].y;
          const float R2 = fmaf(dx, dx, dy * dy);
          float kv;
          if (R2 < thr) {
            const double2 p = nv.pts[s0 + i], q = nv.pts[c0 + t];
            kv = (float)K::eval_exact(r2_exact(p.x, p.y, q.x, q.y), kp);
          } else {
            kv = K::eval32(R2, a32, p32);
          }
          acc = fmaf(kv, sq[t], acc);
        }
        pot[u] += (double)acc;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < MAXT; ++u) {
    int i = threadIdx.x + u * T;
    if (i < n) ys[s0 + i] = pot[u];
  }
}

template <class K>
struct P2p32Run {
  static void run(const NearView& nv, const KernelParams& kp, const float* qs32, double* ys, cudaStream_t s) {
    int T = std::min(256, ((nv.nmax + 3) / 4 + 31) / 32 * 32);
    T = std::max(T, 64);
    size_t smem = (size_t)nv.nmax * (sizeof(float2) + sizeof(float));
    k_p2p32<K><<<(int)nv.nleaf, T, smem, s>>>(nv, kp, qs32, ys);
    AFMM_LAUNCH_CHECK();
  }
};

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void mixed_setup(MatvecPlan& p, std::vector<LevelDev>& lv, MixedState& ms, DevArena& arena, cudaStream_t s,
                 int64_t* launches) {
  const int L = p.L;
  for (int j = 2; j <= L; ++j) {
    LevelDev& d = lv[j];
    const long tr = std::max<long>(d.total_rank, 1);
    const long ne = std::max<long>(d.h_l2p_off[d.nbox], 1);
    d.anchor = arena.alloc<double2>(d.nbox);
    d.skel_rel = arena.alloc<float2>(tr);
    d.span = arena.alloc<float>(d.nbox);
    d.l2p32 = arena.alloc<float>(ne);
    d.l2p32_rm = arena.alloc<float>(ne);
    d.qhat32 = arena.alloc<float>(tr);
    d.qlo32 = arena.alloc<float>(tr);
    k_anchor_level<<<nb(d.nbox, 128), 128, 0, s>>>(d.nbox, d.rank, d.skel_off, d.skel_xy, d.anchor, d.skel_rel, d.span);
    k_to_f32<<<nb(ne, 256), 256, 0, s>>>(d.l2p, d.h_l2p_off[d.nbox], d.l2p32);
    k_to_f32<<<nb(ne, 256), 256, 0, s>>>(d.l2p_rm, d.h_l2p_off[d.nbox], d.l2p32_rm);
    AFMM_LAUNCH_CHECK();
    *launches += 3;
  }
  NearView& nv = p.near;
  ms.leaf_anchor = arena.alloc<double2>(nv.nleaf);
  ms.leaf_span = arena.alloc<float>(nv.nleaf);
  ms.rel = arena.alloc<float2>(p.N);
  k_anchor_leaf<<<(int)nv.nleaf, 64, 0, s>>>(nv.nleaf, nv.leaf_start, nv.leaf_cnt, nv.pts, ms.leaf_anchor, ms.rel,
                                              ms.leaf_span);
  AFMM_LAUNCH_CHECK();
  *launches += 1;
  ms.ready = true;
}

void mixed_reserve(MixedState& ms, int N, int nrhs, DevArena& arena) {
  if (ms.rhs_cap >= nrhs) return;
  ms.qs32 = arena.alloc<float>((size_t)N * nrhs);
  ms.qs = arena.alloc<double>((size_t)N * nrhs);
  ms.ys = arena.alloc<double>((size_t)N * nrhs);
  ms.rhs_cap = nrhs;
}

void mixed_reserve_io(MixedState& ms, int N, int nrhs, DevArena& arena) {
  ms.d_qin = arena.alloc<double>((size_t)N * nrhs);
  ms.d_yout = arena.alloc<double>((size_t)N * nrhs);
  ms.host_cap = nrhs;
}

void matvec_mixed(const MatvecPlan& p, MixedState& ms, const double* q, int64_t ldq, double* y, int64_t ldy, int nrhs,
                  cudaStream_t s, StageTimer* tm, int64_t* launches) {
  if (!ms.ready) throw Error{AFMM_BAD_ARG, "mixed precision operators are not set up"};
  const int N = p.N;
  long boxes = 0;
  int rm = 1;
  for (int j = 0; j < p.levels.nlev; ++j) boxes += p.levels.lv[j].nbox;
  for (int j = 2; j <= p.L; ++j) rm = std::max(rm, p.rmax[j]);
  for (int c = 0; c < nrhs; ++c) {
    double* ys = ms.ys;
    if (tm) tm->mark(s, "gather");
    k_gather_mixed<<<nb(N, 256), 256, 0, s>>>(q + (long)c * ldq, p.perm, N, ms.qs, ms.qs32);
    AFMM_LAUNCH_CHECK();
    ++*launches;
    if (tm) tm->mark(s, "m2m");
    for (int j = p.L; j >= 2; --j) {
      const LevelView& v = p.lv[j];
      k_m2m_mixed<<<(int)v.nbox, SW_T, sizeof(double) * SW_WARPS * std::max(p.rmax[j], 1), s>>>(
          v, j == p.L ? ms.qs : p.lv[j + 1].qhat, j == p.L);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "m2l");
    dispatch_kernel<M2l32Run>(p.kp.id, p.levels, p.kp, boxes, rm, s);
    ++*launches;
    if (tm) tm->mark(s, "l2l");
    for (int j = 2; j <= p.L; ++j) {
      const LevelView& v = p.lv[j];
      k_l2l_mixed<<<(int)v.nbox, sweep_threads(p.n1max[j]), 0, s>>>(v, j < p.L ? p.lv[j + 1].yhat : nullptr, ys,
                                                                    j == p.L);
      AFMM_LAUNCH_CHECK();
      ++*launches;
    }
    if (tm) tm->mark(s, "p2p");
    NearView nv = p.near;
    nv.anchor = ms.leaf_anchor;
    nv.rel = ms.rel;
    nv.span = ms.leaf_span;
    dispatch_kernel<P2p32Run>(p.kp.id, nv, p.kp, ms.qs32, ys, s);
    ++*launches;
    if (tm) tm->mark(s, "scatter");
    k_scatter64<<<nb(N, 256), 256, 0, s>>>(ys, p.perm, N, 1, y + (long)c * ldy, ldy);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

}  // namespace afmm
