// Kernel-templated stages of the batched (multi-RHS) path: M2L on the fly
// and the near fields, instantiated once per kernel functor by the kernel
// tables (kernel_table.cuh).
#pragma once
#include <algorithm>

#include "batched_common.cuh"
#include "mixed.cuh"

namespace afmm {

namespace batched_detail {

template <class K>
__device__ __forceinline__ float fallback_r2_b(float span_b, float span_c) {
  float e = (span_b + span_c) * 0.0078125f;
  float t = e * e;
  if (K::id == AFMM_KERNEL_LOG) t = fmaxf(t, 4e-10f);
  return t;
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
  const double* qh = qhat_lv[ls.src[j]];
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
    double* out = yhat_lv[ls.src[j]] + (long)(r0 + trow) * RC;
#pragma unroll
    for (int t = 0; t < RC / 8; ++t) {
      out[t * 8 + 2 * tsrc] = c[t][0];
      out[t * 8 + 2 * tsrc + 1] = c[t][1];
    }
  }
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
  const long b = nv.leaf0 + blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  if (threadIdx.x < 32) {
    const NearSlots sl = near_slots<8>(nv, b, threadIdx.x);
    if (sl.m >= 0) {
      const double2 ab = nv.anchor[b], ac = nv.anchor[sl.c];
      s_src[sl.m] = sl.start;
      s_cnt[sl.m] = sl.cnt;
      s_coff[sl.m] = sl.off;
      s_dx[sl.m] = (float)(ab.x - ac.x);
      s_dy[sl.m] = (float)(ab.y - ac.y);
      s_thr[sl.m] = fmaxf(fallback_r2_b<K>(nv.span[b], nv.span[sl.c]), 1.0e-30f);
    }
    if (threadIdx.x == 0) {
      s_coff[sl.ns] = sl.total;
      s_ns = sl.ns;
    }
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
                  kv[k][h] = (float)K::at_zero(kp);
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
  const long b = nv.leaf0 + blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  if (threadIdx.x < 32) {
    const NearSlots sl = near_slots<4>(nv, b, threadIdx.x);
    if (sl.m >= 0) {
      s_src[sl.m] = sl.start;
      s_cnt[sl.m] = sl.cnt;
      s_coff[sl.m] = sl.off;
    }
    if (threadIdx.x == 0) {
      s_coff[sl.ns] = sl.total;
      s_ns = sl.ns;
    }
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

// M2L with the entries evaluated on the fly, RC = 8 or 16 columns per pass,
// on FP64 tensor-core tiles (k_m2l_mma).
template <class K, int RC>
void m2l_otf_batched(const LevelSet& ls, const KernelParams& kp, const double* const* qh, double* const* yh,
                     cudaStream_t s) {
  if (ls.row0[ls.nlev] == 0) return;
  const long warps = ls.grp0[ls.nlev];
  k_m2l_mma<K, RC><<<nbk(warps * 32, 128), 128, 0, s>>>(ls, kp, qh, yh);
  AFMM_LAUNCH_CHECK();
}

// Mixed near field of a pass: TF32x3 tensor-core tiles (8 or 16 columns,
// charges as TF32 parts).
template <class K, int RC>
void p2p_mma_batched(const NearView& nv, const KernelParams& kp, const uint2* qhl, double* ys, cudaStream_t s) {
  const int warps = std::min(4, (nv.nmax + 31) / 32);
  const size_t smem = (size_t)9 * ((nv.nmax + 7) / 8 * 8) * sizeof(float2) + (size_t)warps * RC * 32 * sizeof(double);
  allow_smem(k_p2p_mma<K, RC>, smem);
  k_p2p_mma<K, RC><<<(int)nv.nleaf, 32 * warps, smem, s>>>(nv, kp, qhl, ys);
  AFMM_LAUNCH_CHECK();
}

// FP64 near field of an FP64-batched pass (8 or 16 columns).
template <class K, int RC>
void p2p_dmma_batched(const NearView& nv, const KernelParams& kp, const double* qs, double* ys, cudaStream_t s) {
  const int warps = std::min(4, (nv.nmax + 31) / 32);
  const size_t smem = (size_t)9 * ((nv.nmax + 3) / 4 * 4) * sizeof(double2);
  allow_smem(k_p2p_dmma<K, RC>, smem);
  k_p2p_dmma<K, RC><<<(int)nv.nleaf, 32 * warps, smem, s>>>(nv, kp, qs, ys);
  AFMM_LAUNCH_CHECK();
}

}  // namespace batched_detail

}  // namespace afmm
