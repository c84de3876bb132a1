// Kernel-templated stages of the single-RHS mixed path: M2L on the fly in
// FP64 and the FP32 near field, instantiated once per kernel functor by the
// kernel tables (kernel_table.cuh).
#pragma once
#include "mixed.cuh"

namespace afmm {

namespace mixed_detail {

// Threshold below which a near-field pair is re-evaluated in FP64.
template <class K>
__device__ __forceinline__ float fallback_r2(float span_b, float span_c) {
  float e = (span_b + span_c) * 0.0078125f;  // 2^-7 of the combined extent
  float t = e * e;
  if (K::id == AFMM_KERNEL_LOG) t = fmaxf(t, 4e-10f);
  return t;
}

// M2L on the fly in FP64 for every level, one thread per skeleton row
// (upper levels first): row i of box b sums, slot by slot in the reference's
// order, K(R_b[i], R_c[cc]) * qhat_c[cc] with the entries evaluated from the
// skeleton coordinates (a warp's rows share the source points: broadcast
// loads).
template <class K>
__global__ void k_m2l_otf(LevelSet ls, KernelParams kp) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ls.row0[ls.nlev]) return;
  int j = 0;
  while (j + 1 < ls.nlev && g >= ls.row0[j + 1]) ++j;
  const LevelView& v = ls.lv[j];
  const long row = g - ls.row0[j];
  const int b = v.skel_box[row];
  const double2 xi = v.skel_xy[row];
  double acc = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int c = v.il[(long)b * 40 + s];
    if (c < 0) continue;
    const int rc = v.rank[c];
    const double2* xc = v.skel_xy + v.skel_off[c];
    const double* qc = v.qhat + v.skel_off[c];
    double a0 = 0.0, a1 = 0.0;
    int cc = 0;
    for (; cc + 1 < rc; cc += 2) {
      const double2 p0 = xc[cc], p1 = xc[cc + 1];
      const double dx0 = xi.x - p0.x, dy0 = xi.y - p0.y;
      const double dx1 = xi.x - p1.x, dy1 = xi.y - p1.y;
      a0 += K::eval(dx0 * dx0 + dy0 * dy0, kp) * qc[cc];
      a1 += K::eval(dx1 * dx1 + dy1 * dy1, kp) * qc[cc + 1];
    }
    if (cc < rc) {
      const double2 p0 = xc[cc];
      const double dx0 = xi.x - p0.x, dy0 = xi.y - p0.y;
      a0 += K::eval(dx0 * dx0 + dy0 * dy0, kp) * qc[cc];
    }
    acc += a0 + a1;
  }
  v.yhat[row] = acc;
}

template <class K>
struct M2lOtfRun {
  static void run(const LevelSet& ls, const KernelParams& kp, cudaStream_t s) {
    const long rows = ls.row0[ls.nlev];
    if (rows == 0) return;  // every box of ACA rank 0: no far field
    k_m2l_otf<K><<<(int)((rows + 127) / 128), 128, 0, s>>>(ls, kp);
    AFMM_LAUNCH_CHECK();
  }
};

// Kernel entry of a close pair in FP64 from the exact coordinates; a point
// with itself (the diagonal) takes the kernel's value at zero distance
// without any FP64 work, so the self-interaction costs no divergent branch.
template <class K>
__device__ __forceinline__ float near_pair(const NearView& nv, const KernelParams& kp, int p, int q) {
  if (p == q) return (float)K::at_zero(kp);
  const double2 a = nv.pts[p], c = nv.pts[q];
  return (float)K::eval_exact(r2_exact(a.x, a.y, c.x, c.y), kp);
}

// Near field in FP32 from leaf-relative coordinates.  One CTA per leaf; all
// source leaves (neighbours 0..7, then the leaf) are staged in shared memory
// at once, with each source leaf's anchor offset folded in FP64; G groups of
// NT threads split the source leaves, each thread owns one target, FP32
// partial sums per source leaf are added in FP64, and the groups' sums are
// added in group order.
template <class K>
__global__ void k_p2p32(NearView nv, KernelParams kp, const float* __restrict__ qs32, double* __restrict__ ys, int NT,
                        int G) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_src[9], s_cnt[9], s_off[10], s_ns;
  __shared__ float s_dx[9], s_dy[9], s_thr[9];
  const long b = nv.leaf0 + blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const float a32 = (float)kp.a, p32 = (float)kp.param;
  if (threadIdx.x < 32) {
    const NearSlots sl = near_slots<1>(nv, b, threadIdx.x);
    if (sl.m >= 0) {
      const double2 ab = nv.anchor[b], ac = nv.anchor[sl.c];
      s_src[sl.m] = sl.start;
      s_cnt[sl.m] = sl.cnt;
      s_off[sl.m] = sl.off;
      s_dx[sl.m] = (float)(ab.x - ac.x);
      s_dy[sl.m] = (float)(ab.y - ac.y);
      s_thr[sl.m] = fallback_r2<K>(nv.span[b], nv.span[sl.c]);
    }
    if (threadIdx.x == 0) {
      s_off[sl.ns] = sl.total;
      s_ns = sl.ns;
    }
  }
  __syncthreads();
  const int ns = s_ns;
  float2* sx = (float2*)smem;
  float* sq = (float*)(sx + 9 * nv.nmax);
  double* red = (double*)(((uintptr_t)(sq + 9 * nv.nmax) + 15) & ~(uintptr_t)15);  // G x NT
  for (int m = 0; m < ns; ++m)
    for (int t = threadIdx.x; t < s_cnt[m]; t += blockDim.x) {
      sx[s_off[m] + t] = nv.rel[s_src[m] + t];
      sq[s_off[m] + t] = qs32[s_src[m] + t];
    }
  __syncthreads();
  const int i = threadIdx.x % NT, g = threadIdx.x / NT;
  double acc = 0.0;
  if (i < n) {
    const float2 xi = nv.rel[s0 + i];
    for (int m = g; m < ns; m += G) {
      const int o = s_off[m], nc = s_cnt[m];
      const float ox = xi.x + s_dx[m], oy = xi.y + s_dy[m], thr = s_thr[m];
      float a0 = 0.0f, a1 = 0.0f;
      int t = 0;
      for (; t + 1 < nc; t += 2) {
        const float2 p0 = sx[o + t], p1 = sx[o + t + 1];
        const float dx0 = ox - p0.x, dy0 = oy - p0.y, dx1 = ox - p1.x, dy1 = oy - p1.y;
        const float R0 = fmaf(dx0, dx0, dy0 * dy0), R1 = fmaf(dx1, dx1, dy1 * dy1);
        float k0, k1;
        if (R0 < thr) k0 = near_pair<K>(nv, kp, s0 + i, s_src[m] + t);
        else k0 = K::eval32(R0, a32, p32);
        if (R1 < thr) k1 = near_pair<K>(nv, kp, s0 + i, s_src[m] + t + 1);
        else k1 = K::eval32(R1, a32, p32);
        a0 = fmaf(k0, sq[o + t], a0);
        a1 = fmaf(k1, sq[o + t + 1], a1);
      }
      if (t < nc) {
        const float2 p0 = sx[o + t];
        const float dx0 = ox - p0.x, dy0 = oy - p0.y;
        const float R0 = fmaf(dx0, dx0, dy0 * dy0);
        float k0;
        if (R0 < thr) k0 = near_pair<K>(nv, kp, s0 + i, s_src[m] + t);
        else k0 = K::eval32(R0, a32, p32);
        a0 = fmaf(k0, sq[o + t], a0);
      }
      acc += (double)a0 + (double)a1;
    }
  }
  red[g * NT + i] = acc;
  __syncthreads();
  if (g == 0 && i < n) {
    double s = ys[s0 + i];
    for (int h = 0; h < G; ++h) s += red[h * NT + i];
    ys[s0 + i] = s;
  }
}

template <class K>
struct P2p32Run {
  static void run(const NearView& nv, const KernelParams& kp, const float* qs32, double* ys, cudaStream_t s) {
    // one group: every thread sums all of its target's source leaves (the
    // FP32 entries are cheap, so splitting the leaves over groups only adds
    // imbalance and a reduction: 1.12 vs 1.62 ms at 1M uniform points, log)
    P2pShape sh = p2p_shape(nv.nmax);
    sh.g = 1;
    sh.threads = sh.nt;
    size_t smem = (size_t)9 * nv.nmax * (sizeof(float2) + sizeof(float)) + 16 + sizeof(double) * sh.threads;
    allow_smem(k_p2p32<K>, smem);
    k_p2p32<K><<<(int)nv.nleaf, sh.threads, smem, s>>>(nv, kp, qs32, ys, sh.nt, sh.g);
    AFMM_LAUNCH_CHECK();
  }
};

}  // namespace mixed_detail

}  // namespace afmm
