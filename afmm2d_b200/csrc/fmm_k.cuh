// Kernel-templated stages of the FP64 path: the M2L blocks (K5) and the
// FP64 near field (K9), instantiated once per kernel functor by the kernel
// tables (kernel_table.cuh).
#pragma once
#include "fmm.cuh"

namespace afmm {

namespace fmm_detail {

// ------------------------------------------------------------ M2L blocks
// M2L[b][c] = K(R_b, R_c) for every valid inner/outer slot of b, in slot
// order (src/AFMM2DTree.cpp:1070-1097), stored column-major r_b x r_c.
template <class K>
__global__ void k_m2l_assemble(LevelView v, KernelParams kp) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  if (r == 0) return;
  double* out = v.m2l + v.m2l_off[b];
  const double2* xb = v.skel_xy + v.skel_off[b];
  long off = 0;
  for (int s = 0; s < 40; ++s) {
    int c = v.il[b * 40 + s];
    if (c < 0) continue;
    const int rc = v.rank[c];
    const double2* xc = v.skel_xy + v.skel_off[c];
    for (int e = threadIdx.x; e < r * rc; e += blockDim.x) {
      int cc = e / r, i = e - cc * r;
      out[off + e] = K::eval_exact(r2_exact(xb[i].x, xb[i].y, xc[cc].x, xc[cc].y), kp);
    }
    off += (long)r * rc;
  }
}

template <class K>
struct M2lAssembleRun {
  static void run(const LevelView& v, const KernelParams& kp, cudaStream_t s) {
    k_m2l_assemble<K><<<(int)v.nbox, 128, 0, s>>>(v, kp);
    AFMM_LAUNCH_CHECK();
  }
};

// Near field (src/AFMM2DTree.cpp:1199-1213): one CTA per leaf.
template <class K>
__global__ void k_p2p64(NearView nv, KernelParams kp, const double* __restrict__ qs, double* __restrict__ ys, int NT,
                        int G) {
  extern __shared__ __align__(16) unsigned char smem[];
  p2p64_leaf<K>(nv, kp, qs, ys, NT, G, nv.leaf0 + blockIdx.x, smem);
}

template <class K>
struct P2p64Run {
  static void run(const NearView& nv, const KernelParams& kp, const double* qs, double* ys, cudaStream_t s) {
    P2pShape sh = p2p_shape(nv.nmax);
    size_t smem = (size_t)9 * nv.nmax * (sizeof(double2) + sizeof(double)) + sizeof(double) * sh.threads;
    allow_smem(k_p2p64<K>, smem);
    k_p2p64<K><<<(int)nv.nleaf, sh.threads, smem, s>>>(nv, kp, qs, ys, sh.nt, sh.g);
    AFMM_LAUNCH_CHECK();
  }
};

}  // namespace fmm_detail

}  // namespace afmm
