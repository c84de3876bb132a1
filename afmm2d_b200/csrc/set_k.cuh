// Kernel-templated stage of many-problem sets: the fused FP64 near field,
// instantiated once per kernel functor by the kernel tables
// (kernel_table.cuh).
#pragma once
#include "set.cuh"

namespace afmm {

namespace set_detail {

// Near field: one CTA per leaf of every problem, each problem with its own
// (NT, G) shape so the group sums add in the same order as its own launch.
template <class K>
__global__ void k_set_p2p64(SetDev d, SetSegs sg) {
  extern __shared__ __align__(16) unsigned char smem[];
  const long g = blockIdx.x;
  const int s = seg_of(sg, g);
  const int p = sg.prob[s];
  const int2 sh = d.p2p[p];
  p2p64_leaf<K>(d.nv[p], d.kp[p], d.qs[p], d.ys[p], sh.x, sh.y, g - sg.first[s], smem);
}

template <class K>
struct SetP2pRun {
  static void prepare(size_t smem) { allow_smem(k_set_p2p64<K>, smem); }
  static void run(const SetPlan& sp, cudaStream_t s) {
    k_set_p2p64<K><<<(int)sp.p2p.total, sp.p2p_threads, sp.p2p_smem, s>>>(sp.dev, sp.p2p);
    AFMM_LAUNCH_CHECK();
  }
};

}  // namespace set_detail

}  // namespace afmm
