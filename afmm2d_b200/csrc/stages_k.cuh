// Every kernel-templated stage, and make_kernel_table<K>(): the launchers of
// all of them instantiated for one kernel functor K.  Included by the
// built-in kernels' translation units (kernels_*.cu) and by user kernel
// translation units (include/afmm2d_kernel.cuh).
#pragma once
#include "aca_k.cuh"
#include "batched_k.cuh"
#include "capi_k.cuh"
#include "fmm_k.cuh"
#include "kernel_table.cuh"
#include "mixed_k.cuh"
#include "p2p_tc_k.cuh"
#include "set_k.cuh"

namespace afmm {

template <class K>
KernelTable make_kernel_table(const char* name) {
  KernelTable t;
  t.name = name;
  t.m2l_assemble = &fmm_detail::M2lAssembleRun<K>::run;
  t.p2p64 = &fmm_detail::P2p64Run<K>::run;
  t.m2l_otf = &mixed_detail::M2lOtfRun<K>::run;
  t.p2p32 = &mixed_detail::P2p32Run<K>::run;
  t.m2l_otf_mma[0] = &batched_detail::m2l_otf_batched<K, 8>;
  t.m2l_otf_mma[1] = &batched_detail::m2l_otf_batched<K, 16>;
  t.p2p_mma[0] = &batched_detail::p2p_mma_batched<K, 8>;
  t.p2p_mma[1] = &batched_detail::p2p_mma_batched<K, 16>;
  t.p2p_dmma[0] = &batched_detail::p2p_dmma_batched<K, 8>;
  t.p2p_dmma[1] = &batched_detail::p2p_dmma_batched<K, 16>;
  t.p2p_tc16 = &p2p_tc_detail::p2p_tc_batched16<K>;
  t.aca_occupancy = &aca_detail::AcaLaunch<K>::occupancy;
  t.aca_run = &aca_detail::AcaLaunch<K>::run;
  t.l2p_run = &aca_detail::L2pRun<K>::run;
  t.dense_rows = &capi_detail::DenseRun<K>::run;
  t.kernel_pairs = &capi_detail::PairsRun<K>::run;
  t.set_p2p_prepare = &set_detail::SetP2pRun<K>::prepare;
  t.set_p2p_run = &set_detail::SetP2pRun<K>::run;
  return t;
}

}  // namespace afmm
