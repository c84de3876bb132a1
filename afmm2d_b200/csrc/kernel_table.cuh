// Per-kernel function tables: every stage that evaluates the user kernel
// (userkernel::getMatrixEntry, include/kernel.hpp:58) is a template over a
// kernel functor K; a KernelTable holds the launchers of all of them
// instantiated for one K.  The built-in kernels' tables are compiled into the
// library (kernels_*.cu); a user kernel gets its table from a translation unit
// of the user's own that includes include/afmm2d_kernel.cuh and registers it
// with afmm_register_kernel (AFMM_REGISTER_KERNEL).  Kernel-independent code
// calls kernel_table(id).<stage>(...).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "aca.cuh"
#include "fmm.cuh"
#include "set.cuh"

namespace afmm {

// Bumped whenever KernelTable or an argument type of its launchers changes:
// a table compiled against other headers is refused at registration.
constexpr int kKernelTableAbi = 4;

// Fingerprint of the layouts of the launchers' argument types (sizes and a
// few field offsets), recorded in every table where it is compiled: a table
// whose launchers were compiled against headers with other layouts is
// refused at registration even when the version above was not bumped.
constexpr uint32_t layout_mix(uint32_t h, size_t v) { return (h ^ (uint32_t)v) * 16777619u; }
constexpr uint32_t kArgLayout = layout_mix(
    layout_mix(layout_mix(layout_mix(layout_mix(layout_mix(layout_mix(layout_mix(layout_mix(layout_mix(2166136261u,
    sizeof(LevelView)), offsetof(LevelView, m2l_q)), offsetof(LevelView, ptile_par)), sizeof(LevelSet)),
    offsetof(LevelSet, src)), sizeof(NearView)), sizeof(KernelParams)), sizeof(AcaArgs)), sizeof(L2pArgs)),
    sizeof(SetPlan));

struct KernelTable {
  int abi = kKernelTableAbi;
  uint32_t layout = kArgLayout;
  const char* name = nullptr;
  // M2L blocks K(R_b, R_c) of one level, setup arithmetic (fmm_k.cuh)
  void (*m2l_assemble)(const LevelView&, const KernelParams&, cudaStream_t) = nullptr;
  // FP64 near field, one column (fmm_k.cuh)
  void (*p2p64)(const NearView&, const KernelParams&, const double*, double*, cudaStream_t) = nullptr;
  // single-RHS mixed path: M2L on the fly (FP64), FP32 near field (mixed_k.cuh)
  void (*m2l_otf)(const LevelSet&, const KernelParams&, cudaStream_t) = nullptr;
  void (*p2p32)(const NearView&, const KernelParams&, const float*, double*, cudaStream_t) = nullptr;
  // batched passes (batched_k.cuh), [0] 8 / [1] 16 columns: M2L on the fly,
  // mixed near field, FP64 near field
  void (*m2l_otf_mma[2])(const LevelSet&, const KernelParams&, const double* const*, double* const*,
                         cudaStream_t) = {nullptr, nullptr};
  void (*p2p_mma[2])(const NearView&, const KernelParams&, const uint2*, double*, cudaStream_t) = {nullptr, nullptr};
  void (*p2p_dmma[2])(const NearView&, const KernelParams&, const double*, double*, cudaStream_t) = {nullptr, nullptr};
  // mixed near field of 16-column passes on tcgen05 tiles (p2p_tc_k.cuh);
  // leaves of at most 64 points; sets *err on a bounded-wait timeout
  void (*p2p_tc16)(const NearView&, const KernelParams&, const uint2*, double*, int L, int* err,
                   cudaStream_t) = nullptr;
  // ACA and L2P of one level (aca_k.cuh)
  void (*aca_occupancy)(int clusters, size_t smem, int* active) = nullptr;
  void (*aca_run)(const AcaArgs&, int cluster, int clusters, size_t smem, cudaStream_t) = nullptr;
  void (*l2p_run)(const L2pArgs&, size_t smem, bool global_factor, int grid, cudaStream_t) = nullptr;
  // diagnostics (capi_k.cuh): direct FP64 rows, entries of point pairs
  void (*dense_rows)(const double2*, const double*, int, const int32_t*, int, KernelParams, double*,
                     cudaStream_t) = nullptr;
  void (*kernel_pairs)(const double2*, const double2*, long, KernelParams, int, double*) = nullptr;
  // fused near field of a many-problem set (set_k.cuh)
  void (*set_p2p_prepare)(size_t smem) = nullptr;
  void (*set_p2p_run)(const SetPlan&, cudaStream_t) = nullptr;
};

// The table of a kernel id (built-in or registered); AFMM_BAD_ARG otherwise.
const KernelTable& kernel_table(int id);
bool kernel_known(int id);

// Built-in tables (kernels_*.cu).
const KernelTable& builtin_table_one_over_r_scaled();
const KernelTable& builtin_table_log();
const KernelTable& builtin_table_one_over_r();
const KernelTable& builtin_table_gaussian();

}  // namespace afmm
