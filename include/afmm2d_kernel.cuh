/*
 * afmm2d_kernel.cuh -- user kernels for the B200 AFMM2D engine.
 *
 * The reference's plug-in point is a user-defined
 * userkernel::getMatrixEntry(i, j) (include/kernel.hpp:23,58, defined out of
 * line by the user as in examples/testAFMM2D.cpp:9-20).  Here a kernel is a
 * functor of the squared distance R2 between two points, compiled in a CUDA
 * translation unit of the user's own (nvcc -gencode
 * arch=compute_100a,code=sm_100a, linked against libafmm2d.so), with
 *
 *   struct MyKernel {
 *     static constexpr int id = AFMM_KERNEL_USER_FIRST + k;  // its kernel id
 *     // value at R2 = 0 (the diagonal)
 *     __device__ static double at_zero(const afmm::KernelParams& p);
 *     // setup arithmetic: the reference's operation order, IEEE rounding, no
 *     // FMA contraction (__dadd_rn, __dmul_rn, __ddiv_rn, __dsqrt_rn); its
 *     // values decide ACA pivots and ranks
 *     __device__ static double eval_exact(double R2, const afmm::KernelParams& p);
 *     // fast FP64 form for the matvec
 *     __device__ static double eval(double R2, const afmm::KernelParams& p);
 *     // FP32 form (mixed precision), and the form for R2 > 0 normal
 *     __device__ static float eval32(float R2, float a, float param);
 *     __device__ static float eval32_pos(float R2, float a, float param);
 *   };
 *   AFMM_REGISTER_KERNEL(MyKernel)
 *
 * p.a is the smallest box size 2^-nLevels (the reference's `a`,
 * src/AFMM2DTree.cpp:19) and p.param the first entry of afmm_create's
 * kparams (0.01 when absent).  Loading the unit's library registers the
 * kernel; afmm_create(..., MyKernel::id, ...) then uses it for every stage.
 */
#ifndef AFMM2D_KERNEL_CUH
#define AFMM2D_KERNEL_CUH

#include "afmm2d.h"
#include "../afmm2d_b200/csrc/stages_k.cuh"

#define AFMM_REGISTER_KERNEL(FUNCTOR)                                                                       \
  namespace {                                                                                               \
  const ::afmm::KernelTable afmm_kernel_table_##FUNCTOR = ::afmm::make_kernel_table<FUNCTOR>(#FUNCTOR);    \
  const afmm_status afmm_kernel_registered_##FUNCTOR =                                                      \
      afmm_register_kernel(FUNCTOR::id, &afmm_kernel_table_##FUNCTOR, sizeof(::afmm::KernelTable),          \
                           ::afmm::kKernelTableAbi);                                                        \
  }

#endif /* AFMM2D_KERNEL_CUH */
