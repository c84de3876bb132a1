// A user kernel defined outside the library, as a reference user defines
// userkernel::getMatrixEntry out of line (examples/testAFMM2D.cpp:9-20): the
// inverse multiquadric K(r) = 1 / sqrt(r^2 + c), c = kparams[0].  Built into
// its own shared library (afmm2d_b200.build.build_kernel_plugin); loading
// that library registers the kernel under id AFMM_KERNEL_USER_FIRST.
#include "afmm2d_kernel.cuh"

struct InverseMultiquadric {
  static constexpr int id = AFMM_KERNEL_USER_FIRST;
  // the diagonal (R2 = 0)
  __device__ __forceinline__ static double at_zero(const afmm::KernelParams& p) {
    return __ddiv_rn(1.0, __dsqrt_rn(p.param));
  }
  // reference arithmetic: 1.0 / sqrt(R2 + c), IEEE rounding, no contraction
  __device__ __forceinline__ static double eval_exact(double R2, const afmm::KernelParams& p) {
    return __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(R2, p.param)));
  }
  __device__ __forceinline__ static double eval(double R2, const afmm::KernelParams& p) { return rsqrt(R2 + p.param); }
  __device__ __forceinline__ static float eval32(float R2, float, float c) {
    const float x = R2 + c;
    const float y = rsqrtf(x);
    return fmaf(0.5f * y, fmaf(-x * y, y, 1.0f), y);
  }
  __device__ __forceinline__ static float eval32_pos(float R2, float a, float c) { return eval32(R2, a, c); }
};

AFMM_REGISTER_KERNEL(InverseMultiquadric)
