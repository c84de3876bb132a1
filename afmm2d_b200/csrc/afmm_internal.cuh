// Internal declarations shared by the AFMM2D B200 kernels and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/afmm2d.h"
#include "exact_math.cuh"
#include "fast_math.cuh"

namespace afmm {

// ------------------------------------------------------------------ errors
struct Error {
  afmm_status status;
  std::string msg;
};

#define AFMM_CUDA(call)                                                                      \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      cudaGetLastError(); /* clear a non-sticky error so later checks do not report it */    \
      throw ::afmm::Error{AFMM_CUDA_ERR, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    }                                                                                        \
  } while (0)

#define AFMM_LAUNCH_CHECK() AFMM_CUDA(cudaGetLastError())

// ----------------------------------------------------------------- kernels
// User kernels of the reference are `double userkernel::getMatrixEntry(i, j)`
// (include/kernel.hpp:58) reading particles_X[i], particles_X[j] and the
// smallest box size `a` (src/AFMM2DTree.cpp:19).  Here a kernel is a functor
// of the two points' coordinates.  `eval_exact` reproduces the reference's
// double arithmetic operation by operation (no FMA contraction, IEEE sqrt and
// division, correctly rounded log/exp from exact_math.cuh) and is used
// wherever results steer pivoting (ACA, L2P, M2L blocks).  `eval` is the fast FP64 form for the matvec, `eval32` the FP32
// form for the mixed-precision matvec (R2 formed from coordinates relative to
// box anchors; the third argument is the Gaussian parameter).
// `eval32_pos` is `eval32` for R2 at or above the near-field fallback
// threshold (R2 > 0 and normal): hardware approximations (flush-to-zero
// rsqrt, lg2, ex2) with relative error near FP32 rounding, for the TF32x3
// tensor-core near field (whose operand split allows 2^-21).
struct KernelParams {
  int id;
  double a;              // 2^-L
  double param;          // Gaussian: exp(-R2 / param)
  double a2;             // a * a
  double inv_a2;         // 1 / (a * a)
  double neg_inv_param;  // -1 / param (the FP64 Gaussian multiplies instead of dividing)
};

inline KernelParams make_kernel_params(int id, double a, double param) {
  return KernelParams{id, a, param, a * a, 1.0 / (a * a), -1.0 / param};
}

__device__ __forceinline__ double r2_exact(double xi, double yi, double xj, double yj) {
  double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj);
  return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// One over r, scaled (examples/testAFMM2D.cpp:9-20): R < a ? R/a : a/R.
struct KOneOverRScaled {
  static constexpr int id = AFMM_KERNEL_ONE_OVER_R_SCALED;
  __device__ __forceinline__ static double at_zero(const KernelParams&) { return 0.0; }
  __device__ __forceinline__ static double eval_exact(double R2, const KernelParams& p) {
    double R = __dsqrt_rn(R2);
    return (R < p.a) ? __ddiv_rn(R, p.a) : __ddiv_rn(p.a, R);
  }
  __device__ __forceinline__ static double eval(double R2, const KernelParams& p) {
    double R = sqrt(R2);
    return (R < p.a) ? R / p.a : p.a / R;
  }
  __device__ __forceinline__ static float eval32(float R2, float a, float) {
    float R = sqrtf(R2);
    return (R < a) ? __fdiv_rn(R, a) : __fdiv_rn(a, R);
  }
  __device__ __forceinline__ static float eval32_pos(float R2, float a, float p) { return eval32(R2, a, p); }
};


// log(r) with the diagonal convention (examples/tutorial.cpp:22-35).
struct KLog {
  static constexpr int id = AFMM_KERNEL_LOG;
  __device__ __forceinline__ static double at_zero(const KernelParams&) { return 0.0; }
  __device__ __forceinline__ static double eval_exact(double R2, const KernelParams& p) {
    if (R2 < 1e-10) return 0.0;
    const double l = log_cr(R2);
    if (R2 < __dmul_rn(p.a, p.a)) return __ddiv_rn(__ddiv_rn(__dmul_rn(__dmul_rn(0.5, R2), l), p.a), p.a);
    return __dmul_rn(0.5, l);
  }
  // a = 2^-L, so dividing by a twice is the exact scaling by 1/a^2: both
  // branches are evaluated without divergence and selected (same bits as
  // 0.5*R2*l/a/a and 0.5*l); l is the table-driven log (within one ulp)
  __device__ __forceinline__ static double eval(double R2, const KernelParams& p) {
    const double l = log_tang(R2);
    const double near = ((0.5 * R2) * l) * p.inv_a2;
    const double r = R2 < p.a2 ? near : 0.5 * l;
    return R2 < 1e-10 ? 0.0 : r;
  }
  __device__ __forceinline__ static float eval32(float R2, float a, float) {
    if (R2 < 1e-10f) return 0.0f;
    float l = logf(R2);
    if (R2 < a * a) return __fdiv_rn(0.5f * R2 * l, a * a);
    return 0.5f * l;
  }
  // ln(R2) = lg2(R2) ln 2; lg2.approx has absolute error ~2^-22.  a = 2^-L,
  // so 1/a^2 is an exact power of two (loop-invariant): the near branch
  // multiplies instead of dividing
  __device__ __forceinline__ static float eval32_pos(float R2, float a, float) {
    if (R2 < 1e-10f) return 0.0f;
    const float l = __log2f(R2) * 0.693147180559945309f;
    if (R2 < a * a) return (0.5f * R2 * l) * __frcp_rn(a * a);
    return 0.5f * l;
  }
};

// 1/r with 0 at r = 0.
struct KOneOverR {
  static constexpr int id = AFMM_KERNEL_ONE_OVER_R;
  __device__ __forceinline__ static double at_zero(const KernelParams&) { return 0.0; }
  __device__ __forceinline__ static double eval_exact(double R2, const KernelParams&) {
    if (R2 == 0.0) return 0.0;
    return __ddiv_rn(1.0, __dsqrt_rn(R2));
  }
  __device__ __forceinline__ static double eval(double R2, const KernelParams&) {
    return R2 == 0.0 ? 0.0 : rsqrt(R2);
  }
  // rsqrtf refined by one Newton-Raphson step y += y/2 (1 - R2 y^2)
  __device__ __forceinline__ static float eval32(float R2, float, float) {
    if (R2 == 0.0f) return 0.0f;
    float y = rsqrtf(R2);
    float e = fmaf(-R2 * y, y, 1.0f);
    return fmaf(0.5f * y, e, y);
  }
  // rsqrt.approx alone (relative error ~2^-23): the tensor-core near field
  // splits every entry into two 11-bit TF32 parts (error up to 2^-21), so a
  // Newton step would not change its result
  __device__ __forceinline__ static float eval32_pos(float R2, float, float) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(R2));
    return y;
  }
};

// Gaussian exp(-R2/param) (1 on the diagonal).
struct KGaussian {
  static constexpr int id = AFMM_KERNEL_GAUSSIAN;
  __device__ __forceinline__ static double at_zero(const KernelParams&) { return 1.0; }
  __device__ __forceinline__ static double eval_exact(double R2, const KernelParams& p) {
    return exp_cr(-__ddiv_rn(R2, p.param));
  }
  // R2 * (-1/param) is within one rounding of -R2/param (the setup's
  // eval_exact keeps the division)
  __device__ __forceinline__ static double eval(double R2, const KernelParams& p) {
    return exp_tang(R2 * p.neg_inv_param);
  }
  __device__ __forceinline__ static float eval32(float R2, float, float param) {
    return expf(-__fdiv_rn(R2, param));
  }
  // exp(-R2/param) = 2^(R2 c), c = -log2(e)/param (loop-invariant): one
  // multiply and ex2.approx (relative error ~2^-22, inside the TF32 split)
  __device__ __forceinline__ static float eval32_pos(float R2, float, float param) {
    const float c = __fdiv_rn(-1.44269504088896341f, param);
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(R2 * c));
    return y;
  }
};

// ------------------------------------------------------------- allocation
// Every device allocation of the library goes through DevArena::alloc, which
// counts it here (read by afmm_get_device_alloc_count).
std::atomic<int64_t>& device_alloc_counter();

// Device allocations owned by a handle; freed together.
struct DevArena {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  template <class T>
  T* alloc(size_t n) {
    if (n == 0) n = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error{AFMM_OOM, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed"};
    }
    device_alloc_counter().fetch_add(1, std::memory_order_relaxed);
    ptrs.push_back(p);
    bytes += n * sizeof(T);
    return (T*)p;
  }
  void release(void* p) {
    for (auto& q : ptrs)
      if (q == p) {
        cudaFree(q);
        q = nullptr;
      }
  }
  ~DevArena() {
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

// One grow-only device buffer carved into aligned pieces, reused by a
// sequence of launches (the ACA levels of one assemble): an allocation only
// when a request exceeds the capacity, instead of a cudaMalloc / cudaFree
// pair (a device-wide synchronisation) per level.
struct DevScratch {
  void* base = nullptr;
  size_t cap = 0, used = 0;
  // Makes the buffer at least `bytes` long (contents not kept) and restarts carving.
  void reserve(size_t bytes) {
    used = 0;
    if (bytes <= cap) return;
    if (base) cudaFree(base);
    base = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error{AFMM_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed"};
    }
    device_alloc_counter().fetch_add(1, std::memory_order_relaxed);
    cap = bytes;
  }
  // The next n elements of T (256-byte aligned); reserve() must have made room.
  template <class T>
  T* take(size_t n) {
    const size_t off = (used + 255) & ~(size_t)255;
    if (off + n * sizeof(T) > cap) throw Error{AFMM_BAD_ARG, "scratch request beyond its reservation"};
    used = off + n * sizeof(T);
    return reinterpret_cast<T*>(static_cast<unsigned char*>(base) + off);
  }
  // Bytes that pieces of the given sizes need together.
  static size_t need(std::initializer_list<size_t> sizes) {
    size_t t = 0;
    for (size_t s : sizes) t = ((t + 255) & ~(size_t)255) + s;
    return t + 256;
  }
  ~DevScratch() {
    if (base) cudaFree(base);
  }
};

// ------------------------------------------------------------- tree layout
// Per level j (4^j boxes, quadtree numbering k: parent k/4, children 4k+c).
// Rows per warp of the FP64 tensor-core sweeps (five 8-row tiles).
constexpr int kChunkRows = 40;

struct LevelDev {
  long nbox = 0;
  int32_t* il = nullptr;        // nbox*40: inner slots 0..15 then outer 0..23, -1 = none
  int32_t* nbr = nullptr;       // nbox*8 neighbour slots (leaf level)
  int32_t* node_off = nullptr;  // nbox+1 prefix over box node counts
  int32_t* node_ids = nullptr;  // node lists (sorted-point ids)
  int32_t* rank = nullptr;      // nbox
  int32_t* skel_box = nullptr;  // skeleton row -> box
  int32_t* node_box = nullptr;  // node row -> box
  int32_t* grp_box = nullptr;   // row group (<= 8 rows of one box) -> box
  int32_t* grp_row = nullptr;   // row group -> first skeleton row
  long ngroups = 0;
  int32_t* cgrp_box = nullptr;  // row chunk (<= kChunkRows rows of one box) -> box
  int32_t* cgrp_row = nullptr;  // row chunk -> first skeleton row
  long ncgroups = 0;
  int32_t* ncgrp_box = nullptr;  // node-row chunk (<= kChunkRows node rows of one box) -> box
  int32_t* ncgrp_row = nullptr;  // node-row chunk -> first node row
  long nncgroups = 0;
  int32_t* wgrp_box = nullptr;   // row chunk (<= 32 skeleton rows of one box: a warp's lanes) -> box
  int32_t* wgrp_row = nullptr;   // row chunk -> first skeleton row
  long nwgroups = 0;
  int32_t* nwgrp_box = nullptr;  // node-row chunk (<= 32 node rows of one box) -> box
  int32_t* nwgrp_row = nullptr;  // node-row chunk -> first node row
  long nnwgroups = 0;
  int32_t* ptile_par = nullptr;  // parent row tile (<= 128 rows of the parent's four children) -> parent
  int32_t* ptile_row = nullptr;  // parent row tile -> first row in the children's concatenated rows
  long nptiles = 0;
  int32_t* tile_box = nullptr;  // row tile (<= 128 skeleton rows of one box, multiple of 8) -> box
  int32_t* tile_row = nullptr;  // row tile -> first row within the box
  long ntiles = 0;
  int32_t* skel_off = nullptr;  // nbox+1 prefix over ranks
  int32_t* skel_ids = nullptr;  // skeleton (incoming check points), sorted-point ids
  int32_t* cpiv_ids = nullptr;  // pivot columns (incoming charge points)
  double2* skel_xy = nullptr;   // skeleton coordinates
  int64_t* l2p_off = nullptr;   // nbox+1 prefix over n_b*r_b
  double* l2p = nullptr;        // per box n_b x r_b, column-major (row index fastest)
  double* l2p_rm = nullptr;     // the same, row-major (rank index fastest)
  int64_t* m2l_off = nullptr;   // nbox+1 prefix over sum_slots r_b*r_c
  double* m2l = nullptr;        // per box, per valid slot, block r_b x r_c column-major
  // The same blocks in 32-bit fixed point (the mixed-precision paths): entry
  // e of block (b, slot s) is (u - 2^31) * 2^k with u = m2l_q[e] and 2^k the
  // block's power-of-two scale; m2l_dec[b * 40 + s] = (2^k, -(2^52 + 2^31) 2^k)
  // decodes it with one FMA (see decode_q32).
  uint32_t* m2l_q = nullptr;
  double2* m2l_dec = nullptr;
  // The fixed-point blocks as byte planes for the integer tensor-core M2L
  // (m2l_i8_k.cuh): box b's blocks start at m2l_s + m2l_s_off[b].  The
  // charges' byte planes of a pass (qs8, per box from qs8_off[b] x 2 KB) with
  // their per-column exponents and sums.
  unsigned char* m2l_s = nullptr;
  int64_t* m2l_s_off = nullptr;
  unsigned char* qs8 = nullptr;
  int32_t* qs8_off = nullptr;
  int32_t* qs_exp = nullptr;
  int64_t* qs_sum = nullptr;
  double* qhat = nullptr;       // outgoing charges, skel_off layout
  double* yhat = nullptr;       // incoming potentials, skel_off layout
  // host copies
  std::vector<int32_t> h_rank, h_skel_off;
  std::vector<int32_t> h_node_off;
  std::vector<int64_t> h_l2p_off, h_m2l_off;
  int n1max = 0, rmax = 0;
  long total_rank = 0;
};

}  // namespace afmm
