// Device helpers shared by the batched sweeps (batched.cu) and the
// kernel-templated batched stages (batched_k.cuh).
#pragma once
#include <stdint.h>

#include <cuda_runtime.h>

namespace afmm {

namespace batched_common {

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo with both parts TF32 (hi: 11 significant bits, lo: the next 11).
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

template <int RC>
__device__ __forceinline__ void load_vec(const double* __restrict__ p, double (&v)[RC]) {
  const double2* p2 = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int c = 0; c < RC / 2; ++c) {
    double2 t = p2[c];
    v[2 * c] = t.x;
    v[2 * c + 1] = t.y;
  }
}

template <int RC>
__device__ __forceinline__ void store_vec(double* p, const double (&v)[RC]) {
  double2* p2 = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int c = 0; c < RC / 2; ++c) p2[c] = make_double2(v[2 * c], v[2 * c + 1]);
}

// FP64 MMA m8n8k4 (D = A B + C; A 8x4 row-major, B 4x8 column-major): lane l
// holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) .. 2(l%4)+1].
__device__ __forceinline__ void mma_f64_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// FP64 MMA m16n8k4 (sm_90 and later; D = A B + C, A 16x4, B 4x8): lane
// l = 4g + t holds A[g][t], A[g+8][t]; B[t][g]; D[g][2t], D[g][2t+1],
// D[g+8][2t], D[g+8][2t+1].
__device__ __forceinline__ void mma_f64_16x8x4(double (&c)[4], double a0, double a1, double b) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(b));
}

}  // namespace batched_common

using namespace batched_common;

}  // namespace afmm
