// Kernel-templated diagnostics of the C ABI: direct FP64 rows (the error
// check) and kernel entries of point pairs, instantiated once per kernel
// functor by the kernel tables (kernel_table.cuh).
#pragma once
#include "fmm.cuh"

namespace afmm {

namespace capi_detail {

// Direct FP64 potentials at selected sorted points, Neumaier-compensated.
template <class K>
__global__ void k_dense_rows(const double2* __restrict__ pts, const double* __restrict__ qs, int N,
                             const int32_t* __restrict__ rows, KernelParams kp, double* out) {
  const int t = blockIdx.x;
  const double2 xi = pts[rows[t]];
  double s = 0.0, c = 0.0;
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    double v = K::eval(r2_exact(xi.x, xi.y, pts[j].x, pts[j].y), kp) * qs[j];
    double tt = s + v;
    c += (fabs(s) >= fabs(v)) ? ((s - tt) + v) : ((v - tt) + s);
    s = tt;
  }
  __shared__ double ss[256], sc[256];
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0, Cc = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) {
      double v = ss[i];
      double tt = S + v;
      Cc += (fabs(S) >= fabs(v)) ? ((S - tt) + v) : ((v - tt) + S);
      S = tt;
      Cc += sc[i];
    }
    out[t] = S + Cc;
  }
}

template <class K>
struct DenseRun {
  static void run(const double2* pts, const double* qs, int N, const int32_t* rows, int nrows, KernelParams kp,
                  double* out, cudaStream_t s) {
    k_dense_rows<K><<<nrows, 256, 0, s>>>(pts, qs, N, rows, kp, out);
    AFMM_LAUNCH_CHECK();
  }
};

template <class K>
__global__ void k_kernel_pairs(const double2* __restrict__ a, const double2* __restrict__ b, long n, KernelParams kp,
                               int mode, double* out) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double2 p = a[t], q = b[t];
  if (mode == 0) {
    out[t] = K::eval_exact(r2_exact(p.x, p.y, q.x, q.y), kp);
  } else if (mode == 1) {
    double dx = p.x - q.x, dy = p.y - q.y;
    out[t] = K::eval(dx * dx + dy * dy, kp);
  } else {
    float dx = (float)(p.x - q.x), dy = (float)(p.y - q.y);
    out[t] = (double)K::eval32(fmaf(dx, dx, dy * dy), (float)kp.a, (float)kp.param);
  }
}

template <class K>
struct PairsRun {
  static void run(const double2* a, const double2* b, long n, KernelParams kp, int mode, double* out) {
    k_kernel_pairs<K><<<(int)((n + 255) / 256), 256>>>(a, b, n, kp, mode, out);
    AFMM_LAUNCH_CHECK();
  }
};

}  // namespace capi_detail

}  // namespace afmm
