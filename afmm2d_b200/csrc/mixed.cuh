// Mixed-precision matvec (FP32 apply with FP64 where it matters); see mixed.cu.
#pragma once
#include <stdint.h>

#include <vector>

#include "afmm_internal.cuh"
#include "fmm.cuh"

namespace afmm {

struct MixedState {
  bool ready = false;
  size_t host_cap = 0;      // RHS capacity of the staging buffers below
  double* d_qin = nullptr;  // N x host_cap staging for host inputs
  double* d_yout = nullptr; // N x host_cap staging for host outputs
  int rhs_cap = 0;          // RHS capacity of qs32 / ys
  float* qs32 = nullptr;    // sorted charges (FP32)
  double* qs = nullptr;     // sorted charges (FP64)
  double* ys = nullptr;     // sorted potentials (FP64)
  double2* leaf_anchor = nullptr;
  float* leaf_span = nullptr;
  float2* rel = nullptr;    // sorted point minus its leaf anchor (FP32)
};

// Buffers of the batched path (kBatchMax right-hand sides per pass).
constexpr int kBatchMax = 16;
struct BatchState {
  bool ready = false;
  double* qs = nullptr;     // sorted charges, point-major N x kBatchMax
  uint2* qhl = nullptr;     // TF32 high / low parts of the FP32-rounded charges, interleaved
  double* ys = nullptr;     // sorted potentials, point-major
  double* qhat[kMaxLevels] = {nullptr};
  double* yhat[kMaxLevels] = {nullptr};
  const double** d_qhat_lv = nullptr;  // device copies indexed by level - 2
  double** d_yhat_lv = nullptr;
  int* err_host = nullptr;  // host-mapped flag set by a kernel whose bounded wait gave up
  int* err_dev = nullptr;   // its device address
  // The near field runs on its own lower-priority stream beside the far
  // field, into ys_near (zeroed per pass); the scatter adds it to ys.
  double* ys_near = nullptr;
  cudaStream_t s_near = nullptr;
  cudaEvent_t ev_q = nullptr, ev_near = nullptr;
  ~BatchState() {
    if (err_host) cudaFreeHost(err_host);
    if (ev_q) cudaEventDestroy(ev_q);
    if (ev_near) cudaEventDestroy(ev_near);
    if (s_near) cudaStreamDestroy(s_near);
  }
};
void batch_reserve(const MatvecPlan& p, BatchState& bs, DevArena& arena, cudaStream_t s);
// The M2L stage alone of a batched pass of rc columns (on the batch buffers'
// current outgoing charges); returns the launches made.
int m2l_batched(const MatvecPlan& p, BatchState& bs, int rc, int fp64, cudaStream_t s);

// Byte-plane copy of one level's fixed-point blocks for the integer
// tensor-core M2L (m2l_i8_k.cuh); v.m2l_s and v.m2l_s_off must be set.
void m2l_slice(const LevelView& v, cudaStream_t s);
// The near-field stage alone of a batched pass of rc columns (on the batch
// buffers' current charges); returns the launches made.
int p2p_batched(const MatvecPlan& p, MixedState& ms, BatchState& bs, int rc, int fp64, cudaStream_t s);
// y = K q for nrhs > 1 columns in passes of 4, 8 or 16 right-hand sides.
// fp64 = 1: FP64 throughout (FP64 near field on the tensor cores), passes of 8
// or 16 columns.
void matvec_batched(const MatvecPlan& p, MixedState& ms, BatchState& bs, const double* q, int64_t ldq, double* y,
                    int64_t ldy, int nrhs, int fp64, cudaStream_t s, StageTimer* tm, int64_t* launches);

// Builds the FP32 operators and anchors after assembly.
void mixed_setup(MatvecPlan& p, std::vector<LevelDev>& lv, MixedState& ms, DevArena& arena, cudaStream_t s,
                 int64_t* launches);
void mixed_reserve_io(MixedState& ms, int N, int nrhs, DevArena& arena);
void mixed_reserve(MixedState& ms, int N, int nrhs, DevArena& arena);
// y = K q for nrhs columns (q column c at q + c*ldq), original order, device pointers.
void matvec_mixed(const MatvecPlan& p, MixedState& ms, const double* q, int64_t ldq, double* y, int64_t ldy, int nrhs,
                  cudaStream_t s, StageTimer* tm, int64_t* launches);

}  // namespace afmm
