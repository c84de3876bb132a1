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
};

// Builds the FP32 operators and anchors after assembly.
void mixed_setup(MatvecPlan& p, std::vector<LevelDev>& lv, MixedState& ms, DevArena& arena, cudaStream_t s,
                 int64_t* launches);
void mixed_reserve_io(MixedState& ms, int N, int nrhs, DevArena& arena);
// y = K q for nrhs columns (q column c at q + c*ldq), original order, device pointers.
void matvec_mixed(const MatvecPlan& p, MixedState& ms, const double* q, int64_t ldq, double* y, int64_t ldy, int nrhs,
                  cudaStream_t s, StageTimer* tm, int64_t* launches);

}  // namespace afmm
