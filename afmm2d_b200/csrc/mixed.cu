// Mixed-precision matvec (placeholder until the FP32 kernels land).
#include "mixed.cuh"

namespace afmm {

void mixed_setup(MatvecPlan&, std::vector<LevelDev>&, MixedState& ms, DevArena&, cudaStream_t, int64_t*) {
  ms.ready = false;
}

void mixed_reserve_io(MixedState& ms, int N, int nrhs, DevArena& arena) {
  ms.d_qin = arena.alloc<double>((size_t)N * nrhs);
  ms.d_yout = arena.alloc<double>((size_t)N * nrhs);
  ms.host_cap = nrhs;
}

void matvec_mixed(const MatvecPlan&, MixedState&, const double*, int64_t, double*, int64_t, int, cudaStream_t,
                  StageTimer*, int64_t*) {
  throw Error{AFMM_BAD_ARG, "mixed precision is not available in this build"};
}

}  // namespace afmm
