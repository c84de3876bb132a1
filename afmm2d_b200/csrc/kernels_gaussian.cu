// Stage table of the built-in kernel KGaussian (afmm_internal.cuh).
#include "stages_k.cuh"

namespace afmm {

const KernelTable& builtin_table_gaussian() {
  static const KernelTable t = make_kernel_table<KGaussian>("gaussian");
  return t;
}

}  // namespace afmm
