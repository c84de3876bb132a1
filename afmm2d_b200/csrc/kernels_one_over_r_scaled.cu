// Stage table of the built-in kernel KOneOverRScaled (afmm_internal.cuh).
#include "stages_k.cuh"

namespace afmm {

const KernelTable& builtin_table_one_over_r_scaled() {
  static const KernelTable t = make_kernel_table<KOneOverRScaled>("one_over_r_scaled");
  return t;
}

}  // namespace afmm
