// Stage table of the built-in kernel KOneOverR (afmm_internal.cuh).
#include "stages_k.cuh"

namespace afmm {

const KernelTable& builtin_table_one_over_r() {
  static const KernelTable t = make_kernel_table<KOneOverR>("one_over_r");
  return t;
}

}  // namespace afmm
