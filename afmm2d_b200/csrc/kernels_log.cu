// Stage table of the built-in kernel KLog (afmm_internal.cuh).
#include "stages_k.cuh"

namespace afmm {

const KernelTable& builtin_table_log() {
  static const KernelTable t = make_kernel_table<KLog>("log");
  return t;
}

}  // namespace afmm
