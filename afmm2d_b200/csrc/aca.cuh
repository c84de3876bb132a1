// K3/K4: ACA skeletonisation and L2P of one level (see aca.cu).
#pragma once
#include <stdint.h>

#include <vector>

#include "afmm_internal.cuh"

namespace afmm {

struct AcaLevelIn {
  long nbox;
  const double2* pts;       // sorted points
  const int32_t* node_off;  // nbox + 1
  const int32_t* node_ids;
  const int32_t* il;        // nbox * 40
  std::vector<int32_t> h_node_off;
  int n1max, n2max;
  double tol;
  KernelParams kp;
  int32_t* rank_out;        // nbox (device)
};

struct AcaLevelOut {
  int rcap = 0, rmax = 0, cluster = 0, clusters = 0;
  int32_t* rank = nullptr;
  int32_t* skel_off = nullptr;
  int64_t* l2p_off = nullptr;
  int32_t* skel_ids = nullptr;
  int32_t* cpiv_ids = nullptr;
  double2* skel_xy = nullptr;
  double* l2p = nullptr;  // per box n x r, column-major
  std::vector<int32_t> h_rank, h_skel_off;
  std::vector<int64_t> h_l2p_off;
  double aca_s = 0, l2p_s = 0;  // wall clock of the two phases
};

// Runs the ACA and L2P kernels for one level; outputs are allocated in
// `arena`.  Synchronises `s`.
void aca_level(const AcaLevelIn& in, AcaLevelOut& out, DevArena& arena, cudaStream_t s, int64_t* launches);

}  // namespace afmm
