// K3/K4: ACA skeletonisation and L2P of one level (see aca.cu).
#pragma once
#include <stdint.h>

#include <vector>

#include "afmm_internal.cuh"

namespace afmm {

// Launch parameters of the ACA kernel (aca_k.cuh) and of the L2P solve,
// shared by the level planner (aca.cu) and the kernel instantiations.
constexpr int ACA_T = 256;
constexpr int ACA_WARPS = ACA_T / 32;
enum { AR_ROWS = 0, AR_COLS, AR_V, AR_U, AR_XDOT, AR_SMALL, AR_OK, AR_XARG, AR_N };

struct AcaArgs {
  int nbox;
  const double2* pts;
  const int32_t* node_off;
  const int32_t* node_ids;
  const int32_t* il;
  double tol;
  KernelParams kp;
  int rcap;       // max rank stored per box
  int n1max;
  int chunk;      // columns per CTA
  int vcap;       // ranks of V held in shared memory
  int ucap;       // ranks of U held in shared memory
  double* vspill; // [cluster][C][rcap - vcap][chunk]
  double* uspill; // [cluster][C][rcap - ucap][n1max]
  // Placement of the per-CTA arrays: byte offset into shared memory when the
  // flag is set, else into this CTA's slot of `gscr` (gslot bytes per CTA).
  unsigned char* gscr;
  size_t gslot;
  size_t off[8];
  int in_smem[8];
  int32_t* rank_out;
  int32_t* rowpiv;  // nbox * rcap, local row index
  int32_t* colpiv;  // nbox * rcap, sorted point id
};

// ------------------------------------------------------------------ L2P
// One CTA per box: D = K(R, C) (r x r), A = D^T factorised with partial
// pivoting; each thread solves A x = (K(row_i, C))^T for one row i of L2P.
constexpr int L2P_T = 128;

struct L2pArgs {
  int nbox;
  const double2* pts;
  const int32_t* node_off;
  const int32_t* node_ids;
  const int32_t* rank;
  const int32_t* rowpiv;
  const int32_t* colpiv;
  int rcap;
  KernelParams kp;
  const int32_t* skel_off;
  const int64_t* l2p_off;
  int32_t* skel_ids;
  int32_t* cpiv_ids;
  double2* skel_xy;
  double* l2p;
  int xs;            // rows of L2P solved at once (one per thread)
  int rmax;          // largest rank of the level
  double* gscratch;  // gridDim.x * rmax^2 when the factor lives in global memory
  double* gx;        // gridDim.x * rmax * xs solve columns, with the factor in global memory
};

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
  int cluster = 0;          // CTAs per box (power of two <= 16); 0: the planner's choice
  int ctas_per_sm = 0;      // 1 (full shared-memory budget) or 2 (half); 0: the planner's choice
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
  double scratch_s = 0;         // wall clock of the working-memory reservation
  size_t scratch_bytes = 0;     // working memory the level's ACA needs
};

// Working memory of the ACA and L2P kernels, kept across the levels of one
// assemble: spill slots and pivots, and the L2P's global factor slots.
struct AcaScratch {
  DevScratch work, factors;
};

// Runs the ACA and L2P kernels for one level; outputs are allocated in
// `arena`, the kernels' working memory carved from `scratch`.  Synchronises `s`.
void aca_level(const AcaLevelIn& in, AcaLevelOut& out, DevArena& arena, AcaScratch& scratch, cudaStream_t s,
               int64_t* launches);

}  // namespace afmm
