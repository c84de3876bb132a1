// Tree views handed to the sweep kernels (see fmm.cu, mixed.cu).
#pragma once
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "afmm_internal.cuh"

namespace afmm {

constexpr int kMaxLevels = 16;
// CTA shape of the per-box sweep kernels.
constexpr int SW_T = 256;
constexpr int SW_WARPS = SW_T / 32;
// threads for a per-box kernel whose work runs over up to n rows
inline int sweep_threads(int n) { return n <= 64 ? 64 : (n <= 128 ? 128 : 256); }

// Allows `bytes` of dynamic shared memory for kernel `fn` (needed above 48 KB).
template <class F>
inline void allow_smem(F* fn, size_t bytes) {
  if (bytes > 48 * 1024) {
    if (bytes > 227 * 1024) throw Error{AFMM_BAD_ARG, "per-box rank too large for the sweep kernels"};
    AFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  }
}

// Device pointers of one level, passed by value to kernels.
struct LevelView {
  long nbox = 0;
  const int32_t* il = nullptr;
  const int32_t* rank = nullptr;
  const int32_t* skel_off = nullptr;
  const int32_t* node_off = nullptr;
  const int32_t* leaf_start = nullptr;  // leaf level only (quadtree order)
  const int64_t* l2p_off = nullptr;
  const double* l2p = nullptr;     // column-major (row index fastest)
  const double* l2p_rm = nullptr;  // row-major copy (rank index fastest)
  const int64_t* m2l_off = nullptr;
  double* m2l = nullptr;
  const double2* skel_xy = nullptr;
  double* qhat = nullptr;
  double* yhat = nullptr;
  const int32_t* skel_box = nullptr;  // skeleton row -> box
  const int32_t* node_box = nullptr;  // node row -> box
  const int32_t* grp_box = nullptr;   // row group (<= 8 rows of one box) -> box
  const int32_t* grp_row = nullptr;   // row group -> first skeleton row
  long ngroups = 0;
  const int32_t* cgrp_box = nullptr;  // row chunk (<= kChunkRows rows of one box) -> box
  const int32_t* cgrp_row = nullptr;  // row chunk -> first skeleton row
  long ncgroups = 0;
  const int32_t* ncgrp_box = nullptr;  // node-row chunk (<= kChunkRows node rows of one box) -> box
  const int32_t* ncgrp_row = nullptr;  // node-row chunk -> first node row
  long nncgroups = 0;
  long nrows = 0;                     // skeleton rows (sum of ranks)
  long nnodes = 0;                    // node rows (sum of node counts)
};

// Levels 2..L and the prefix of their skeleton row counts: the M2L kernels
// run one thread per skeleton row over this flat row space.
struct LevelSet {
  int nlev = 0;
  LevelView lv[kMaxLevels];
  long row0[kMaxLevels + 1] = {0};
  long grp0[kMaxLevels + 1] = {0};   // prefix of row-group counts
  long cgrp0[kMaxLevels + 1] = {0};  // prefix of row-chunk counts
};

// Leaf-level data for the near field.
struct NearView {
  long nleaf = 0;
  int nmax = 0;
  const double2* pts = nullptr;        // sorted points
  const int32_t* leaf_start = nullptr; // quadtree order
  const int32_t* leaf_cnt = nullptr;
  const int32_t* nbr = nullptr;        // nleaf * 8
  const double2* anchor = nullptr;     // leaf anchors (FP64)
  const float2* rel = nullptr;         // point minus its leaf anchor (FP32), sorted order
  const float* span = nullptr;         // per leaf max |rel| component
};

// CUDA-event marks for per-stage device timing.
struct StageTimer {
  std::vector<std::pair<std::string, cudaEvent_t>> marks;
  size_t used = 0;
  void reset() { used = 0; }
  void mark(cudaStream_t s, const char* name) {
    if (used == marks.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      marks.push_back({name, e});
    }
    marks[used].first = name;
    cudaEventRecord(marks[used].second, s);
    ++used;
  }
  // durations between consecutive marks, accumulated by name
  void collect(std::vector<std::pair<std::string, double>>& out) {
    out.clear();
    for (size_t i = 0; i + 1 < used; ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, marks[i].second, marks[i + 1].second);
      bool found = false;
      for (auto& o : out)
        if (o.first == marks[i].first) {
          o.second += ms;
          found = true;
        }
      if (!found) out.push_back({marks[i].first, ms});
    }
  }
  ~StageTimer() {
    for (auto& m : marks) cudaEventDestroy(m.second);
  }
};

struct MatvecPlan {
  int N = 0, L = 0;
  KernelParams kp;
  const int64_t* perm = nullptr;
  const int32_t* iperm = nullptr;  // original index -> sorted position
  double* qs = nullptr;  // sorted charges
  double* ys = nullptr;  // sorted potentials
  LevelView lv[kMaxLevels];
  int rmax[kMaxLevels] = {0};   // largest rank per level
  int n1max[kMaxLevels] = {0};  // largest node count per level
  LevelSet levels;       // levels 2..L for the M2L launch
  NearView near;
};

// M2L kernels work on (slot, row) items; rows are processed in chunks of at
// most M2L_RCH so that the per-slot partial sums (40 x M2L_RCH doubles) fit
// in shared memory.
constexpr int M2L_RCH = 256;

// Valid interaction-list slots of a box, staged by one thread.
struct SlotTable {
  int n;
  int box[40];
  int rank[40];
  int skel[40];
  long off[40];  // block offset within the box's M2L data (stored form)
};

// Near-field launch shape: NT threads per target group (targets rounded up to
// a warp multiple), G groups splitting the (up to 9) source leaves.
struct P2pShape {
  int nt, g, threads;
};
inline P2pShape p2p_shape(int nmax) {
  P2pShape p;
  p.nt = (nmax + 31) / 32 * 32;
  p.g = std::max(1, std::min(9, 256 / p.nt));
  p.threads = p.nt * p.g;
  return p;
}

void build_lists(int j, long nbox, int32_t* nbr, int32_t* il, cudaStream_t s);
// map[off[b] + l] = b for l < off[b+1] - off[b]
void fill_box_map(const int32_t* off, long nbox, int32_t* map, cudaStream_t s);
// iperm[perm[i]] = i
void invert_permutation(const int64_t* perm, int n, int32_t* iperm, cudaStream_t s);
void m2l_assemble(const LevelView& v, const KernelParams& kp, cudaStream_t s);
void l2p_transpose(const LevelView& v, const double* cm, double* rm, cudaStream_t s);
void matvec_fp64(const MatvecPlan& p, const double* q, double* y, cudaStream_t s, StageTimer* tm, int64_t* launches);
// The FP64 sweeps shared by both precisions (leaf charges qs in FP64).
void sweep_m2m(const MatvecPlan& p, const double* qs, cudaStream_t s, int64_t* launches);
void sweep_l2l(const MatvecPlan& p, double* ys, cudaStream_t s, int64_t* launches);

}  // namespace afmm
