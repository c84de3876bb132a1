// A set of independent assembled problems applied together: every stage of
// the FP64 matvec runs as one fused launch over all problems, and the whole
// sequence is captured once in a CUDA graph.
#pragma once
#include <vector>

#include "fmm.cuh"

namespace afmm {

// Device tables of the set (pointers to device memory), passed by value.
struct SetDev {
  int nprob = 0;
  const LevelView* lv = nullptr;    // nprob x kMaxLevels, level j of problem p at p*kMaxLevels + j
  const NearView* nv = nullptr;     // nprob
  const KernelParams* kp = nullptr; // nprob
  const int2* p2p = nullptr;        // nprob: near-field launch shape (NT, G)
  const int64_t* const* perm = nullptr;  // nprob: sorted -> original index
  double* const* qs = nullptr;      // nprob: sorted charges
  double* const* ys = nullptr;      // nprob: sorted potentials
  const int64_t* off = nullptr;     // nprob + 1: problem p's points at [off[p], off[p+1]) of the set vectors
};

// Work items of one fused launch: segment s covers items [first[s], first[s+1])
// of problem prob[s] at level level[s].
struct SetSegs {
  const int64_t* first = nullptr;  // n + 1
  const int32_t* prob = nullptr;
  const int32_t* level = nullptr;
  int n = 0;
  long total = 0;
};

// Segment of flat item g: the largest s with first[s] <= g.
__device__ __forceinline__ int seg_of(const SetSegs& sg, long g) {
  int lo = 0, hi = sg.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sg.first[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Host description of one problem of the set.
struct SetProblem {
  const MatvecPlan* plan;
  P2pShape shape;
};

// A persistent sweep (every level of every problem in one launch): items are
// tiles of kSweepTile rows of one depth's flat row space (segs[depth]), listed
// in dependency order; CTAs take them in list order from a ticket counter.
constexpr int kSweepTile = 128;
struct SweepPlan {
  const SetSegs* segs = nullptr;    // per depth (device array)
  const int32_t* item_depth = nullptr;
  const int64_t* item_row0 = nullptr;
  int nitems = 0;
  int grid = 0;                     // resident CTAs launched
  int margin = 0;                   // added to every awaited row count (0; > 0 only to test the time limit)
};

// Counters of the persistent sweeps, zeroed at the start of every replay.
struct SweepSync {
  int* ticket = nullptr;  // [2]: up-sweep, down-sweep
  int* done_up = nullptr; // nprob x kMaxLevels: M2M rows published per (problem, level)
  int* done_dn = nullptr; // nprob x kMaxLevels: L2L node rows published per (problem, level)
  int* err = nullptr;     // [1]: a wait gave up (AFMM_TIMEOUT)
  size_t bytes = 0;       // size of the block starting at ticket
};

struct SetPlan {
  SetDev dev;
  SweepPlan up, down;
  SweepSync sync;
  int* h_err = nullptr;     // pinned copy of sync.err, written at the end of every replay
  int kernel_id = 0;
  long total_points = 0;
  int p2p_threads = 0;
  size_t p2p_smem = 0;
  SetSegs gather, m2l, p2p;
  std::vector<SetSegs> m2m;  // by depth below each problem's leaf level
  std::vector<SetSegs> l2l;  // by level 2, 3, ...
  double* q = nullptr;       // set input (original order, problems concatenated)
  double* y = nullptr;       // set output
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches_per_matvec = 0;
  // events recorded inside the graph between stages (per-stage device time)
  std::vector<std::pair<std::string, cudaEvent_t>> marks;
};

// Per-stage milliseconds of the last replay, accumulated by stage name.
void set_stage_times(const SetPlan& sp, std::vector<std::pair<std::string, double>>& out);

// Builds the device tables (allocated from `arena`) and the graph on stream s.
void set_build(SetPlan& sp, const std::vector<SetProblem>& probs, DevArena& arena, cudaStream_t s);
// One FP64 matvec of every problem: sp.q -> sp.y (graph replay on s).  After
// the stream completes, *sp.h_err is nonzero if a sweep's bounded wait gave up.
void set_matvec(SetPlan& sp, cudaStream_t s);
// Re-records the graph after a change of the sweeps' parameters.
void set_recapture(SetPlan& sp, cudaStream_t s);
void set_release(SetPlan& sp);

}  // namespace afmm
