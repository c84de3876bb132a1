// Many independent problems in fused launches (one launch per stage across
// all problems, each sweep over the levels one persistent launch, captured in
// one CUDA graph).  Each output row is computed by
// the same device functions as the single-problem FP64 path (fmm.cuh), so
// every problem's result is bit-identical to its own FP64 matvec.
#include <algorithm>

#include "kernel_table.cuh"
#include "set.cuh"

namespace afmm {

namespace {

// qs_p[i] = q[off[p] + perm_p[i]]  (src/AFMM2D.cpp:49-51 per problem)
__global__ void k_set_gather(SetDev d, SetSegs sg, const double* __restrict__ q) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  const int p = sg.prob[s];
  const long i = g - sg.first[s];
  d.qs[p][i] = q[d.off[p] + d.perm[p][i]];
}

// y[off[p] + perm_p[i]] = ys_p[i]  (src/AFMM2D.cpp:61-63 per problem)
__global__ void k_set_scatter(SetDev d, SetSegs sg, double* __restrict__ y) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  const int p = sg.prob[s];
  const long i = g - sg.first[s];
  y[d.off[p] + d.perm[p][i]] = d.ys[p][i];
}

// ------------------------------------------------ persistent sweeps
// The M2M of every level of every problem runs in one launch (the up-sweep),
// and so does the L2L (the down-sweep).  Items are tiles of kSweepTile rows
// of one depth, listed in dependency order (M2M: each problem's leaf level
// first; L2L: level 2 first); a CTA takes the next item from a ticket counter,
// waits until every row that the item reads has been published (per problem
// and level counters), computes its rows with the FP64 path's row arithmetic
// (same bits) and publishes them.  An item only waits for items earlier in
// the list, which CTAs already running hold, so the sweep cannot deadlock;
// each wait is still bounded in time, and a wait that gives up sets
// sync.err, makes every other wait give up and ends the launch early.

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s of device time per wait

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One thread waits until *c >= need; false if it gave up (time limit, or
// another wait gave up first).
__device__ bool wait_published(const int* c, long need, int* err) {
  if (ld_acquire(c) >= need) return true;
  const unsigned long long t0 = global_ns();
  for (int it = 0; it < (1 << 26); ++it) {
    __nanosleep(128);
    if (ld_acquire(c) >= need) return true;
    if (*(volatile int*)err) return false;
    if (global_ns() - t0 > kWaitNs) break;
  }
  atomicExch(err, 1);
  return false;
}

// The next item of a sweep for the calling CTA (all threads), or -1.
__device__ __forceinline__ int next_item(int* ticket, int nitems, int* s_item) {
  __syncthreads();  // every thread has read the previous item
  if (threadIdx.x == 0) *s_item = atomicAdd(ticket, 1);
  __syncthreads();
  const int it = *s_item;
  return it < nitems ? it : -1;
}

// Publishes the tile [r0, r1) of depth table sg: rows per (problem, level).
__device__ __forceinline__ void publish_rows(const SetSegs& sg, long r0, long r1, int s0, int s1, int* done) {
  __threadfence();
  __syncthreads();
  for (int s = s0 + (int)threadIdx.x; s <= s1; s += blockDim.x) {
    const long a = max(r0, sg.first[s]), b = min(r1, sg.first[s + 1]);
    __threadfence();
    atomicAdd(done + (long)sg.prob[s] * kMaxLevels + sg.level[s], (int)(b - a));
  }
}

// Streams into L2 the interpolation blocks that the item's rows [r0, r1)
// read -- the row-major copy for the M2M (skeleton rows), the column-major
// L2P for the L2L (node rows): one contiguous region per problem and level
// the item touches (a box's block follows its predecessor's).  Warp 0, before
// the item waits for its inputs, so the fetch overlaps the wait.  Used by the
// down-sweep (0.85 -> 0.67 ms on 256 problems of 2K-64K points); the
// up-sweep's row-major reads are already contiguous per warp and measured
// slower with it (0.41 -> 0.48 ms).
__device__ __forceinline__ void prefetch_item_l2p(const SetDev& d, const SetSegs& sg, long r0, long r1, int s0,
                                                  int s1, bool up, int lane) {
  for (int s = s0; s <= s1; ++s) {
    const LevelView& v = d.lv[(long)sg.prob[s] * kMaxLevels + sg.level[s]];
    const long a = max(r0, sg.first[s]) - sg.first[s], e = min(r1, sg.first[s + 1]) - sg.first[s];
    const int32_t* box = up ? v.skel_box : v.node_box;
    const double* P = up ? v.l2p_rm : v.l2p;
    prefetch_l2_region(P + v.l2p_off[box[a]], P + v.l2p_off[box[e - 1] + 1], lane);
  }
}

// Up-sweep: M2M of every problem from its leaf level up to level 2 (skeleton
// rows).  A non-leaf level reads the outgoing charges of the level below.
__global__ void __launch_bounds__(kSweepTile) k_set_up(SetDev d, SweepPlan sw, SweepSync sy) {
  __shared__ int s_item, s_ok;
  for (int it; (it = next_item(sy.ticket, sw.nitems, &s_item)) >= 0;) {
    const SetSegs sg = sw.segs[sw.item_depth[it]];
    const long r0 = sw.item_row0[it], r1 = min(r0 + (long)kSweepTile, sg.total);
    const int s0 = seg_of(sg, r0), s1 = seg_of(sg, r1 - 1);
    if (threadIdx.x == 0) s_ok = 1;
    __syncthreads();
    for (int s = s0 + (int)threadIdx.x; s <= s1; s += blockDim.x) {
      const long pl = (long)sg.prob[s] * kMaxLevels + sg.level[s];
      if (d.lv[pl].leaf_start == nullptr &&
          !wait_published(sy.done_up + pl + 1, d.lv[pl + 1].nrows + sw.margin, sy.err))
        s_ok = 0;
    }
    __threadfence();
    __syncthreads();
    if (!s_ok) return;  // the same in every thread of the CTA
    const long g = r0 + threadIdx.x;
    if (g < r1) {
      const int s = seg_of(sg, g);
      const int p = sg.prob[s], j = sg.level[s];
      const LevelView& v = d.lv[(long)p * kMaxLevels + j];
      const bool leaf = v.leaf_start != nullptr;
      const double* src = leaf ? d.qs[p] : d.lv[(long)p * kMaxLevels + j + 1].qhat;
      m2m_row<true>(v, src, leaf ? 1 : 0, g - sg.first[s]);
    }
    publish_rows(sg, r0, r1, s0, s1, sy.done_up);
  }
}

// M2L of every level of every problem (skeleton rows).
__global__ void k_set_m2l(SetDev d, SetSegs sg) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  m2l_row(d.lv[(long)sg.prob[s] * kMaxLevels + sg.level[s]], g - sg.first[s]);
}

// Down-sweep: L2L of every problem from level 2 down to its leaf level (node
// rows).  Level j > 2 reads incoming potentials that the L2L of level j - 1
// adds into.
__global__ void __launch_bounds__(kSweepTile) k_set_down(SetDev d, SweepPlan sw, SweepSync sy) {
  __shared__ int s_item, s_ok;
  for (int it; (it = next_item(sy.ticket + 1, sw.nitems, &s_item)) >= 0;) {
    const SetSegs sg = sw.segs[sw.item_depth[it]];
    const long r0 = sw.item_row0[it], r1 = min(r0 + (long)kSweepTile, sg.total);
    const int s0 = seg_of(sg, r0), s1 = seg_of(sg, r1 - 1);
    if (threadIdx.x == 0) s_ok = 1;
    if (threadIdx.x < 32) prefetch_item_l2p(d, sg, r0, r1, s0, s1, false, threadIdx.x);
    __syncthreads();
    for (int s = s0 + (int)threadIdx.x; s <= s1; s += blockDim.x) {
      const long pl = (long)sg.prob[s] * kMaxLevels + sg.level[s];
      if (sg.level[s] > 2 && !wait_published(sy.done_dn + pl - 1, d.lv[pl - 1].nnodes + sw.margin, sy.err))
        s_ok = 0;
    }
    __threadfence();
    __syncthreads();
    if (!s_ok) return;  // the same in every thread of the CTA
    const long g = r0 + threadIdx.x;
    if (g < r1) {
      const int s = seg_of(sg, g);
      const int p = sg.prob[s], j = sg.level[s];
      const LevelView& v = d.lv[(long)p * kMaxLevels + j];
      const bool leaf = v.leaf_start != nullptr;
      double* child = leaf ? nullptr : d.lv[(long)p * kMaxLevels + j + 1].yhat;
      l2l_row<true>(v, child, d.ys[p], leaf ? 1 : 0, g - sg.first[s]);
    }
    publish_rows(sg, r0, r1, s0, s1, sy.done_dn);
  }
}

struct SegBuilder {
  std::vector<int64_t> first{0};
  std::vector<int32_t> prob, level;
  void add(int p, int j, long count) {
    if (count <= 0) return;
    prob.push_back(p);
    level.push_back(j);
    first.push_back(first.back() + count);
  }
  SetSegs upload(DevArena& arena, cudaStream_t s) const {
    SetSegs sg;
    sg.n = (int)prob.size();
    sg.total = first.back();
    int64_t* f = arena.alloc<int64_t>(first.size());
    int32_t* pr = arena.alloc<int32_t>(std::max<size_t>(prob.size(), 1));
    int32_t* lv = arena.alloc<int32_t>(std::max<size_t>(level.size(), 1));
    AFMM_CUDA(cudaMemcpyAsync(f, first.data(), sizeof(int64_t) * first.size(), cudaMemcpyHostToDevice, s));
    if (!prob.empty()) {
      AFMM_CUDA(cudaMemcpyAsync(pr, prob.data(), sizeof(int32_t) * prob.size(), cudaMemcpyHostToDevice, s));
      AFMM_CUDA(cudaMemcpyAsync(lv, level.data(), sizeof(int32_t) * level.size(), cudaMemcpyHostToDevice, s));
    }
    AFMM_CUDA(cudaStreamSynchronize(s));
    sg.first = f;
    sg.prob = pr;
    sg.level = lv;
    return sg;
  }
};

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

template <class T>
T* upload(const std::vector<T>& h, DevArena& arena, cudaStream_t s) {
  T* d = arena.alloc<T>(std::max<size_t>(h.size(), 1));
  if (!h.empty()) AFMM_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
  return d;
}

void record(SetPlan& sp, cudaStream_t s) {
  int n = 0, m = 0;
  auto mark = [&](const char* name) {
    if ((size_t)m == sp.marks.size()) {
      cudaEvent_t e;
      AFMM_CUDA(cudaEventCreate(&e));
      sp.marks.push_back({name, e});
    }
    // an external record becomes an event-record node of the graph
    AFMM_CUDA(cudaEventRecordWithFlags(sp.marks[m].second, s, cudaEventRecordExternal));
    ++m;
  };
  // the sweeps' tickets and counters start at zero in every replay
  AFMM_CUDA(cudaMemsetAsync(sp.sync.ticket, 0, sp.sync.bytes, s));
  mark("gather");
  k_set_gather<<<nb(sp.gather.total, 256), 256, 0, s>>>(sp.dev, sp.gather, sp.q);
  AFMM_LAUNCH_CHECK();
  ++n;
  mark("m2m");
  if (sp.up.nitems > 0) {
    k_set_up<<<sp.up.grid, kSweepTile, 0, s>>>(sp.dev, sp.up, sp.sync);
    AFMM_LAUNCH_CHECK();
    ++n;
  }
  mark("m2l");
  if (sp.m2l.total > 0) {
    k_set_m2l<<<nb(sp.m2l.total, 128), 128, 0, s>>>(sp.dev, sp.m2l);
    AFMM_LAUNCH_CHECK();
    ++n;
  }
  mark("l2l");
  if (sp.down.nitems > 0) {
    k_set_down<<<sp.down.grid, kSweepTile, 0, s>>>(sp.dev, sp.down, sp.sync);
    AFMM_LAUNCH_CHECK();
    ++n;
  }
  mark("p2p");
  kernel_table(sp.kernel_id).set_p2p_run(sp, s);
  ++n;
  mark("scatter");
  k_set_scatter<<<nb(sp.gather.total, 256), 256, 0, s>>>(sp.dev, sp.gather, sp.y);
  AFMM_LAUNCH_CHECK();
  ++n;
  mark("end");
  AFMM_CUDA(cudaMemcpyAsync(sp.h_err, sp.sync.err, sizeof(int), cudaMemcpyDeviceToHost, s));
  sp.launches_per_matvec = n;
}

}  // namespace

void set_build(SetPlan& sp, const std::vector<SetProblem>& probs, DevArena& arena, cudaStream_t s) {
  const int np = (int)probs.size();
  std::vector<LevelView> lv((size_t)np * kMaxLevels);
  std::vector<NearView> nv(np);
  std::vector<KernelParams> kp(np);
  std::vector<int2> shape(np);
  std::vector<const int64_t*> perm(np);
  std::vector<double*> qs(np), ys(np);
  std::vector<int64_t> off(np + 1, 0);
  SegBuilder g, m2l, p2p;
  int maxL = 0;
  sp.p2p_threads = 0;
  sp.p2p_smem = 0;
  for (int p = 0; p < np; ++p) {
    const MatvecPlan& mp = *probs[p].plan;
    for (int j = 0; j <= mp.L; ++j) lv[(size_t)p * kMaxLevels + j] = mp.lv[j];
    nv[p] = mp.near;
    kp[p] = mp.kp;
    shape[p] = make_int2(probs[p].shape.nt, probs[p].shape.g);
    perm[p] = mp.perm;
    qs[p] = mp.qs;
    ys[p] = mp.ys;
    off[p + 1] = off[p] + mp.N;
    g.add(p, 0, mp.N);
    for (int j = 2; j <= mp.L; ++j) m2l.add(p, j, mp.lv[j].nrows);
    p2p.add(p, mp.L, mp.near.nleaf);
    maxL = std::max(maxL, mp.L);
    sp.p2p_threads = std::max(sp.p2p_threads, probs[p].shape.threads);
    sp.p2p_smem = std::max(sp.p2p_smem, (size_t)9 * mp.near.nmax * (sizeof(double2) + sizeof(double)) +
                                            sizeof(double) * probs[p].shape.threads);
  }
  // M2M by depth below the leaf level; L2L by level from the top; each
  // sweep's items are the depth tables' row tiles in that order
  sp.m2m.clear();
  sp.l2l.clear();
  std::vector<int32_t> up_d, dn_d;
  std::vector<int64_t> up_r, dn_r;
  auto tiles = [](long total, int depth, std::vector<int32_t>& dd, std::vector<int64_t>& rr) {
    for (long r = 0; r < total; r += kSweepTile) {
      dd.push_back(depth);
      rr.push_back(r);
    }
  };
  for (int depth = 0; depth + 2 <= maxL; ++depth) {
    SegBuilder b;
    for (int p = 0; p < np; ++p) {
      const MatvecPlan& mp = *probs[p].plan;
      const int j = mp.L - depth;
      if (j >= 2) b.add(p, j, mp.lv[j].nrows);
    }
    if (b.first.back() > 0) {
      tiles(b.first.back(), (int)sp.m2m.size(), up_d, up_r);
      sp.m2m.push_back(b.upload(arena, s));
    }
  }
  for (int j = 2; j <= maxL; ++j) {
    SegBuilder b;
    for (int p = 0; p < np; ++p) {
      const MatvecPlan& mp = *probs[p].plan;
      if (j <= mp.L) b.add(p, j, mp.lv[j].nnodes);
    }
    if (b.first.back() > 0) {
      tiles(b.first.back(), (int)sp.l2l.size(), dn_d, dn_r);
      sp.l2l.push_back(b.upload(arena, s));
    }
  }
  int nsm = 0, dev = 0, per_sm_up = 0, per_sm_dn = 0;
  AFMM_CUDA(cudaGetDevice(&dev));
  AFMM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  AFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_up, k_set_up, kSweepTile, 0));
  AFMM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_dn, k_set_down, kSweepTile, 0));
  sp.up.segs = upload(sp.m2m, arena, s);
  sp.up.item_depth = upload(up_d, arena, s);
  sp.up.item_row0 = upload(up_r, arena, s);
  sp.up.nitems = (int)up_d.size();
  sp.up.grid = (int)std::min<long>(sp.up.nitems, (long)std::max(per_sm_up, 1) * nsm);
  sp.down.segs = upload(sp.l2l, arena, s);
  sp.down.item_depth = upload(dn_d, arena, s);
  sp.down.item_row0 = upload(dn_r, arena, s);
  sp.down.nitems = (int)dn_d.size();
  sp.down.grid = (int)std::min<long>(sp.down.nitems, (long)std::max(per_sm_dn, 1) * nsm);
  const size_t ncnt = (size_t)np * kMaxLevels;
  sp.sync.bytes = sizeof(int) * (3 + 2 * ncnt);
  sp.sync.ticket = arena.alloc<int>(3 + 2 * ncnt);
  sp.sync.err = sp.sync.ticket + 2;
  sp.sync.done_up = sp.sync.ticket + 3;
  sp.sync.done_dn = sp.sync.done_up + ncnt;
  if (!sp.h_err) {
    AFMM_CUDA(cudaHostAlloc((void**)&sp.h_err, sizeof(int), cudaHostAllocDefault));
    *sp.h_err = 0;
  }
  sp.gather = g.upload(arena, s);
  sp.m2l = m2l.upload(arena, s);
  sp.p2p = p2p.upload(arena, s);
  sp.dev.nprob = np;
  sp.dev.lv = upload(lv, arena, s);
  sp.dev.nv = upload(nv, arena, s);
  sp.dev.kp = upload(kp, arena, s);
  sp.dev.p2p = upload(shape, arena, s);
  sp.dev.perm = upload(perm, arena, s);
  sp.dev.qs = upload(qs, arena, s);
  sp.dev.ys = upload(ys, arena, s);
  sp.dev.off = upload(off, arena, s);
  sp.total_points = off[np];
  sp.q = arena.alloc<double>(off[np]);
  sp.y = arena.alloc<double>(off[np]);
  AFMM_CUDA(cudaStreamSynchronize(s));
  // kernel attributes are set before capture; then the graph is recorded once
  kernel_table(sp.kernel_id).set_p2p_prepare(sp.p2p_smem);
  set_recapture(sp, s);
}

void set_recapture(SetPlan& sp, cudaStream_t s) {
  if (sp.exec) AFMM_CUDA(cudaGraphExecDestroy(sp.exec));
  if (sp.graph) AFMM_CUDA(cudaGraphDestroy(sp.graph));
  sp.exec = nullptr;
  sp.graph = nullptr;
  AFMM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    record(sp, s);
  } catch (...) {
    cudaGraph_t tmp = nullptr;
    cudaStreamEndCapture(s, &tmp);
    if (tmp) cudaGraphDestroy(tmp);
    cudaGetLastError();
    throw;
  }
  AFMM_CUDA(cudaStreamEndCapture(s, &sp.graph));
  AFMM_CUDA(cudaGraphInstantiate(&sp.exec, sp.graph, 0));
}

void set_matvec(SetPlan& sp, cudaStream_t s) { AFMM_CUDA(cudaGraphLaunch(sp.exec, s)); }

void set_stage_times(const SetPlan& sp, std::vector<std::pair<std::string, double>>& out) {
  out.clear();
  for (size_t i = 0; i + 1 < sp.marks.size(); ++i) {
    float ms = 0;
    AFMM_CUDA(cudaEventElapsedTime(&ms, sp.marks[i].second, sp.marks[i + 1].second));
    out.push_back({sp.marks[i].first, ms});
  }
}

void set_release(SetPlan& sp) {
  if (sp.h_err) cudaFreeHost(sp.h_err);
  sp.h_err = nullptr;
  if (sp.exec) cudaGraphExecDestroy(sp.exec);
  if (sp.graph) cudaGraphDestroy(sp.graph);
  for (auto& m : sp.marks) cudaEventDestroy(m.second);
  sp.marks.clear();
  sp.exec = nullptr;
  sp.graph = nullptr;
}

}  // namespace afmm
