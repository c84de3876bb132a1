// Many independent problems in fused launches (one launch per stage across
// all problems, captured in one CUDA graph).  Each output row is computed by
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

// M2M of one depth: level L_p - depth of every problem (skeleton rows).
__global__ void k_set_m2m(SetDev d, SetSegs sg) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  const int p = sg.prob[s], j = sg.level[s];
  const LevelView& v = d.lv[(long)p * kMaxLevels + j];
  const bool leaf = v.leaf_start != nullptr;
  const double* src = leaf ? d.qs[p] : d.lv[(long)p * kMaxLevels + j + 1].qhat;
  m2m_row(v, src, leaf ? 1 : 0, g - sg.first[s]);
}

// M2L of every level of every problem (skeleton rows).
__global__ void k_set_m2l(SetDev d, SetSegs sg) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  m2l_row(d.lv[(long)sg.prob[s] * kMaxLevels + sg.level[s]], g - sg.first[s]);
}

// L2L of one level of every problem that has it (node rows).
__global__ void k_set_l2l(SetDev d, SetSegs sg) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= sg.total) return;
  const int s = seg_of(sg, g);
  const int p = sg.prob[s], j = sg.level[s];
  const LevelView& v = d.lv[(long)p * kMaxLevels + j];
  const bool leaf = v.leaf_start != nullptr;
  double* child = leaf ? nullptr : d.lv[(long)p * kMaxLevels + j + 1].yhat;
  l2l_row(v, child, d.ys[p], leaf ? 1 : 0, g - sg.first[s]);
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
  mark("gather");
  k_set_gather<<<nb(sp.gather.total, 256), 256, 0, s>>>(sp.dev, sp.gather, sp.q);
  AFMM_LAUNCH_CHECK();
  ++n;
  mark("m2m");
  for (const SetSegs& sg : sp.m2m) {
    k_set_m2m<<<nb(sg.total, 128), 128, 0, s>>>(sp.dev, sg);
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
  for (const SetSegs& sg : sp.l2l) {
    k_set_l2l<<<nb(sg.total, 128), 128, 0, s>>>(sp.dev, sg);
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
  // M2M by depth below the leaf level; L2L by level from the top
  sp.m2m.clear();
  sp.l2l.clear();
  for (int depth = 0; depth + 2 <= maxL; ++depth) {
    SegBuilder b;
    for (int p = 0; p < np; ++p) {
      const MatvecPlan& mp = *probs[p].plan;
      const int j = mp.L - depth;
      if (j >= 2) b.add(p, j, mp.lv[j].nrows);
    }
    if (b.first.back() > 0) sp.m2m.push_back(b.upload(arena, s));
  }
  for (int j = 2; j <= maxL; ++j) {
    SegBuilder b;
    for (int p = 0; p < np; ++p) {
      const MatvecPlan& mp = *probs[p].plan;
      if (j <= mp.L) b.add(p, j, mp.lv[j].nnodes);
    }
    if (b.first.back() > 0) sp.l2l.push_back(b.upload(arena, s));
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
  if (sp.exec) cudaGraphExecDestroy(sp.exec);
  if (sp.graph) cudaGraphDestroy(sp.graph);
  for (auto& m : sp.marks) cudaEventDestroy(m.second);
  sp.marks.clear();
  sp.exec = nullptr;
  sp.graph = nullptr;
}

}  // namespace afmm
