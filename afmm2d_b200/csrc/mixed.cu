// Mixed-precision matvec: FP32 where the work is and the error is small, FP64
// where cancellation would amplify rounding.
//
// Same sweeps as the FP64 path (src/AFMM2DTree.cpp:1129-1213), changed in two
// places:
//  * M2L reads the 32-bit fixed-point copy of the blocks (half the bytes of
//    FP64; entries within 2^-31 of their block's largest) or evaluates the
//    entries on the fly from the skeleton coordinates (the blocks are plain
//    kernel entries between skeleton points, src/AFMM2DTree.cpp:1080); the
//    fixed-point copy when kept, otherwise whichever of the FP64 blocks and
//    the on-the-fly form the first matvec measures faster.  The arithmetic stays FP64
//    because the outgoing charges are combinations with large, mixed-sign
//    weights (ACA interpolation matrices) and FP32 entries lose ~10x to
//    cancellation.
//  * The near field is evaluated in FP32 from coordinates relative to a
//    per-leaf anchor point (anchor differences formed in FP64 before
//    rounding, so dx keeps ~2^-24 relative precision however clustered the
//    points are); pairs closer than 2^-7 of the two leaves' extents, and for
//    the log kernel every pair with R2 near its 1e-10 diagonal convention,
//    are re-evaluated in FP64 from the exact coordinates.  FP32 partial sums
//    cover one source leaf and are accumulated in FP64.
// M2M / L2L keep FP64 operators (they move ~2 GB at N = 4M and carry the same
// cancellation); inputs and outputs are FP64.
#include <algorithm>

#include "kernel_table.cuh"
#include "mixed.cuh"

namespace afmm {

namespace {

// Leaves: anchor = first point of the leaf; rel for every sorted point;
// span = max |rel| component.
__global__ void k_anchor_leaf(long nleaf, const int32_t* __restrict__ start, const int32_t* __restrict__ cnt,
                              const double2* __restrict__ pts, double2* anchor, float2* rel, float* span) {
  const long b = blockIdx.x;
  const int s0 = start[b], n = cnt[b];
  const double2 a = pts[s0];
  float sp = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 p = pts[s0 + i];
    float2 d = make_float2((float)(p.x - a.x), (float)(p.y - a.y));
    rel[s0 + i] = d;
    sp = fmaxf(sp, fmaxf(fabsf(d.x), fabsf(d.y)));
  }
  for (int o = 16; o > 0; o >>= 1) sp = fmaxf(sp, __shfl_down_sync(0xffffffffu, sp, o));
  __shared__ float ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = sp;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.0f;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmaxf(m, ws[w]);
    anchor[b] = a;
    span[b] = m;
  }
}

// qs[i] = q[perm[i]] in FP64 and FP32
__global__ void k_gather_mixed(const double* __restrict__ q, const int64_t* __restrict__ perm, int N, double* qs,
                               float* qs32) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double v = q[perm[i]];
  qs[i] = v;
  qs32[i] = (float)v;
}

__global__ void k_scatter64(const double* __restrict__ ys, const int64_t* __restrict__ perm, int N, double* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) y[perm[i]] = ys[i];
}

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void m2l_apply_otf(const MatvecPlan& p, const LevelSet& levels, cudaStream_t s) {
  if (levels.row0[levels.nlev] == 0) return;
  kernel_table(p.kp.id).m2l_otf(levels, p.kp, s);
}


void mixed_setup(MatvecPlan& p, std::vector<LevelDev>&, MixedState& ms, DevArena& arena, cudaStream_t s,
                 int64_t* launches) {
  NearView& nv = p.near;
  ms.leaf_anchor = arena.alloc<double2>(nv.nleaf);
  ms.leaf_span = arena.alloc<float>(nv.nleaf);
  ms.rel = arena.alloc<float2>(p.N);
  k_anchor_leaf<<<(int)nv.nleaf, 64, 0, s>>>(nv.nleaf, nv.leaf_start, nv.leaf_cnt, nv.pts, ms.leaf_anchor, ms.rel,
                                              ms.leaf_span);
  AFMM_LAUNCH_CHECK();
  *launches += 1;
  ms.ready = true;
}

void mixed_reserve(MixedState& ms, int N, int nrhs, DevArena& arena) {
  if (ms.rhs_cap >= nrhs) return;
  ms.qs32 = arena.alloc<float>((size_t)N * nrhs);
  ms.qs = arena.alloc<double>((size_t)N * nrhs + 2);  // + 16 B: whole-piece L2 prefetches
  ms.ys = arena.alloc<double>((size_t)N * nrhs);
  ms.rhs_cap = nrhs;
}

void mixed_reserve_io(MixedState& ms, int N, int nrhs, DevArena& arena) {
  ms.d_qin = arena.alloc<double>((size_t)N * nrhs);
  ms.d_yout = arena.alloc<double>((size_t)N * nrhs);
  ms.host_cap = nrhs;
}

void matvec_mixed(const MatvecPlan& p, MixedState& ms, const double* q, int64_t ldq, double* y, int64_t ldy, int nrhs,
                  cudaStream_t s, StageTimer* tm, int64_t* launches) {
  if (!ms.ready) throw Error{AFMM_BAD_ARG, "mixed precision operators are not set up"};
  const int N = p.N;
  NearView nv = p.near_own;
  nv.anchor = ms.leaf_anchor;
  nv.rel = ms.rel;
  nv.span = ms.leaf_span;
  for (int c = 0; c < nrhs; ++c) {
    if (tm) tm->mark(s, "gather");
    if (p.shard_count > 1) AFMM_CUDA(cudaMemsetAsync(ms.ys, 0, sizeof(double) * (size_t)N, s));
    k_gather_mixed<<<nb(N, 256), 256, 0, s>>>(q + (long)c * ldq, p.perm, N, ms.qs, ms.qs32);
    AFMM_LAUNCH_CHECK();
    ++*launches;
    if (tm) tm->mark(s, "m2m");
    sweep_m2m(p, ms.qs, s, launches);
    if (tm) tm->mark(s, "m2l");
    // stored form: the 32-bit fixed-point blocks when kept, else the FP64
    // ones; the levels of the tuning mask (or all, without stored blocks)
    // evaluate the entries on the fly
    const bool q32 = p.levels.nlev > 0 && p.levels.lv[0].m2l_q != nullptr;
    const bool stored = q32 || (p.levels.nlev > 0 && p.levels.lv[0].m2l != nullptr);
    const uint32_t otf = stored ? p.tune.otf_mixed : 0xffffffffu;
    // a shard's boxes at the sharded levels for the stored form; the on-the-fly levels whole
    const LevelSet st = level_subset(p.levels_m2l, otf, false), fly = level_subset(p.levels, otf, true);
    if (st.nlev > 0) {
      m2l_apply_stored(p, st, q32, s);
      ++*launches;
    }
    if (fly.nlev > 0) {
      m2l_apply_otf(p, fly, s);
      ++*launches;
    }
    if (tm) tm->mark(s, "l2l");
    sweep_l2l(p, ms.ys, s, launches);
    if (tm) tm->mark(s, "p2p");
    kernel_table(p.kp.id).p2p32(nv, p.kp, ms.qs32, ms.ys, s);
    ++*launches;
    if (tm) tm->mark(s, "scatter");
    k_scatter64<<<nb(N, 256), 256, 0, s>>>(ms.ys, p.perm, N, y + (long)c * ldy);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

}  // namespace afmm
