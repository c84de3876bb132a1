// C ABI of the AFMM2D B200 engine (include/afmm2d.h): handle, setup
// orchestration and matvec dispatch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "aca.cuh"
#include "afmm_internal.cuh"
#include "fmm.cuh"
#include "kd_sort.cuh"
#include "kernel_table.cuh"
#include "mixed.cuh"
#include "set.cuh"

using namespace afmm;

// ------------------------------------------------------- kernel registry
namespace {
std::mutex g_kernel_mu;
const KernelTable* g_user_kernels[AFMM_KERNEL_USER_COUNT] = {};
}  // namespace

bool afmm::kernel_known(int id) {
  if (id >= 0 && id <= AFMM_KERNEL_GAUSSIAN) return true;
  if (id < AFMM_KERNEL_USER_FIRST || id >= AFMM_KERNEL_USER_FIRST + AFMM_KERNEL_USER_COUNT) return false;
  std::lock_guard<std::mutex> lock(g_kernel_mu);
  return g_user_kernels[id - AFMM_KERNEL_USER_FIRST] != nullptr;
}

const KernelTable& afmm::kernel_table(int id) {
  switch (id) {
    case AFMM_KERNEL_ONE_OVER_R_SCALED: return builtin_table_one_over_r_scaled();
    case AFMM_KERNEL_LOG: return builtin_table_log();
    case AFMM_KERNEL_ONE_OVER_R: return builtin_table_one_over_r();
    case AFMM_KERNEL_GAUSSIAN: return builtin_table_gaussian();
    default: break;
  }
  if (id >= AFMM_KERNEL_USER_FIRST && id < AFMM_KERNEL_USER_FIRST + AFMM_KERNEL_USER_COUNT) {
    std::lock_guard<std::mutex> lock(g_kernel_mu);
    if (const KernelTable* t = g_user_kernels[id - AFMM_KERNEL_USER_FIRST]) return *t;
  }
  throw Error{AFMM_BAD_ARG, "unknown kernel id " + std::to_string(id)};
}

std::atomic<int64_t>& afmm::device_alloc_counter() {
  static std::atomic<int64_t> n{0};
  return n;
}

struct afmm_set {
  SetPlan plan;
  DevArena arena;
  cudaStream_t stream = nullptr;
  std::vector<int64_t> offsets;
  int64_t graph_launches = 0;
  std::vector<std::pair<std::string, double>> stage_ms;
  std::string err;
};

struct afmm_handle {
  int N = 0, M = 0, tol_pow = 0, L = 0, kernel_id = 0;
  int device = 0;
  int m2l_mode = AFMM_M2L_AUTO;  // afmm_m2l_storage
  bool m2l_stored = false;
  int m2l_q_mode = 1;            // 1: also keep a 32-bit fixed-point copy for the mixed paths; 2: and its byte planes
  int aca_cluster = 0, aca_ctas_per_sm = 0;  // ACA planner overrides (0: automatic)
  int shard_index = 0, shard_count = 1;      // afmm_set_shard
  bool m2l_q_stored = false;
  bool m2l_s_stored = false;     // byte-plane copy for the integer tensor-core M2L
  KernelParams kp{};
  cudaStream_t stream = nullptr;
  DevArena arena;
  double2* d_pts = nullptr;
  int64_t* d_perm = nullptr;
  int32_t* d_iperm = nullptr;  // original index -> sorted position
  std::vector<int32_t> h_counts, h_boxnum;          // DFS order
  std::vector<int32_t> h_leaf_start, h_leaf_cnt;    // quadtree order
  int32_t* d_leaf_start = nullptr;
  int32_t* d_leaf_cnt = nullptr;
  std::vector<LevelDev> lv;
  std::vector<std::vector<int32_t>> h_il;
  bool assembled = false;
  double* d_qs = nullptr;
  double* d_ys = nullptr;
  double* d_q = nullptr;
  double* d_y = nullptr;
  MatvecPlan plan;
  MixedState mixed;
  BatchState batch;
  StageTimer timer;
  bool profiling = false;
  std::vector<std::pair<std::string, double>> stage_ms;
  double t_create = 0, t_assemble = 0;
  int64_t launches = 0;
  int64_t counts[7] = {0, 0, 0, 0, 0, 0, 0};
  // assemble phases (wall clock, s): the rest of assemble is host work
  std::vector<std::pair<std::string, double>> setup_phase{
      {"aca", 0.0}, {"l2p", 0.0}, {"m2l_blocks", 0.0}, {"transpose_mixed", 0.0}, {"tables_alloc", 0.0},
      {"m2l_cudamalloc", 0.0}, {"level_prep", 0.0}, {"aca_alloc_other", 0.0}, {"aca_scratch_reserve", 0.0}};
  bool have_last = false;
  // host-pointer matvecs: copy streams
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
  cudaEvent_t ev_sync = nullptr;
  std::string err;
  ~afmm_handle() {
    for (cudaEvent_t e : {ev_in[0], ev_in[1], ev_done[0], ev_done[1], ev_out[0], ev_out[1], ev_sync})
      if (e) cudaEventDestroy(e);
    if (s_h2d) cudaStreamDestroy(s_h2d);
    if (s_d2h) cudaStreamDestroy(s_d2h);
  }
};

namespace {

thread_local std::string g_err;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class F>
afmm_status guard(afmm_handle* h, F&& f) {
  try {
    f();
    return AFMM_OK;
  } catch (const Error& e) {
    (h ? h->err : g_err) = e.msg;
    return e.status;
  } catch (const std::bad_alloc&) {
    (h ? h->err : g_err) = "host allocation failed";
    return AFMM_OOM;
  } catch (const std::exception& e) {
    (h ? h->err : g_err) = e.what();
    return AFMM_CUDA_ERR;
  }
}

// src/AFMM2D.cpp:7 -- nLevels = log(N/M)/log(4) with integer N/M, truncated.
int n_levels(int N, int M) {
  if (N <= 0 || M <= 0 || N / M < 1) return -1;
  unsigned L = std::log(N / M) / std::log(4);
  return (int)L;
}

void check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw Error{AFMM_NO_DEVICE, "no CUDA device available"};
  }
  int dev = 0;
  AFMM_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp p;
  AFMM_CUDA(cudaGetDeviceProperties(&p, dev));
  if (p.major != 10) throw Error{AFMM_NO_DEVICE, std::string("device is not sm_100 (B200): ") + p.name};
}

// Splitmix64, for the seeded choice of leaves in afmm_eval_error.
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// FMA throughput: 8 independent chains per thread, `iters` rounds.
template <class T>
__global__ void k_fma_peak(T seed, int iters, T* out) {
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + (T)(threadIdx.x + k);
  const T m = (T)0.999999, c = (T)1e-7;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = a[k] * m + c;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == (T)-1) out[0] = s;  // never true; keeps the chains live
}

template <class T>
double fma_peak_tflops() {
  int dev = 0, sms = 0;
  AFMM_CUDA(cudaGetDevice(&dev));
  AFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DevArena tmp;
  T* out = tmp.alloc<T>(1);
  const int blocks = sms * 8, threads = 256, iters = sizeof(T) == 8 ? 8192 : 16384;
  k_fma_peak<T><<<blocks, threads>>>((T)1, 64, out);  // warm-up
  cudaEvent_t e0, e1;
  AFMM_CUDA(cudaEventCreate(&e0));
  AFMM_CUDA(cudaEventCreate(&e1));
  AFMM_CUDA(cudaEventRecord(e0));
  k_fma_peak<T><<<blocks, threads>>>((T)1, iters, out);
  AFMM_CUDA(cudaEventRecord(e1));
  AFMM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  AFMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  AFMM_LAUNCH_CHECK();
  return 2.0 * 8.0 * (double)blocks * threads * iters / (ms * 1e-3) / 1e12;
}

// FP64 tensor (mma.sync m8n8k4) and FP64 FMA throughput: MODE 0 issues 8
// independent DMMA chains per warp, MODE 1 16 independent FMA chains per
// thread, MODE 2 both in the same loop (whether the two share a datapath).
template <int MODE>
__global__ void k_fp64_pipes(int iters, double* out) {
  double c[8][2], f[16];
  const double a = 0.999999, b = 1e-7;
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = threadIdx.x * 1e-9;
#pragma unroll
  for (int i = 0; i < 16; ++i) f[i] = threadIdx.x * 1e-9 + i;
  for (int it = 0; it < iters; ++it) {
    if (MODE != 1) {
#pragma unroll
      for (int i = 0; i < 8; ++i)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                     : "+d"(c[i][0]), "+d"(c[i][1])
                     : "d"(a), "d"(b));
    }
    if (MODE != 0) {
#pragma unroll
      for (int i = 0; i < 16; ++i) f[i] = fma(f[i], a, b);
    }
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
#pragma unroll
  for (int i = 0; i < 16; ++i) s += f[i];
  if (s == -1.0) out[0] = s;  // never true; keeps the chains live
}

// TFLOP/s of k_fp64_pipes<MODE>: {DMMA part, FMA part}.
template <int MODE>
std::pair<double, double> fp64_pipes_tflops() {
  int dev = 0, sms = 0;
  AFMM_CUDA(cudaGetDevice(&dev));
  AFMM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DevArena tmp;
  double* out = tmp.alloc<double>(1);
  const int blocks = sms * 4, threads = 256, iters = 4096;
  k_fp64_pipes<MODE><<<blocks, threads>>>(16, out);  // warm-up
  cudaEvent_t e0, e1;
  AFMM_CUDA(cudaEventCreate(&e0));
  AFMM_CUDA(cudaEventCreate(&e1));
  AFMM_CUDA(cudaEventRecord(e0));
  k_fp64_pipes<MODE><<<blocks, threads>>>(iters, out);
  AFMM_CUDA(cudaEventRecord(e1));
  AFMM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  AFMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  AFMM_LAUNCH_CHECK();
  const double warps = (double)blocks * threads / 32, s = ms * 1e-3 * 1e12;
  const double mma = MODE != 1 ? warps * iters * 8 * 512.0 / s : 0.0;
  const double fma_ = MODE != 0 ? (double)blocks * threads * iters * 16 * 2.0 / s : 0.0;
  return {mma, fma_};
}

// Narrows a box-ordered chunk table (box ids, first rows, count) to the
// chunks of boxes [bl, bh).
void narrow_table(const int32_t*& box, const int32_t*& row, long& n, long bl, long bh) {
  if (n == 0) return;
  std::vector<int32_t> hb((size_t)n);
  AFMM_CUDA(cudaMemcpy(hb.data(), box, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
  const long c0 = std::lower_bound(hb.begin(), hb.end(), (int32_t)bl) - hb.begin();
  const long c1 = std::lower_bound(hb.begin(), hb.end(), (int32_t)bh) - hb.begin();
  box += c0;
  row += c0;
  n = c1 - c0;
}

// The plan's shard views (MatvecPlan::levels_m2l, lv_down, near_own) for the
// handle's shard: at the sharded level and below, the M2L and L2L chunk
// tables narrowed to the shard's subtrees and the near field to its leaves.
void apply_shard(afmm_handle* h) {
  MatvecPlan& p = h->plan;
  p.levels_m2l = p.levels;
  p.near_own = p.near;
  for (int j = 0; j <= h->L; ++j) p.lv_down[j] = p.lv[j];
  p.shard_index = 0;
  p.shard_count = 1;
  p.shard_level = 0;
  if (h->shard_count <= 1) return;
  int lev = 0;
  long k0 = 0, k1 = 0;
  if (!shard_range(h->L, h->shard_index, h->shard_count, lev, k0, k1))
    throw Error{AFMM_BAD_ARG, "the tree has fewer leaves than shards"};
  for (int j = lev; j <= h->L; ++j) {
    const long sc = 1L << (2 * (j - lev)), bl = k0 * sc, bh = k1 * sc;
    LevelView& d = p.lv_down[j];
    narrow_table(d.ncgrp_box, d.ncgrp_row, d.nncgroups, bl, bh);
    narrow_table(d.nwgrp_box, d.nwgrp_row, d.nnwgroups, bl, bh);
    if (j >= 2) {
      LevelView m = p.lv[j];
      narrow_table(m.cgrp_box, m.cgrp_row, m.ncgroups, bl, bh);
      narrow_table(m.wgrp_box, m.wgrp_row, m.nwgroups, bl, bh);
      p.levels_m2l.lv[j - 2] = m;
    }
  }
  LevelSet& ls = p.levels_m2l;
  for (int t = 0; t < ls.nlev; ++t) {
    ls.cgrp0[t + 1] = ls.cgrp0[t] + ls.lv[t].ncgroups;
    ls.wgrp0[t + 1] = ls.wgrp0[t] + ls.lv[t].nwgroups;
  }
  const long sl = 1L << (2 * (h->L - lev));
  p.near_own.leaf0 = k0 * sl;
  p.near_own.nleaf = (k1 - k0) * sl;
  p.shard_index = h->shard_index;
  p.shard_count = h->shard_count;
  p.shard_level = lev;
}

void build_plan(afmm_handle* h) {
  MatvecPlan& p = h->plan;
  p.N = h->N;
  p.L = h->L;
  p.kp = h->kp;
  p.perm = h->d_perm;
  p.iperm = h->d_iperm;
  p.qs = h->d_qs;
  p.ys = h->d_ys;
  for (int j = 0; j <= h->L; ++j) {
    LevelDev& d = h->lv[j];
    LevelView& v = p.lv[j];
    v = LevelView();
    v.nbox = d.nbox;
    v.il = d.il;
    v.rank = d.rank;
    v.skel_off = d.skel_off;
    v.node_off = d.node_off;
    v.leaf_start = (j == h->L) ? h->d_leaf_start : nullptr;
    v.l2p_off = d.l2p_off;
    v.l2p = d.l2p;
    v.l2p_rm = d.l2p_rm;
    v.m2l_off = d.m2l_off;
    v.m2l = d.m2l;
    v.skel_xy = d.skel_xy;
    v.qhat = d.qhat;
    v.yhat = d.yhat;
    v.skel_box = d.skel_box;
    v.node_box = d.node_box;
    v.grp_box = d.grp_box;
    v.grp_row = d.grp_row;
    v.ngroups = d.ngroups;
    v.cgrp_box = d.cgrp_box;
    v.cgrp_row = d.cgrp_row;
    v.ncgroups = d.ncgroups;
    v.ncgrp_box = d.ncgrp_box;
    v.ncgrp_row = d.ncgrp_row;
    v.nncgroups = d.nncgroups;
    v.wgrp_box = d.wgrp_box;
    v.wgrp_row = d.wgrp_row;
    v.nwgroups = d.nwgroups;
    v.nwgrp_box = d.nwgrp_box;
    v.nwgrp_row = d.nwgrp_row;
    v.nnwgroups = d.nnwgroups;
    v.ptile_par = d.ptile_par;
    v.ptile_row = d.ptile_row;
    v.nptiles = d.nptiles;
    v.tile_box = d.tile_box;
    v.tile_row = d.tile_row;
    v.ntiles = d.ntiles;
    v.m2l_s = d.m2l_s;
    v.m2l_s_off = d.m2l_s_off;
    v.qs8 = d.qs8;
    v.qs8_off = d.qs8_off;
    v.qs_exp = d.qs_exp;
    v.qs_sum = d.qs_sum;
    v.m2l_q = d.m2l_q;
    v.m2l_dec = d.m2l_dec;
    v.nrows = d.total_rank;
    v.nnodes = d.h_node_off.empty() ? 0 : d.h_node_off[d.nbox];
  }
  p.levels.nlev = 0;
  p.levels.row0[0] = 0;
  p.levels.grp0[0] = 0;
  p.levels.cgrp0[0] = 0;
  p.levels.wgrp0[0] = 0;
  p.levels.pt0[0] = 0;
  p.levels.t0[0] = 0;
  p.levels.b0[0] = 0;
  for (int j = 2; j <= h->L; ++j) {
    p.levels.lv[p.levels.nlev] = p.lv[j];
    p.levels.src[p.levels.nlev] = p.levels.nlev;
    p.levels.row0[p.levels.nlev + 1] = p.levels.row0[p.levels.nlev] + p.lv[j].nrows;
    p.levels.grp0[p.levels.nlev + 1] = p.levels.grp0[p.levels.nlev] + p.lv[j].ngroups;
    p.levels.cgrp0[p.levels.nlev + 1] = p.levels.cgrp0[p.levels.nlev] + p.lv[j].ncgroups;
    p.levels.wgrp0[p.levels.nlev + 1] = p.levels.wgrp0[p.levels.nlev] + p.lv[j].nwgroups;
    p.levels.pt0[p.levels.nlev + 1] = p.levels.pt0[p.levels.nlev] + p.lv[j].nptiles;
    p.levels.t0[p.levels.nlev + 1] = p.levels.t0[p.levels.nlev] + p.lv[j].ntiles;
    p.levels.b0[p.levels.nlev + 1] = p.levels.b0[p.levels.nlev] + p.lv[j].nbox;
    ++p.levels.nlev;
  }
  for (int j = 0; j <= h->L; ++j) {
    p.rmax[j] = h->lv[j].rmax;
    p.n1max[j] = h->lv[j].n1max;
  }
  NearView& nv = p.near;
  nv.nleaf = h->lv[h->L].nbox;
  nv.nmax = *std::max_element(h->h_leaf_cnt.begin(), h->h_leaf_cnt.end());
  nv.pts = h->d_pts;
  nv.leaf_start = h->d_leaf_start;
  nv.leaf_cnt = h->d_leaf_cnt;
  nv.nbr = h->lv[h->L].nbr;
  apply_shard(h);
}

void create_layout(afmm_handle* h);

// Streams and events of a handle (afmm_create, afmm_load).
void create_streams(afmm_handle* h) {
  AFMM_CUDA(cudaGetDevice(&h->device));
  // the handle's stream at the highest priority: batched passes run their
  // near field beside the far field on a lowest-priority stream
  int least = 0, greatest = 0;
  AFMM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  AFMM_CUDA(cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, greatest));
  AFMM_CUDA(cudaStreamCreateWithFlags(&h->s_h2d, cudaStreamNonBlocking));
  AFMM_CUDA(cudaStreamCreateWithFlags(&h->s_d2h, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&h->ev_in[0], &h->ev_in[1], &h->ev_done[0], &h->ev_done[1], &h->ev_out[0], &h->ev_out[1],
                         &h->ev_sync})
    AFMM_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
}

void do_create(afmm_handle* h, const double* loc, int layout) {
  const int N = h->N, L = h->L;
  std::vector<double> xy(2 * (size_t)N);
  for (int i = 0; i < N; ++i) {
    double x = layout == AFMM_LOC_COLMAJOR ? loc[i] : loc[2 * (size_t)i];
    double y = layout == AFMM_LOC_COLMAJOR ? loc[(size_t)N + i] : loc[2 * (size_t)i + 1];
    if (!std::isfinite(x) || !std::isfinite(y))
      throw Error{AFMM_BAD_ARG, "point " + std::to_string(i) + " has a non-finite coordinate"};
    xy[2 * (size_t)i] = x;
    xy[2 * (size_t)i + 1] = y;
  }
  if ((int64_t)N >= (1LL << 28)) throw Error{AFMM_BAD_ARG, "N must be below 2^28"};
  {
    auto sz = kd_segment_sizes(N, L);
    int64_t nmax = *std::max_element(sz[L].begin(), sz[L].end());
    if (nmax > 1024) throw Error{AFMM_BAD_ARG, "leaf size " + std::to_string(nmax) + " exceeds 1024; use a smaller M"};
  }
  check_device();
  create_streams(h);
  cudaStream_t s = h->stream;
  double* d_xy = h->arena.alloc<double>(2 * (size_t)N);
  AFMM_CUDA(cudaMemcpyAsync(d_xy, xy.data(), sizeof(double) * 2 * N, cudaMemcpyHostToDevice, s));
  h->d_perm = h->arena.alloc<int64_t>(N);
  h->d_pts = h->arena.alloc<double2>(N);
  kd_sort_device(d_xy, N, L, h->d_perm, (double*)h->d_pts, s, &h->launches);
  h->arena.release(d_xy);
  create_layout(h);
}

// Everything of afmm_create after the KD sort (d_perm and d_pts set): the
// inverse permutation, the leaf layout, the lists of every level and the
// matvec buffers.
void create_layout(afmm_handle* h) {
  const int N = h->N, L = h->L;
  cudaStream_t s = h->stream;
  h->d_iperm = h->arena.alloc<int32_t>(N);
  invert_permutation(h->d_perm, N, h->d_iperm, s);
  ++h->launches;
  // Leaf layout: DFS leaf d owns a contiguous sorted range; its quadtree box
  // number follows src/KDTree.cpp:211-223 (children 4p+0, 4p+3, 4p+1, 4p+2).
  auto sizes = kd_segment_sizes(N, L);
  h->h_counts.assign(sizes[L].begin(), sizes[L].end());
  std::vector<int32_t> bn(1, 0);
  for (int j = 1; j <= L; ++j) {
    std::vector<int32_t> nx;
    nx.reserve(bn.size() * 4);
    for (int32_t p : bn) {
      nx.push_back(4 * p + 0);
      nx.push_back(4 * p + 3);
      nx.push_back(4 * p + 1);
      nx.push_back(4 * p + 2);
    }
    bn.swap(nx);
  }
  h->h_boxnum = bn;
  const long nleaf = (long)bn.size();
  h->h_leaf_start.assign(nleaf, 0);
  h->h_leaf_cnt.assign(nleaf, 0);
  int64_t st = 0;
  for (long d = 0; d < nleaf; ++d) {
    h->h_leaf_start[bn[d]] = (int32_t)st;
    h->h_leaf_cnt[bn[d]] = h->h_counts[d];
    st += h->h_counts[d];
  }
  int nmax = *std::max_element(h->h_leaf_cnt.begin(), h->h_leaf_cnt.end());
  if (nmax > 1024) throw Error{AFMM_BAD_ARG, "leaf size " + std::to_string(nmax) + " exceeds 1024; use a smaller M"};
  h->d_leaf_start = h->arena.alloc<int32_t>(nleaf);
  h->d_leaf_cnt = h->arena.alloc<int32_t>(nleaf);
  AFMM_CUDA(cudaMemcpyAsync(h->d_leaf_start, h->h_leaf_start.data(), sizeof(int32_t) * nleaf, cudaMemcpyHostToDevice, s));
  AFMM_CUDA(cudaMemcpyAsync(h->d_leaf_cnt, h->h_leaf_cnt.data(), sizeof(int32_t) * nleaf, cudaMemcpyHostToDevice, s));
  // Interaction lists of every level (closed form on the device).
  h->lv.resize(L + 1);
  h->h_il.resize(L + 1);
  for (int j = 0; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    v.nbox = 1L << (2 * j);
    v.il = h->arena.alloc<int32_t>(v.nbox * 40);
    v.nbr = h->arena.alloc<int32_t>(v.nbox * 8);
    build_lists(j, v.nbox, v.nbr, v.il, s);
    ++h->launches;
    h->h_il[j].resize(v.nbox * 40);
    AFMM_CUDA(cudaMemcpyAsync(h->h_il[j].data(), v.il, sizeof(int32_t) * v.nbox * 40, cudaMemcpyDeviceToHost, s));
  }
  // Leaf node lists (quadtree order): box k's nodes are its sorted range.
  LevelDev& lf = h->lv[L];
  lf.h_node_off.assign(nleaf + 1, 0);
  for (long k = 0; k < nleaf; ++k) lf.h_node_off[k + 1] = lf.h_node_off[k] + h->h_leaf_cnt[k];
  std::vector<int32_t> ids(N);
  for (long k = 0; k < nleaf; ++k)
    for (int i = 0; i < h->h_leaf_cnt[k]; ++i) ids[lf.h_node_off[k] + i] = h->h_leaf_start[k] + i;
  lf.node_off = h->arena.alloc<int32_t>(nleaf + 1);
  lf.node_ids = h->arena.alloc<int32_t>(N);
  AFMM_CUDA(cudaMemcpyAsync(lf.node_off, lf.h_node_off.data(), sizeof(int32_t) * (nleaf + 1), cudaMemcpyHostToDevice, s));
  AFMM_CUDA(cudaMemcpyAsync(lf.node_ids, ids.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
  h->d_qs = h->arena.alloc<double>(N + 2);  // + 16 B: whole-piece L2 prefetches of source rows
  h->d_ys = h->arena.alloc<double>(N);
  h->d_q = h->arena.alloc<double>(N);
  h->d_y = h->arena.alloc<double>(N);
  AFMM_CUDA(cudaStreamSynchronize(s));
}

void finish_assemble(afmm_handle* h);

void do_assemble(afmm_handle* h) {
  cudaStream_t s = h->stream;
  const int L = h->L;
  double tol = std::pow(10, -1.0 * h->tol_pow);  // src/ACA.cpp:7
  AcaScratch aca_scratch;  // working memory of every level's ACA and L2P, grown as needed
  for (int j = L; j >= 2; --j) {
    const double t_lv = now_s();
    LevelDev& v = h->lv[j];
    if (j < L) {
      // a box's nodes are its children's skeletons (src/AFMM2DTree.cpp:997-1007)
      LevelDev& c = h->lv[j + 1];
      v.h_node_off.assign(v.nbox + 1, 0);
      for (long b = 0; b <= v.nbox; ++b) v.h_node_off[b] = c.h_skel_off[4 * b];
      v.node_off = h->arena.alloc<int32_t>(v.nbox + 1);
      AFMM_CUDA(cudaMemcpyAsync(v.node_off, v.h_node_off.data(), sizeof(int32_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
      v.node_ids = c.skel_ids;
    }
    AcaLevelIn in;
    in.nbox = v.nbox;
    in.pts = h->d_pts;
    in.node_off = v.node_off;
    in.node_ids = v.node_ids;
    in.il = v.il;
    in.h_node_off = v.h_node_off;
    in.tol = tol;
    in.kp = h->kp;
    in.cluster = h->aca_cluster;
    in.ctas_per_sm = h->aca_ctas_per_sm;
    int n1max = 0, n2max = 0;
    const std::vector<int32_t>& il = h->h_il[j];
    for (long b = 0; b < v.nbox; ++b) {
      n1max = std::max(n1max, v.h_node_off[b + 1] - v.h_node_off[b]);
      int n2 = 0;
      for (int t = 0; t < 40; ++t) {
        int c = il[b * 40 + t];
        if (c >= 0) n2 += v.h_node_off[c + 1] - v.h_node_off[c];
      }
      n2max = std::max(n2max, n2);
    }
    in.n1max = n1max;
    in.n2max = n2max;
    v.rank = h->arena.alloc<int32_t>(v.nbox);
    in.rank_out = v.rank;
    AcaLevelOut out;
    const double t_call = now_s();
    h->setup_phase[6].second += t_call - t_lv;
    aca_level(in, out, h->arena, aca_scratch, s, &h->launches);
    h->setup_phase[7].second += now_s() - t_call - out.aca_s - out.l2p_s;
    h->setup_phase[0].second += out.aca_s;
    h->setup_phase[1].second += out.l2p_s;
    h->setup_phase.push_back({"aca_level" + std::to_string(j), out.aca_s});
    h->setup_phase.push_back({"aca_cluster_level" + std::to_string(j), (double)out.cluster});
    h->setup_phase[8].second += out.scratch_s;
    h->setup_phase.push_back({"aca_scratch_gb_level" + std::to_string(j), (double)out.scratch_bytes * 1e-9});
    v.skel_off = out.skel_off;
    v.skel_ids = out.skel_ids;
    v.cpiv_ids = out.cpiv_ids;
    v.skel_xy = out.skel_xy;
    v.l2p_off = out.l2p_off;
    v.l2p = out.l2p;
    v.h_rank = out.h_rank;
    v.h_skel_off = out.h_skel_off;
    v.h_l2p_off = out.h_l2p_off;
    v.n1max = n1max;
    v.rmax = out.rmax;
    v.total_rank = out.h_skel_off[v.nbox];
  }
  finish_assemble(h);
}

// Everything of afmm_assemble after the skeletons (rank, skel_off/ids, cpiv,
// skel_xy, l2p and their host copies of every level 2..L): M2L block sizes
// and storage, row tables, M2L blocks (FP64 and fixed point), the row-major
// L2P copy, the mixed-precision set-up and the structure counts.
// Byte planes of the fixed-point blocks (integer tensor-core M2L) and the
// per-pass buffers of the charges' planes, when they fit beside the rest.
// Per box the blocks follow in slot order, block (b, slot) taking
// ceil(r_c / 16) x 4 x ceil(r_b / 8) x 128 bytes; per box the charges take
// ceil(r / 32) x 2 KB.
void build_byte_planes(afmm_handle* h, double l2p_total, double rows_total) {
  cudaStream_t s = h->stream;
  const int L = h->L;
  std::vector<std::vector<int64_t>> soff(L + 1), qoff(L + 1);
  double need = 0.0;
  for (int j = 2; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    const std::vector<int32_t>& il = h->h_il[j];
    soff[j].assign(v.nbox + 1, 0);
    qoff[j].assign(v.nbox + 1, 0);
    for (long b = 0; b < v.nbox; ++b) {
      const int rb = v.h_rank[b];
      int64_t bytes = 0;
      for (int t = 0; t < 40 && rb > 0; ++t) {
        const int c = il[b * 40 + t];
        const int rc = c >= 0 ? v.h_rank[c] : 0;
        if (rc > 0) bytes += (int64_t)((rc + 15) / 16) * 4 * ((rb + 7) / 8) * 128;
      }
      soff[j][b + 1] = soff[j][b] + bytes;
      qoff[j][b + 1] = qoff[j][b] + (rb + 31) / 32;
    }
    need += (double)soff[j][v.nbox] + 2048.0 * (double)qoff[j][v.nbox] + 12.0 * 16 * (double)v.nbox;
  }
  size_t free_b = 0, total_b = 0;
  AFMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double reserve = 8.0 * l2p_total + (double)h->N * (16 * 8 * 4 + 64) + rows_total * 16 * 8 * 2 + 2e9;
  if (need > (double)free_b - reserve) return;
  const double t_ph = now_s();
  for (int j = 2; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    v.m2l_s_off = h->arena.alloc<int64_t>(v.nbox + 1);
    v.m2l_s = h->arena.alloc<unsigned char>((size_t)soff[j][v.nbox] + 256);
    std::vector<int32_t> q32(qoff[j].begin(), qoff[j].end());
    v.qs8_off = h->arena.alloc<int32_t>(v.nbox + 1);
    v.qs8 = h->arena.alloc<unsigned char>((size_t)qoff[j][v.nbox] * 2048 + 256);
    v.qs_exp = h->arena.alloc<int32_t>((size_t)v.nbox * 16);
    v.qs_sum = h->arena.alloc<int64_t>((size_t)v.nbox * 16);
    AFMM_CUDA(cudaMemcpyAsync(v.m2l_s_off, soff[j].data(), sizeof(int64_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
    AFMM_CUDA(cudaMemcpyAsync(v.qs8_off, q32.data(), sizeof(int32_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
    AFMM_CUDA(cudaStreamSynchronize(s));
  }
  build_plan(h);
  for (int j = 2; j <= L; ++j) {
    m2l_slice(h->plan.lv[j], s);
    ++h->launches;
  }
  AFMM_CUDA(cudaStreamSynchronize(s));
  h->m2l_s_stored = true;
  h->setup_phase[2].second += now_s() - t_ph;
}

void finish_assemble(afmm_handle* h) {
  cudaStream_t s = h->stream;
  const int L = h->L;
  // M2L blocks, levels 2..L: sizes first, then the storage decision
  const double t_tab = now_s();
  int64_t m2l_total = 0, l2p_total = 0, rows_total = 0;
  for (int j = 2; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    const std::vector<int32_t>& il = h->h_il[j];
    v.h_m2l_off.assign(v.nbox + 1, 0);
    for (long b = 0; b < v.nbox; ++b) {
      int64_t e = 0;
      for (int t = 0; t < 40; ++t) {
        int c = il[b * 40 + t];
        if (c >= 0) e += (int64_t)v.h_rank[b] * v.h_rank[c];
      }
      v.h_m2l_off[b + 1] = v.h_m2l_off[b] + e;
    }
    m2l_total += v.h_m2l_off[v.nbox];
    l2p_total += v.h_l2p_off[v.nbox];
    rows_total += v.total_rank;
  }
  {
    // AUTO stores the blocks when they fit beside what the matvecs still
    // allocate (the row-major L2P copy, the mixed and 16-column batched
    // buffers) with 2 GB to spare
    size_t free_b = 0, total_b = 0;
    AFMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double need = 8.0 * (double)m2l_total;
    const double reserve = 8.0 * (double)l2p_total + (double)h->N * (16 * 8 * 4 + 64) +
                           (double)rows_total * 16 * 8 * 2 + 2e9;
    h->m2l_stored = h->m2l_mode == AFMM_M2L_STORE ||
                    (h->m2l_mode == AFMM_M2L_AUTO && need <= (double)free_b - reserve);
  }
  for (int j = 2; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    v.m2l_off = h->arena.alloc<int64_t>(v.nbox + 1);
    AFMM_CUDA(cudaMemcpyAsync(v.m2l_off, v.h_m2l_off.data(), sizeof(int64_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
    // + 256 B for whole-piece L2 prefetches
    const double t_al = now_s();
    v.m2l = h->m2l_stored ? h->arena.alloc<double>(v.h_m2l_off[v.nbox] + 32) : nullptr;
    h->setup_phase[5].second += now_s() - t_al;
    v.qhat = h->arena.alloc<double>(v.total_rank + 2);  // + 16 B: whole-piece L2 prefetches
    v.yhat = h->arena.alloc<double>(v.total_rank);
    // row -> box maps for the thread-per-row sweeps
    v.skel_box = h->arena.alloc<int32_t>(v.total_rank);
    v.node_box = h->arena.alloc<int32_t>(v.h_node_off[v.nbox]);
    fill_box_map(v.skel_off, v.nbox, v.skel_box, s);
    fill_box_map(v.node_off, v.nbox, v.node_box, s);
    h->launches += 2;
    // row groups of at most 8 skeleton rows of one box (on-the-fly M2L
    // tiles), balanced chunks of at most kChunkRows skeleton rows (M2L / M2M
    // tiles) or node rows (L2L tiles): a box of n rows is cut into
    // ceil(n / kChunkRows) chunks of equal size rounded up to 8 rows; and
    // balanced chunks of at most 32 skeleton rows (a warp's lanes, the
    // one-column M2L)
    // (and the same of at most 32 node rows, the one-column L2L); and tiles
    // of 128 skeleton rows (the last shorter: the integer tensor-core M2L)
    for (int kind = 0; kind < 6; ++kind) {
      const int span = kind == 0 ? 8 : (kind == 5 ? 128 : (kind >= 3 ? 32 : kChunkRows));
      const bool nodes = kind == 2 || kind == 4;
      std::vector<int32_t> gb, gr;
      for (long b = 0; b < v.nbox; ++b) {
        const int rows = nodes ? v.h_node_off[b + 1] - v.h_node_off[b] : v.h_rank[b];
        const int first = nodes ? v.h_node_off[b] : v.h_skel_off[b];
        const int nch = (rows + span - 1) / span;
        int step = nch > 0 ? (rows + nch - 1) / nch : 0;
        if (kind == 1 || kind == 2) step = (step + 7) / 8 * 8;
        if (kind == 5) step = span;  // whole 128-row tiles, the last one shorter
        for (int i = 0; i < rows; i += (kind == 0 ? 8 : step)) {
          gb.push_back((int32_t)b);
          gr.push_back(kind == 5 ? i : first + i);  // 128-row tiles: the row within the box
        }
      }
      int32_t* db = h->arena.alloc<int32_t>(gb.size());
      int32_t* dr = h->arena.alloc<int32_t>(gr.size());
      if (!gb.empty()) {
        AFMM_CUDA(cudaMemcpyAsync(db, gb.data(), sizeof(int32_t) * gb.size(), cudaMemcpyHostToDevice, s));
        AFMM_CUDA(cudaMemcpyAsync(dr, gr.data(), sizeof(int32_t) * gr.size(), cudaMemcpyHostToDevice, s));
        AFMM_CUDA(cudaStreamSynchronize(s));
      }
      if (kind == 0) {
        v.ngroups = (long)gb.size();
        v.grp_box = db;
        v.grp_row = dr;
      } else if (kind == 1) {
        v.ncgroups = (long)gb.size();
        v.cgrp_box = db;
        v.cgrp_row = dr;
      } else if (kind == 2) {
        v.nncgroups = (long)gb.size();
        v.ncgrp_box = db;
        v.ncgrp_row = dr;
      } else if (kind == 3) {
        v.nwgroups = (long)gb.size();
        v.wgrp_box = db;
        v.wgrp_row = dr;
      } else if (kind == 5) {
        v.ntiles = (long)gb.size();
        v.tile_box = db;
        v.tile_row = dr;
      } else {
        v.nnwgroups = (long)gb.size();
        v.nwgrp_box = db;
        v.nwgrp_row = dr;
      }
    }
    {
      // row tiles of the tcgen05 M2L: per parent box, the four children's
      // skeleton rows concatenated and cut into ceil(R / 128) balanced tiles
      std::vector<int32_t> tp, tr;
      for (long P = 0; P < v.nbox / 4; ++P) {
        int R = 0;
        for (int c = 0; c < 4; ++c) R += v.h_rank[4 * P + c];
        const int nt = (R + 127) / 128;
        for (int t = 0; t < nt; ++t) {
          tp.push_back((int32_t)P);
          tr.push_back((int32_t)((long)t * R / nt));
        }
      }
      v.nptiles = (long)tp.size();
      v.ptile_par = h->arena.alloc<int32_t>(std::max<size_t>(tp.size(), 1));
      v.ptile_row = h->arena.alloc<int32_t>(std::max<size_t>(tr.size(), 1));
      if (!tp.empty()) {
        AFMM_CUDA(cudaMemcpyAsync(v.ptile_par, tp.data(), sizeof(int32_t) * tp.size(), cudaMemcpyHostToDevice, s));
        AFMM_CUDA(cudaMemcpyAsync(v.ptile_row, tr.data(), sizeof(int32_t) * tr.size(), cudaMemcpyHostToDevice, s));
        AFMM_CUDA(cudaStreamSynchronize(s));
      }
    }
  }
  for (int j = 2; j <= L; ++j) {
    LevelDev& v = h->lv[j];
    v.l2p_rm = h->arena.alloc<double>(v.h_l2p_off[v.nbox] + 4);  // + 32 B for whole-piece L2 prefetches
  }
  build_plan(h);
  AFMM_CUDA(cudaStreamSynchronize(s));
  h->setup_phase[4].second += now_s() - t_tab;
  AFMM_CUDA(cudaStreamSynchronize(s));
  double t_ph = now_s();
  for (int j = 2; j <= L; ++j) {
    if (h->m2l_stored) {
      m2l_assemble(h->plan.lv[j], h->kp, s);
      ++h->launches;
    }
  }
  AFMM_CUDA(cudaStreamSynchronize(s));
  h->setup_phase[2].second += now_s() - t_ph;
  // 32-bit fixed-point copy of the blocks for the mixed-precision paths, when
  // it fits beside the rest (half the bytes of the FP64 blocks)
  if (h->m2l_stored && h->m2l_q_mode) {
    size_t free_b = 0, total_b = 0;
    AFMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double need = 4.0 * (double)m2l_total;
    const double reserve = 8.0 * (double)l2p_total + (double)h->N * (16 * 8 * 4 + 64) +
                           (double)rows_total * 16 * 8 * 2 + 2e9;
    if (need <= (double)free_b - reserve) {
      t_ph = now_s();
      for (int j = 2; j <= L; ++j) {
        LevelDev& v = h->lv[j];
        v.m2l_q = h->arena.alloc<uint32_t>(v.h_m2l_off[v.nbox] + 64);  // + 256 B for whole-piece L2 prefetches
        v.m2l_dec = h->arena.alloc<double2>((size_t)v.nbox * 40);
      }
      build_plan(h);
      for (int j = 2; j <= L; ++j) {
        m2l_compress(h->plan.lv[j], s);
        ++h->launches;
      }
      AFMM_CUDA(cudaStreamSynchronize(s));
      h->m2l_q_stored = true;
      h->setup_phase[2].second += now_s() - t_ph;
      if (h->m2l_q_mode == 2) build_byte_planes(h, l2p_total, rows_total);
    }
  }
  t_ph = now_s();
  for (int j = 2; j <= L; ++j) {
    l2p_transpose(h->plan.lv[j], h->lv[j].l2p, h->lv[j].l2p_rm, s);
    ++h->launches;
  }
  mixed_setup(h->plan, h->lv, h->mixed, h->arena, s, &h->launches);
  build_plan(h);
  AFMM_CUDA(cudaStreamSynchronize(s));
  h->setup_phase[3].second += now_s() - t_ph;
  // structure counts
  int64_t sum_rank = 0, l2p_entries = 0;
  for (int j = 2; j <= L; ++j) {
    sum_rank += h->lv[j].total_rank;
    l2p_entries += h->lv[j].h_l2p_off[h->lv[j].nbox];
  }
  int64_t near = 0;
  const std::vector<int32_t>& il = h->h_il[L];
  (void)il;
  std::vector<int32_t> nbr(h->lv[L].nbox * 8);
  AFMM_CUDA(cudaMemcpy(nbr.data(), h->lv[L].nbr, sizeof(int32_t) * nbr.size(), cudaMemcpyDeviceToHost));
  for (long b = 0; b < h->lv[L].nbox; ++b) {
    int64_t src = h->h_leaf_cnt[b];
    for (int t = 0; t < 8; ++t)
      if (nbr[b * 8 + t] >= 0) src += h->h_leaf_cnt[nbr[b * 8 + t]];
    near += src * h->h_leaf_cnt[b];
  }
  h->counts[0] = L;
  h->counts[1] = h->N;
  h->counts[2] = sum_rank;
  h->counts[3] = l2p_entries;
  h->counts[4] = m2l_total;
  h->counts[5] = near;
  h->counts[6] = m2l_total;
  h->assembled = true;
}

// ------------------------------------------------------- setup files
// Versioned binary image of an assembled handle (afmm_save / afmm_load):
// everything ACA decided -- the KD permutation and sorted points, and per
// level the ranks, skeletons (incoming check points), pivot columns and L2P
// operators -- so that a later process skips the KD sort and the ACA.  The
// lists, row tables and M2L blocks are rebuilt from these by the same code
// as afmm_assemble, so a loaded handle's matvecs have the bits of the
// original's.  Layout (little-endian, native widths):
//   char[8] "AFMM2DB\n"; u32 version; u32 0x01020304 (byte order check)
//   i32 N, M, TOL_POW, L, kernel id, M2L storage mode, fixed-point flag, 0
//   f64 a, kernel parameter
//   f64 sorted points [2N]; i64 permutation [N]
//   per level j = L..2: i64 boxes, i64 skeleton rows, i64 L2P entries;
//     i32 ranks [boxes]; i32 skeleton ids [rows]; i32 pivot columns [rows];
//     f64 L2P [entries] (per box n_b x r_b, column-major)
//   u64 FNV-1a digest of all bytes before (64-bit words, then the tail bytes)
constexpr char kSetupMagic[8] = {'A', 'F', 'M', 'M', '2', 'D', 'B', '\n'};
constexpr uint32_t kSetupVersion = 1;

// FNV-1a over the byte stream taken 8 bytes at a time (little-endian
// words), the last partial word byte by byte; independent of how the stream
// is split into add() calls.
struct Fnv64 {
  static constexpr uint64_t kPrime = 1099511628211ull;
  uint64_t h = 1469598103934665603ull;
  unsigned char buf[8];
  int nb = 0;
  void word(const unsigned char* b) {
    uint64_t x;
    std::memcpy(&x, b, 8);
    h = (h ^ x) * kPrime;
  }
  void add(const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    while (n && nb) {
      buf[nb++] = *b++;
      --n;
      if (nb == 8) {
        word(buf);
        nb = 0;
      }
    }
    for (; n >= 8; n -= 8, b += 8) word(b);
    while (n) {
      buf[nb++] = *b++;
      --n;
    }
  }
  uint64_t digest() {
    for (int i = 0; i < nb; ++i) h = (h ^ buf[i]) * kPrime;
    nb = 0;
    return h;
  }
};

struct SetupWriter {
  FILE* f = nullptr;
  Fnv64 dig;
  explicit SetupWriter(const char* path) : f(std::fopen(path, "wb")) {
    if (!f) throw Error{AFMM_BAD_ARG, std::string("cannot open ") + path + " for writing"};
  }
  ~SetupWriter() {
    if (f) std::fclose(f);
  }
  void put(const void* p, size_t n) {
    dig.add(p, n);
    if (n && std::fwrite(p, 1, n, f) != n) throw Error{AFMM_BAD_ARG, "write failed"};
  }
  template <class T>
  void put_vec(const std::vector<T>& v) {
    put(v.data(), sizeof(T) * v.size());
  }
  void finish() {
    const uint64_t d = dig.digest();
    if (std::fwrite(&d, 8, 1, f) != 1 || std::fclose(f) != 0) {
      f = nullptr;
      throw Error{AFMM_BAD_ARG, "write failed"};
    }
    f = nullptr;
  }
};

struct SetupReader {
  FILE* f = nullptr;
  Fnv64 dig;
  explicit SetupReader(const char* path) : f(std::fopen(path, "rb")) {
    if (!f) throw Error{AFMM_BAD_ARG, std::string("cannot open ") + path};
  }
  ~SetupReader() {
    if (f) std::fclose(f);
  }
  void get(void* p, size_t n) {
    if (n && std::fread(p, 1, n, f) != n) throw Error{AFMM_BAD_ARG, "setup file is truncated"};
    dig.add(p, n);
  }
  template <class T>
  T val() {
    T x;
    get(&x, sizeof(T));
    return x;
  }
  template <class T>
  void get_vec(std::vector<T>& v, int64_t n) {
    if (n < 0 || n > (int64_t)1 << 40) throw Error{AFMM_BAD_ARG, "setup file has a bad size field"};
    v.resize((size_t)n);
    get(v.data(), sizeof(T) * (size_t)n);
  }
  void finish() {
    uint64_t d = 0;
    if (std::fread(&d, 8, 1, f) != 1) throw Error{AFMM_BAD_ARG, "setup file is truncated"};
    if (d != dig.digest()) throw Error{AFMM_BAD_ARG, "setup file digest mismatch (corrupted file)"};
    if (std::fgetc(f) != EOF) throw Error{AFMM_BAD_ARG, "setup file has trailing bytes"};
  }
};

struct SetupLevel {
  std::vector<int32_t> rank, skel_ids, cpiv_ids;
  std::vector<double> l2p;
};

struct SetupImage {
  int N = 0, M = 0, tol_pow = 0, L = 0, kernel_id = 0, m2l_mode = 0, q_mode = 0;
  double a = 0, param = 0;
  std::vector<double> pts;
  std::vector<int64_t> perm;
  std::vector<SetupLevel> lv;  // index j = level
};

void do_save(afmm_handle* h, const char* path) {
  if (!h->assembled) throw Error{AFMM_NOT_ASSEMBLED, "afmm_save before afmm_assemble"};
  const int N = h->N, L = h->L;
  AFMM_CUDA(cudaStreamSynchronize(h->stream));
  std::vector<double> pts(2 * (size_t)N);
  std::vector<int64_t> perm(N);
  AFMM_CUDA(cudaMemcpy(pts.data(), h->d_pts, sizeof(double) * pts.size(), cudaMemcpyDeviceToHost));
  AFMM_CUDA(cudaMemcpy(perm.data(), h->d_perm, sizeof(int64_t) * N, cudaMemcpyDeviceToHost));
  SetupWriter w(path);
  w.put(kSetupMagic, 8);
  const uint32_t ver[2] = {kSetupVersion, 0x01020304u};
  w.put(ver, sizeof(ver));
  const int32_t hdr[8] = {N, h->M, h->tol_pow, L, h->kernel_id, h->m2l_mode, h->m2l_q_mode, 0};
  w.put(hdr, sizeof(hdr));
  const double par[2] = {h->kp.a, h->kp.param};
  w.put(par, sizeof(par));
  w.put_vec(pts);
  w.put_vec(perm);
  for (int j = L; j >= 2; --j) {
    const LevelDev& v = h->lv[j];
    const int64_t tr = v.total_rank, ne = v.h_l2p_off[v.nbox];
    const int64_t sz[3] = {v.nbox, tr, ne};
    w.put(sz, sizeof(sz));
    w.put_vec(v.h_rank);
    std::vector<int32_t> ids(tr);
    std::vector<double> l2p(ne);
    if (tr) AFMM_CUDA(cudaMemcpy(ids.data(), v.skel_ids, sizeof(int32_t) * tr, cudaMemcpyDeviceToHost));
    w.put_vec(ids);
    if (tr) AFMM_CUDA(cudaMemcpy(ids.data(), v.cpiv_ids, sizeof(int32_t) * tr, cudaMemcpyDeviceToHost));
    w.put_vec(ids);
    if (ne) AFMM_CUDA(cudaMemcpy(l2p.data(), v.l2p, sizeof(double) * ne, cudaMemcpyDeviceToHost));
    w.put_vec(l2p);
  }
  w.finish();
}

// Reads and checks a setup file on the host (no device work).
SetupImage read_setup(const char* path) {
  SetupReader r(path);
  char magic[8];
  r.get(magic, 8);
  if (std::memcmp(magic, kSetupMagic, 8) != 0) throw Error{AFMM_BAD_ARG, "not an AFMM2D setup file"};
  const uint32_t ver = r.val<uint32_t>(), bom = r.val<uint32_t>();
  if (bom != 0x01020304u) throw Error{AFMM_BAD_ARG, "setup file written with another byte order"};
  if (ver != kSetupVersion) throw Error{AFMM_BAD_ARG, "setup file version " + std::to_string(ver) + " not supported"};
  SetupImage im;
  int32_t hdr[8];
  r.get(hdr, sizeof(hdr));
  im.N = hdr[0];
  im.M = hdr[1];
  im.tol_pow = hdr[2];
  im.L = hdr[3];
  im.kernel_id = hdr[4];
  im.m2l_mode = hdr[5];
  im.q_mode = hdr[6];
  double par[2];
  r.get(par, sizeof(par));
  im.a = par[0];
  im.param = par[1];
  if (im.N < 1 || im.M < 1 || im.L < 2 || im.L >= kMaxLevels || im.L != n_levels(im.N, im.M) || im.m2l_mode < 0 ||
      im.m2l_mode > 2 || im.q_mode < 0 || im.q_mode > 2)
    throw Error{AFMM_BAD_ARG, "setup file header is inconsistent"};
  if (!kernel_known(im.kernel_id))
    throw Error{AFMM_BAD_ARG, "setup file uses kernel id " + std::to_string(im.kernel_id) + ", which is not registered"};
  const int N = im.N, L = im.L;
  r.get_vec(im.pts, 2 * (int64_t)N);
  r.get_vec(im.perm, N);
  std::vector<char> seen(N, 0);
  for (int64_t p : im.perm) {
    if (p < 0 || p >= N || seen[p]) throw Error{AFMM_BAD_ARG, "setup file permutation is not a permutation"};
    seen[p] = 1;
  }
  for (double x : im.pts)
    if (!std::isfinite(x)) throw Error{AFMM_BAD_ARG, "setup file holds a non-finite point"};
  im.lv.resize(L + 1);
  for (int j = L; j >= 2; --j) {
    SetupLevel& lv = im.lv[j];
    int64_t sz[3];
    r.get(sz, sizeof(sz));
    if (sz[0] != ((int64_t)1 << (2 * j))) throw Error{AFMM_BAD_ARG, "setup file level size mismatch"};
    r.get_vec(lv.rank, sz[0]);
    int64_t tr = 0;
    for (int32_t x : lv.rank) {
      if (x < 0) throw Error{AFMM_BAD_ARG, "setup file holds a negative rank"};
      tr += x;
    }
    if (tr != sz[1]) throw Error{AFMM_BAD_ARG, "setup file rank sum mismatch"};
    r.get_vec(lv.skel_ids, sz[1]);
    r.get_vec(lv.cpiv_ids, sz[1]);
    for (int32_t x : lv.skel_ids)
      if (x < 0 || x >= N) throw Error{AFMM_BAD_ARG, "setup file skeleton id out of range"};
    for (int32_t x : lv.cpiv_ids)
      if (x < 0 || x >= N) throw Error{AFMM_BAD_ARG, "setup file pivot id out of range"};
    r.get_vec(lv.l2p, sz[2]);
  }
  r.finish();
  return im;
}

// The ACA results of every level from a setup image (in place of the level
// loop of do_assemble); the L2P sizes are checked against the node counts.
void load_levels(afmm_handle* h, SetupImage& im) {
  cudaStream_t s = h->stream;
  const int L = h->L;
  for (int j = L; j >= 2; --j) {
    LevelDev& v = h->lv[j];
    SetupLevel& f = im.lv[j];
    if (j < L) {
      LevelDev& c = h->lv[j + 1];
      v.h_node_off.assign(v.nbox + 1, 0);
      for (long b = 0; b <= v.nbox; ++b) v.h_node_off[b] = c.h_skel_off[4 * b];
      v.node_off = h->arena.alloc<int32_t>(v.nbox + 1);
      AFMM_CUDA(cudaMemcpyAsync(v.node_off, v.h_node_off.data(), sizeof(int32_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
      v.node_ids = c.skel_ids;
    }
    v.h_rank = f.rank;
    v.h_skel_off.assign(v.nbox + 1, 0);
    v.h_l2p_off.assign(v.nbox + 1, 0);
    int n1max = 0, rmax = 0;
    for (long b = 0; b < v.nbox; ++b) {
      const int n = v.h_node_off[b + 1] - v.h_node_off[b];
      if (v.h_rank[b] > n) throw Error{AFMM_BAD_ARG, "setup file rank exceeds its box's node count"};
      v.h_skel_off[b + 1] = v.h_skel_off[b] + v.h_rank[b];
      v.h_l2p_off[b + 1] = v.h_l2p_off[b] + (int64_t)n * v.h_rank[b];
      n1max = std::max(n1max, n);
      rmax = std::max(rmax, v.h_rank[b]);
    }
    if (v.h_l2p_off[v.nbox] != (int64_t)f.l2p.size()) throw Error{AFMM_BAD_ARG, "setup file L2P size mismatch"};
    v.n1max = n1max;
    v.rmax = rmax;
    v.total_rank = v.h_skel_off[v.nbox];
    const long tr = v.total_rank;
    v.rank = h->arena.alloc<int32_t>(v.nbox);
    v.skel_off = h->arena.alloc<int32_t>(v.nbox + 1);
    v.l2p_off = h->arena.alloc<int64_t>(v.nbox + 1);
    v.skel_ids = h->arena.alloc<int32_t>(tr);
    v.cpiv_ids = h->arena.alloc<int32_t>(tr);
    v.skel_xy = h->arena.alloc<double2>(tr);
    v.l2p = h->arena.alloc<double>(f.l2p.size() + 4);  // + 32 B for whole-piece L2 prefetches
    AFMM_CUDA(cudaMemcpyAsync(v.rank, v.h_rank.data(), sizeof(int32_t) * v.nbox, cudaMemcpyHostToDevice, s));
    AFMM_CUDA(cudaMemcpyAsync(v.skel_off, v.h_skel_off.data(), sizeof(int32_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
    AFMM_CUDA(cudaMemcpyAsync(v.l2p_off, v.h_l2p_off.data(), sizeof(int64_t) * (v.nbox + 1), cudaMemcpyHostToDevice, s));
    if (tr) {
      AFMM_CUDA(cudaMemcpyAsync(v.skel_ids, f.skel_ids.data(), sizeof(int32_t) * tr, cudaMemcpyHostToDevice, s));
      AFMM_CUDA(cudaMemcpyAsync(v.cpiv_ids, f.cpiv_ids.data(), sizeof(int32_t) * tr, cudaMemcpyHostToDevice, s));
    }
    if (!f.l2p.empty())
      AFMM_CUDA(cudaMemcpyAsync(v.l2p, f.l2p.data(), sizeof(double) * f.l2p.size(), cudaMemcpyHostToDevice, s));
    gather_points(h->d_pts, v.skel_ids, tr, v.skel_xy, s);
    ++h->launches;
    AFMM_CUDA(cudaStreamSynchronize(s));  // the host vectors of f may be freed after this
  }
}

// Host-pointer matvec: passes of at most W columns, each copied in on the
// h2d stream, computed on the handle's stream and copied out on the d2h
// stream, with two staging buffers so that the copies of one pass overlap the
// computation of its neighbours.  compute(qd, yd, nc) runs nc columns from
// device staging (leading dimension N) on the handle's stream.
template <class F>
void host_pipeline(afmm_handle* h, const double* q, double* y, int nrhs, int64_t ld, int W, F&& compute) {
  const int N = h->N;
  const size_t need = 2 * (size_t)W;
  if (h->mixed.host_cap < need) {
    if (h->mixed.d_qin) h->arena.release(h->mixed.d_qin);
    if (h->mixed.d_yout) h->arena.release(h->mixed.d_yout);
    mixed_reserve_io(h->mixed, N, (int)need, h->arena);
  }
  cudaStream_t s = h->stream, si = h->s_h2d, so = h->s_d2h;
  const size_t bytes = sizeof(double) * (size_t)N;
  // the copy streams start after the work already queued on the handle's stream
  AFMM_CUDA(cudaEventRecord(h->ev_sync, s));
  AFMM_CUDA(cudaStreamWaitEvent(si, h->ev_sync, 0));
  AFMM_CUDA(cudaStreamWaitEvent(so, h->ev_sync, 0));
  int k = 0;
  for (int c0 = 0; c0 < nrhs; c0 += W, ++k) {
    const int nc = std::min(W, nrhs - c0), buf = k & 1;
    double* qb = h->mixed.d_qin + (size_t)buf * W * N;
    double* yb = h->mixed.d_yout + (size_t)buf * W * N;
    if (k >= 2) AFMM_CUDA(cudaStreamWaitEvent(si, h->ev_done[buf], 0));  // pass k-2 has read qb
    for (int c = 0; c < nc; ++c)
      AFMM_CUDA(cudaMemcpyAsync(qb + (size_t)c * N, q + (size_t)(c0 + c) * ld, bytes, cudaMemcpyHostToDevice, si));
    AFMM_CUDA(cudaEventRecord(h->ev_in[buf], si));
    AFMM_CUDA(cudaStreamWaitEvent(s, h->ev_in[buf], 0));
    if (k >= 2) AFMM_CUDA(cudaStreamWaitEvent(s, h->ev_out[buf], 0));  // pass k-2's results have left yb
    compute(qb, yb, nc);
    AFMM_CUDA(cudaEventRecord(h->ev_done[buf], s));
    AFMM_CUDA(cudaStreamWaitEvent(so, h->ev_done[buf], 0));
    for (int c = 0; c < nc; ++c)
      AFMM_CUDA(cudaMemcpyAsync(y + (size_t)(c0 + c) * ld, yb + (size_t)c * N, bytes, cudaMemcpyDeviceToHost, so));
    AFMM_CUDA(cudaEventRecord(h->ev_out[buf], so));
  }
  // the handle's stream ends after the last copy out
  AFMM_CUDA(cudaEventRecord(h->ev_sync, so));
  AFMM_CUDA(cudaStreamWaitEvent(s, h->ev_sync, 0));
}


// A kernel whose bounded device wait gave up leaves the batch error flag set
// (host-mapped): report it once the stream is synchronised.
void check_device_flag(afmm_handle* h) {
  AFMM_CUDA(cudaStreamSynchronize(h->stream));
  if (h->batch.err_host && *(volatile int*)h->batch.err_host) {
    *(volatile int*)h->batch.err_host = 0;
    throw Error{AFMM_TIMEOUT, "a bounded device wait gave up (tcgen05 near field); the results are incomplete"};
  }
}

// ------------------------------------------------------------ autotuner
// Times the tunable launch parameters (Tuning) on the handle's own problem
// with CUDA events on its stream and keeps the fastest: the L2 prefetch
// windows of the stored-block M2L kernels, per level the stored or on-the-fly
// M2L form of the one-column and batched mixed paths, and the pass width of
// host-pointer batched calls.  None changes the FP64 path's results; the
// mixed forms agree within the mixed tolerance.  A cache file keyed by the
// device and the problem's structure makes repeated tuning free.

// Median of `reps` timed runs of f (after one warm-up), ms.
template <class F>
float time_ms(cudaStream_t s, int reps, F&& f) {
  cudaEvent_t e0, e1;
  AFMM_CUDA(cudaEventCreate(&e0));
  AFMM_CUDA(cudaEventCreate(&e1));
  f();
  std::vector<float> t;
  for (int r = 0; r < reps; ++r) {
    AFMM_CUDA(cudaEventRecord(e0, s));
    f();
    AFMM_CUDA(cudaEventRecord(e1, s));
    AFMM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    AFMM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    t.push_back(ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::sort(t.begin(), t.end());
  return t[t.size() / 2];
}

std::string tuning_key(afmm_handle* h) {
  cudaDeviceProp pr;
  AFMM_CUDA(cudaGetDeviceProperties(&pr, h->device));
  std::string name = pr.name;
  for (char& c : name)
    if (c == ' ' || c == '|') c = '_';
  return "dev=" + name + "|N=" + std::to_string(h->N) + "|M=" + std::to_string(h->M) + "|L=" + std::to_string(h->L) +
         "|kernel=" + std::to_string(h->kernel_id) + "|tol=" + std::to_string(h->tol_pow) +
         "|stored=" + std::to_string((h->m2l_stored ? 1 : 0) + (h->m2l_q_stored ? 2 : 0)) +
         "|ranks=" + std::to_string(h->counts[2]) + "|entries=" + std::to_string(h->counts[4]);
}

constexpr int kTuningValues = 8;
constexpr int kTuningValuesMin = 7;  // callers written before the eighth value (m2l_tc) pass 7

void tuning_to(const Tuning& t, int64_t* v) {
  v[0] = t.pf_fp64;
  v[1] = t.pf_batched;
  v[2] = t.otf_mixed;
  v[3] = t.otf_batched;
  v[4] = t.host_pass_cols;
  v[5] = t.m2l_t16;
  v[6] = t.p2p_tc;
  v[7] = t.m2l_tc;
}

Tuning tuning_from(const int64_t* v) {
  if (v[0] < 0 || v[0] > (1 << 20) || v[1] < 0 || v[1] > (1 << 20) || v[2] < 0 || v[2] > 0xffffffffll || v[3] < 0 ||
      v[3] > 0xffffffffll || v[4] < 0 || v[4] > kBatchMax || (v[0] % 16) || (v[1] % 16) || v[5] < 0 || v[5] > 1 ||
      v[6] < 0 || v[6] > 1 || v[7] < 0 || v[7] > 2)
    throw Error{AFMM_BAD_ARG,
                "tuning values out of range (windows: multiples of 16 up to 1 MiB; pass width <= 16; switches 0 or 1)"};
  Tuning t;
  t.pf_fp64 = (uint32_t)v[0];
  t.pf_batched = (uint32_t)v[1];
  t.otf_mixed = (uint32_t)v[2];
  t.otf_batched = (uint32_t)v[3];
  t.host_pass_cols = (int)v[4];
  t.m2l_t16 = (int)v[5];
  t.p2p_tc = (int)v[6];
  t.m2l_tc = (int)v[7];
  return t;
}

bool cache_lookup(const char* path, const std::string& key, Tuning& t) {
  if (!path) return false;
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  char line[4096];
  bool hit = false;
  while (std::fgets(line, sizeof(line), f)) {
    std::string l(line);
    const size_t sp = l.find(' ');
    if (sp == std::string::npos || l.compare(0, sp, key) != 0 || sp != key.size()) continue;
    long long v[kTuningValues];
    if (std::sscanf(l.c_str() + sp, "%lld %lld %lld %lld %lld %lld %lld %lld", &v[0], &v[1], &v[2], &v[3], &v[4],
                    &v[5], &v[6], &v[7]) == kTuningValues) {
      int64_t w[kTuningValues] = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
      try {
        t = tuning_from(w);
        hit = true;  // the last matching line wins
      } catch (const Error&) {
      }
    }
  }
  std::fclose(f);
  return hit;
}

void cache_store(const char* path, const std::string& key, const Tuning& t) {
  if (!path) return;
  FILE* f = std::fopen(path, "a");
  if (!f) throw Error{AFMM_BAD_ARG, std::string("cannot write the tuning cache ") + path};
  int64_t v[kTuningValues];
  tuning_to(t, v);
  std::fprintf(f, "%s %lld %lld %lld %lld %lld %lld %lld %lld\n", key.c_str(), (long long)v[0], (long long)v[1],
               (long long)v[2], (long long)v[3], (long long)v[4], (long long)v[5], (long long)v[6], (long long)v[7]);
  std::fclose(f);
}

void do_autotune(afmm_handle* h, int what) {
  cudaStream_t s = h->stream;
  MatvecPlan& p = h->plan;
  const int N = h->N;
  const int nlev = p.levels.nlev;
  const bool q32 = h->m2l_q_stored, fp64b = h->m2l_stored;
  // outgoing charges of every level for the M2L timings: one FP64 matvec and
  // one 16-column mixed pass of seeded random charges
  DevArena tmp;
  const int R = kBatchMax;
  double* dq = tmp.alloc<double>((size_t)N * R);
  double* dy = tmp.alloc<double>((size_t)N * R);
  {
    std::vector<double> hq((size_t)N * R);
    uint64_t st = 0xA5A5F00Dull;
    for (double& x : hq) x = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    AFMM_CUDA(cudaMemcpyAsync(dq, hq.data(), sizeof(double) * hq.size(), cudaMemcpyHostToDevice, s));
    AFMM_CUDA(cudaStreamSynchronize(s));
  }
  mixed_reserve(h->mixed, N, 1, h->arena);
  batch_reserve(p, h->batch, h->arena, s);
  int64_t launches = 0;
  matvec_fp64(p, dq, dy, s, nullptr, &launches);
  matvec_batched(p, h->mixed, h->batch, dq, N, dy, N, R, 0, s, nullptr, &launches);
  const int reps = 5;
  const uint32_t windows[] = {0, 4096, 8192, 12288, 16384, 24576, 32768};
  if ((what & 1) && nlev > 0 && (fp64b || q32)) {
    // prefetch window of the one-column stored M2L (FP64 blocks when stored:
    // the FP64 path's kernel; else the fixed-point copy)
    float best = 1e30f;
    uint32_t arg = p.tune.pf_fp64;
    for (uint32_t w : windows) {
      p.tune.pf_fp64 = w;
      const float ms = time_ms(s, reps, [&] { m2l_apply_stored(p, p.levels, !fp64b, s); });
      if (ms < best) {
        best = ms;
        arg = w;
      }
    }
    p.tune.pf_fp64 = arg;
    // prefetch window of the batched stored-block M2L (mixed: fixed point)
    best = 1e30f;
    arg = p.tune.pf_batched;
    const uint32_t keep = p.tune.otf_batched;
    p.tune.otf_batched = 0;
    for (uint32_t w : windows) {
      p.tune.pf_batched = w;
      const float ms = time_ms(s, reps, [&] { m2l_batched(p, h->batch, R, 0, s); });
      if (ms < best) {
        best = ms;
        arg = w;
      }
    }
    p.tune.pf_batched = arg;
    p.tune.otf_batched = keep;
  }
  if ((what & 2) && nlev > 0 && (fp64b || q32)) {
    // per level: stored blocks or entries on the fly, one column and batched
    uint32_t om = 0, ob = 0;
    for (int t = 0; t < nlev; ++t) {
      const LevelSet one = level_subset(p.levels, 1u << t, true);
      if (one.row0[one.nlev] == 0) continue;
      const float st_ms = time_ms(s, reps, [&] { m2l_apply_stored(p, one, q32, s); });
      const float of_ms = time_ms(s, reps, [&] { m2l_apply_otf(p, one, s); });
      if (of_ms < 0.97f * st_ms) om |= 1u << t;
      MatvecPlan pc = p;
      pc.levels = one;
      pc.levels_m2l = one;  // (unsharded views while tuning)
      pc.tune.otf_batched = 0;
      const float sb = time_ms(s, reps, [&] { m2l_batched(pc, h->batch, R, 0, s); });
      pc.tune.otf_batched = 0xffffffffu;
      const float fb = time_ms(s, reps, [&] { m2l_batched(pc, h->batch, R, 0, s); });
      if (fb < 0.97f * sb) ob |= 1u << t;
    }
    // the masks as a whole against all stored: per-level timings miss how
    // the levels share the GPU inside one launch, so keep a mask only when
    // the combined launch confirms it
    if (om) {
      const LevelSet st = level_subset(p.levels, om, false), fly = level_subset(p.levels, om, true);
      const float mask_ms = time_ms(s, reps, [&] {
        m2l_apply_stored(p, st, q32, s);
        m2l_apply_otf(p, fly, s);
      });
      const float all_ms = time_ms(s, reps, [&] { m2l_apply_stored(p, p.levels, q32, s); });
      if (!(mask_ms < 0.97f * all_ms)) om = 0;
    }
    if (ob) {
      p.tune.otf_batched = ob;
      const float mask_ms = time_ms(s, reps, [&] { m2l_batched(p, h->batch, R, 0, s); });
      p.tune.otf_batched = 0;
      const float all_ms = time_ms(s, reps, [&] { m2l_batched(p, h->batch, R, 0, s); });
      if (!(mask_ms < 0.97f * all_ms)) ob = 0;
    }
    p.tune.otf_mixed = om;
    p.tune.otf_batched = ob;
  }
  if ((what & 8) && nlev > 0 && (fp64b || q32)) {
    // form of the 16-column stored M2L (the levels kept stored): FP64 tiles
    // 8x8x4 or transposed m16n8k4, or exact integer products on tcgen05 from
    // the byte planes (m2l_tc = 2).  The tcgen05 TF32 form (m2l_tc = 1) is not
    // a candidate: its FP32 far field leaves the mixed tolerance on deep
    // trees, so it stays an explicit choice.
    float best = 1e30f;
    int arg = p.tune.m2l_t16, arg_tc = p.tune.m2l_tc == 1 ? 0 : p.tune.m2l_tc;
    for (int form = 0; form < (h->m2l_s_stored ? 3 : 2); ++form) {
      p.tune.m2l_t16 = form == 1;
      p.tune.m2l_tc = form == 2 ? 2 : 0;
      const float ms = time_ms(s, reps, [&] { m2l_batched(p, h->batch, R, 0, s); });
      if (ms < best) {
        best = ms;
        arg = p.tune.m2l_t16;
        arg_tc = p.tune.m2l_tc;
      }
    }
    p.tune.m2l_t16 = arg;
    p.tune.m2l_tc = arg_tc;
    check_device_flag(h);
  }
  if ((what & 16) && p.near.nmax <= 64) {
    // near field of 16-column mixed passes: tcgen05 or mma.sync tiles
    float best = 1e30f;
    int arg = p.tune.p2p_tc;
    for (int tc : {0, 1}) {
      p.tune.p2p_tc = tc;
      const float ms = time_ms(s, reps, [&] { p2p_batched(p, h->mixed, h->batch, R, 0, s); });
      if (ms < best) {
        best = ms;
        arg = tc;
      }
    }
    p.tune.p2p_tc = arg;
    check_device_flag(h);
  }
  if (what & 4) {
    // pass width of host-pointer batched calls: 16 columns as one pass or as
    // two overlapped passes of 8 (pinned staging for the timing only)
    double* hq = nullptr;
    double* hy = nullptr;
    AFMM_CUDA(cudaMallocHost(&hq, sizeof(double) * (size_t)N * R));
    device_alloc_counter().fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaMallocHost(&hy, sizeof(double) * (size_t)N * R);
    if (e != cudaSuccess) {
      cudaFreeHost(hq);
      AFMM_CUDA(e);
    }
    try {
      AFMM_CUDA(cudaMemcpy(hq, dq, sizeof(double) * (size_t)N * R, cudaMemcpyDeviceToHost));
      float best = 1e30f;
      int arg = 0;
      for (int W : {8, 16}) {
        p.tune.host_pass_cols = W;
        const float ms = time_ms(s, 3, [&] {
          host_pipeline(h, hq, hy, R, N, W, [&](const double* qd, double* yd, int nc) {
            matvec_batched(p, h->mixed, h->batch, qd, N, yd, N, nc, 0, s, nullptr, &launches);
          });
        });
        if (ms < best) {
          best = ms;
          arg = W;
        }
      }
      p.tune.host_pass_cols = arg;
    } catch (...) {
      cudaFreeHost(hq);
      cudaFreeHost(hy);
      throw;
    }
    cudaFreeHost(hq);
    cudaFreeHost(hy);
  }
  AFMM_CUDA(cudaStreamSynchronize(s));
  h->launches += launches;
}

}  // namespace

extern "C" {

afmm_status afmm_create(int N, int min_particles_in_leaf, int tol_pow, const double* loc, int loc_layout,
                        int kernel_id, const double* kparams, int nkparams, afmm_handle** out) {
  if (!out) {
    g_err = "out is NULL";
    return AFMM_BAD_ARG;
  }
  *out = nullptr;
  afmm_handle* h = nullptr;
  afmm_status st = guard(nullptr, [&] {
    if (N < 1 || min_particles_in_leaf < 1) throw Error{AFMM_BAD_ARG, "N and MinParticlesInLeaf must be >= 1"};
    if (!loc) throw Error{AFMM_BAD_ARG, "loc is NULL"};
    if (loc_layout != AFMM_LOC_COLMAJOR && loc_layout != AFMM_LOC_INTERLEAVED) throw Error{AFMM_BAD_ARG, "bad loc_layout"};
    if (!kernel_known(kernel_id)) throw Error{AFMM_BAD_ARG, "unknown kernel_id " + std::to_string(kernel_id)};
    int L = n_levels(N, min_particles_in_leaf);
    if (L < 2)
      throw Error{AFMM_BAD_ARG, "N/MinParticlesInLeaf gives nLevels = " + std::to_string(L) + " < 2"};
    if (L >= kMaxLevels) throw Error{AFMM_BAD_ARG, "too many levels"};
    double param = (kparams && nkparams > 0) ? kparams[0] : 0.01;
    if (kernel_id == AFMM_KERNEL_GAUSSIAN && !(param > 0)) throw Error{AFMM_BAD_ARG, "Gaussian parameter must be > 0"};
    h = new afmm_handle();
    h->N = N;
    h->M = min_particles_in_leaf;
    h->tol_pow = tol_pow;
    h->L = L;
    h->kernel_id = kernel_id;
    // a = boxRadius[L], halving from 1 (src/AFMM2DTree.cpp:14-19)
    double a = 1.0;
    for (int j = 0; j < L; ++j) a *= 0.5;
    h->kp = make_kernel_params(kernel_id, a, param);
    double t0 = now_s();
    do_create(h, loc, loc_layout);
    h->t_create = now_s() - t0;
  });
  if (st != AFMM_OK) {
    delete h;
    return st;
  }
  *out = h;
  return AFMM_OK;
}

afmm_status afmm_save(afmm_handle* h, const char* path) {
  if (!h || !path) return AFMM_BAD_ARG;
  return guard(h, [&] { do_save(h, path); });
}

afmm_status afmm_load(const char* path, afmm_handle** out) {
  if (!out || !path) {
    g_err = "path and out must not be NULL";
    return AFMM_BAD_ARG;
  }
  *out = nullptr;
  afmm_handle* h = nullptr;
  afmm_status st = guard(nullptr, [&] {
    const double t0 = now_s();
    SetupImage im = read_setup(path);
    check_device();
    h = new afmm_handle();
    h->N = im.N;
    h->M = im.M;
    h->tol_pow = im.tol_pow;
    h->L = im.L;
    h->kernel_id = im.kernel_id;
    h->m2l_mode = im.m2l_mode;
    h->m2l_q_mode = im.q_mode;
    h->kp = make_kernel_params(im.kernel_id, im.a, im.param);
    create_streams(h);
    h->d_pts = h->arena.alloc<double2>(im.N);
    h->d_perm = h->arena.alloc<int64_t>(im.N);
    AFMM_CUDA(cudaMemcpyAsync(h->d_pts, im.pts.data(), sizeof(double) * im.pts.size(), cudaMemcpyHostToDevice, h->stream));
    AFMM_CUDA(cudaMemcpyAsync(h->d_perm, im.perm.data(), sizeof(int64_t) * im.N, cudaMemcpyHostToDevice, h->stream));
    create_layout(h);
    const double t1 = now_s();
    h->t_create = t1 - t0;
    load_levels(h, im);
    finish_assemble(h);
    h->t_assemble = now_s() - t1;
  });
  if (st != AFMM_OK) {
    delete h;
    return st;
  }
  *out = h;
  return AFMM_OK;
}

afmm_status afmm_assemble(afmm_handle* h) {
  if (!h) return AFMM_BAD_ARG;
  return guard(h, [&] {
    if (h->assembled) return;
    double t0 = now_s();
    do_assemble(h);
    h->t_assemble = now_s() - t0;
  });
}

afmm_status afmm_matvec(afmm_handle* h, const double* q, double* y, int nrhs, int64_t ld, int precision,
                        int mem_device) {
  if (!h) return AFMM_BAD_ARG;
  return guard(h, [&] {
    if (!h->assembled) throw Error{AFMM_NOT_ASSEMBLED, "afmm_matvec before afmm_assemble"};
    if (!q || !y || nrhs < 1 || ld < h->N) throw Error{AFMM_BAD_ARG, "bad q/y/nrhs/ld"};
    if (precision != AFMM_PREC_FP64 && precision != AFMM_PREC_MIXED && precision != AFMM_PREC_FP64_BATCHED)
      throw Error{AFMM_BAD_ARG, "bad precision"};
    cudaStream_t s = h->stream;
    if (h->profiling) h->timer.reset();
    StageTimer* tm = h->profiling ? &h->timer : nullptr;
    if (precision != AFMM_PREC_FP64) {
      mixed_reserve(h->mixed, h->N, 1, h->arena);
      if (nrhs > 1) batch_reserve(h->plan, h->batch, h->arena, s);
    }
    // nc columns (leading dimensions ldq, ldy) on the handle's stream.  A
    // one-column call in FP64 batched mode is the plain FP64 apply, and in
    // mixed mode the single-RHS path; every pass of a multi-column call takes
    // the batched passes, so that host and device calls give the same bits
    auto compute = [&](const double* qq, int64_t ldq, double* yy, int64_t ldy, int nc) {
      if (precision == AFMM_PREC_FP64 || (precision == AFMM_PREC_FP64_BATCHED && nrhs == 1)) {
        for (int c = 0; c < nc; ++c)
          matvec_fp64(h->plan, qq + (size_t)c * ldq, yy + (size_t)c * ldy, s, tm, &h->launches);
        h->have_last = true;
      } else if (nrhs > 1) {
        matvec_batched(h->plan, h->mixed, h->batch, qq, ldq, yy, ldy, nc, precision == AFMM_PREC_FP64_BATCHED, s, tm,
                       &h->launches);
      } else {
        matvec_mixed(h->plan, h->mixed, qq, ldq, yy, ldy, 1, s, tm, &h->launches);
      }
    };
    if (mem_device) {
      compute(q, ld, y, ld, nrhs);
    } else {
      // pass width: one column for the column-by-column FP64 apply; for the
      // batched modes at most 8 columns, so that 16 columns make two passes
      // whose copies overlap each other's computation
      int W = 1;
      if (precision != AFMM_PREC_FP64)
        W = h->plan.tune.host_pass_cols > 0 ? std::min(nrhs, h->plan.tune.host_pass_cols) : std::min(nrhs, 8);
      host_pipeline(h, q, y, nrhs, ld, W,
                    [&](const double* qd, double* yd, int nc) { compute(qd, h->N, yd, h->N, nc); });
    }
    if (tm) tm->mark(s, "end");
    check_device_flag(h);
    if (tm) tm->collect(h->stage_ms);
  });
}

afmm_status afmm_eval_error(afmm_handle* h, int nsample, uint64_t seed, double* rel_err) {
  if (!h || !rel_err) return AFMM_BAD_ARG;
  return guard(h, [&] {
    if (!h->have_last) throw Error{AFMM_BAD_ARG, "no FP64 matvec has been computed yet"};
    if (h->plan.shard_count > 1) throw Error{AFMM_BAD_ARG, "afmm_eval_error on a sharded handle (its output is partial)"};
    const long nleaf = h->lv[h->L].nbox;
    std::vector<long> leaves;
    if (nsample <= 0 || nsample >= nleaf) {
      for (long k = 0; k < nleaf; ++k) leaves.push_back(k);
    } else {
      std::vector<char> used(nleaf, 0);
      uint64_t st = seed;
      while ((int)leaves.size() < nsample) {
        long k = (long)(splitmix(st) % (uint64_t)nleaf);
        if (!used[k]) {
          used[k] = 1;
          leaves.push_back(k);
        }
      }
    }
    std::vector<int32_t> rows;
    for (long k : leaves)
      for (int i = 0; i < h->h_leaf_cnt[k]; ++i) rows.push_back(h->h_leaf_start[k] + i);
    DevArena tmp;
    int32_t* d_rows = tmp.alloc<int32_t>(rows.size());
    double* d_out = tmp.alloc<double>(rows.size());
    cudaStream_t s = h->stream;
    AFMM_CUDA(cudaMemcpyAsync(d_rows, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice, s));
    kernel_table(h->kp.id).dense_rows(h->d_pts, h->d_qs, h->N, d_rows, (int)rows.size(), h->kp, d_out, s);
    ++h->launches;
    std::vector<double> dense(rows.size()), ys(h->N);
    AFMM_CUDA(cudaMemcpyAsync(dense.data(), d_out, sizeof(double) * rows.size(), cudaMemcpyDeviceToHost, s));
    AFMM_CUDA(cudaMemcpyAsync(ys.data(), h->d_ys, sizeof(double) * h->N, cudaMemcpyDeviceToHost, s));
    AFMM_CUDA(cudaStreamSynchronize(s));
    double num = 0, den = 0;
    for (size_t t = 0; t < rows.size(); ++t) {
      double d = ys[rows[t]] - dense[t];
      num += d * d;
      den += dense[t] * dense[t];
    }
    *rel_err = den > 0 ? std::sqrt(num / den) : std::sqrt(num);
  });
}

afmm_status afmm_get_permutation(afmm_handle* h, int64_t* perm) {
  if (!h || !perm) return AFMM_BAD_ARG;
  return guard(h, [&] { AFMM_CUDA(cudaMemcpy(perm, h->d_perm, sizeof(int64_t) * h->N, cudaMemcpyDeviceToHost)); });
}

afmm_status afmm_get_sorted_locations(afmm_handle* h, double* xy) {
  if (!h || !xy) return AFMM_BAD_ARG;
  return guard(h, [&] { AFMM_CUDA(cudaMemcpy(xy, h->d_pts, sizeof(double) * 2 * h->N, cudaMemcpyDeviceToHost)); });
}

afmm_status afmm_get_params(afmm_handle* h, int* i5, double* kparam) {
  if (!h || !i5) return AFMM_BAD_ARG;
  i5[0] = h->N;
  i5[1] = h->M;
  i5[2] = h->tol_pow;
  i5[3] = h->L;
  i5[4] = h->kernel_id;
  if (kparam) *kparam = h->kp.param;
  return AFMM_OK;
}

afmm_status afmm_get_nlevels(afmm_handle* h, int* nlevels) {
  if (!h || !nlevels) return AFMM_BAD_ARG;
  *nlevels = h->L;
  return AFMM_OK;
}

afmm_status afmm_get_leaves(afmm_handle* h, int32_t* counts, int32_t* box_numbers) {
  if (!h || !counts || !box_numbers) return AFMM_BAD_ARG;
  std::copy(h->h_counts.begin(), h->h_counts.end(), counts);
  std::copy(h->h_boxnum.begin(), h->h_boxnum.end(), box_numbers);
  return AFMM_OK;
}

afmm_status afmm_get_lists(afmm_handle* h, int level, int32_t* nbr, int32_t* inner, int32_t* outer) {
  if (!h || level < 0 || level > h->L || !nbr || !inner || !outer) return AFMM_BAD_ARG;
  return guard(h, [&] {
    const LevelDev& v = h->lv[level];
    AFMM_CUDA(cudaMemcpy(nbr, v.nbr, sizeof(int32_t) * v.nbox * 8, cudaMemcpyDeviceToHost));
    const std::vector<int32_t>& il = h->h_il[level];
    for (long b = 0; b < v.nbox; ++b) {
      std::copy(il.begin() + b * 40, il.begin() + b * 40 + 16, inner + b * 16);
      std::copy(il.begin() + b * 40 + 16, il.begin() + b * 40 + 40, outer + b * 24);
    }
  });
}

afmm_status afmm_get_ranks(afmm_handle* h, int level, int32_t* ranks) {
  if (!h || !ranks || level < 2 || level > h->L) return AFMM_BAD_ARG;
  if (!h->assembled) return AFMM_NOT_ASSEMBLED;
  std::copy(h->lv[level].h_rank.begin(), h->lv[level].h_rank.end(), ranks);
  return AFMM_OK;
}

static afmm_status get_ids(afmm_handle* h, int level, int32_t* ids, int64_t* count, bool skel) {
  if (!h || !count || level < 2 || level > h->L) return AFMM_BAD_ARG;
  if (!h->assembled) return AFMM_NOT_ASSEMBLED;
  return guard(h, [&] {
    const LevelDev& v = h->lv[level];
    *count = v.total_rank;
    if (ids && v.total_rank > 0)
      AFMM_CUDA(cudaMemcpy(ids, skel ? v.skel_ids : v.cpiv_ids, sizeof(int32_t) * v.total_rank, cudaMemcpyDeviceToHost));
  });
}

afmm_status afmm_get_skeletons(afmm_handle* h, int level, int32_t* ids, int64_t* count) {
  return get_ids(h, level, ids, count, true);
}

afmm_status afmm_get_charge_points(afmm_handle* h, int level, int32_t* ids, int64_t* count) {
  return get_ids(h, level, ids, count, false);
}

afmm_status afmm_get_l2p(afmm_handle* h, int level, int k, int32_t* rows, int32_t* cols, double* out) {
  if (!h || !rows || !cols || level < 2 || level > h->L || k < 0 || k >= h->lv[level].nbox) return AFMM_BAD_ARG;
  if (!h->assembled) return AFMM_NOT_ASSEMBLED;
  return guard(h, [&] {
    const LevelDev& v = h->lv[level];
    int r = v.h_rank[k];
    int n = v.h_node_off[k + 1] - v.h_node_off[k];
    *rows = r ? n : 0;
    *cols = r;
    if (out && r) {
      std::vector<double> cm((size_t)n * r);
      AFMM_CUDA(cudaMemcpy(cm.data(), v.l2p + v.h_l2p_off[k], sizeof(double) * cm.size(), cudaMemcpyDeviceToHost));
      for (int i = 0; i < n; ++i)
        for (int c = 0; c < r; ++c) out[(size_t)i * r + c] = cm[(size_t)c * n + i];
    }
  });
}

afmm_status afmm_set_m2l_storage(afmm_handle* h, int mode) {
  if (!h) return AFMM_BAD_ARG;
  if (mode != AFMM_M2L_AUTO && mode != AFMM_M2L_STORE && mode != AFMM_M2L_ON_THE_FLY) {
    h->err = "bad M2L storage mode";
    return AFMM_BAD_ARG;
  }
  if (h->assembled) {
    h->err = "afmm_set_m2l_storage after afmm_assemble";
    return AFMM_BAD_ARG;
  }
  h->m2l_mode = mode;
  return AFMM_OK;
}

afmm_status afmm_set_aca_plan(afmm_handle* h, int cluster, int ctas_per_sm) {
  if (!h) return AFMM_BAD_ARG;
  if (h->assembled || cluster < 0 || cluster > 16 || (cluster & (cluster - 1)) || ctas_per_sm < 0 || ctas_per_sm > 2) {
    h->err = "afmm_set_aca_plan: before afmm_assemble; cluster 0 or a power of two <= 16; ctas_per_sm 0, 1 or 2";
    return AFMM_BAD_ARG;
  }
  h->aca_cluster = cluster;
  h->aca_ctas_per_sm = ctas_per_sm;
  return AFMM_OK;
}

afmm_status afmm_set_m2l_fixed_point(afmm_handle* h, int on) {
  if (!h) return AFMM_BAD_ARG;
  if (h->assembled) {
    h->err = "afmm_set_m2l_fixed_point after afmm_assemble";
    return AFMM_BAD_ARG;
  }
  if (on < 0 || on > 2) {
    h->err = "afmm_set_m2l_fixed_point: mode is 0, 1 or 2";
    return AFMM_BAD_ARG;
  }
  h->m2l_q_mode = on;
  return AFMM_OK;
}

afmm_status afmm_shard_range(int nlevels, int index, int count, int* level, int64_t* k0, int64_t* k1) {
  if (!level || !k0 || !k1) return AFMM_BAD_ARG;
  int lev = 0;
  long a = 0, b = 0;
  if (!shard_range(nlevels, index, count, lev, a, b)) {
    g_err = "afmm_shard_range: need 0 <= index < count and at least count leaves";
    return AFMM_BAD_ARG;
  }
  *level = lev;
  *k0 = a;
  *k1 = b;
  return AFMM_OK;
}

afmm_status afmm_set_shard(afmm_handle* h, int index, int count) {
  if (!h) return AFMM_BAD_ARG;
  return guard(h, [&] {
    if (!h->assembled) throw Error{AFMM_NOT_ASSEMBLED, "afmm_set_shard before afmm_assemble"};
    int lev = 0;
    long a = 0, b = 0;
    if (count < 1 || index < 0 || index >= count || (count > 1 && !shard_range(h->L, index, count, lev, a, b)))
      throw Error{AFMM_BAD_ARG, "afmm_set_shard: need 0 <= index < count and at least count leaves"};
    h->shard_index = index;
    h->shard_count = count;
    apply_shard(h);
  });
}

afmm_status afmm_get_shard(afmm_handle* h, int* index, int* count, int* level) {
  if (!h || !index || !count || !level) return AFMM_BAD_ARG;
  *index = h->plan.shard_index;
  *count = h->plan.shard_count;
  *level = h->plan.shard_level;
  return AFMM_OK;
}

afmm_status afmm_get_m2l_fixed_point(afmm_handle* h, int* stored) {
  if (!h || !stored) return AFMM_BAD_ARG;
  *stored = h->m2l_q_stored ? 1 : 0;
  return AFMM_OK;
}

afmm_status afmm_get_m2l_stored(afmm_handle* h, int* stored) {
  if (!h || !stored) return AFMM_BAD_ARG;
  *stored = h->m2l_stored ? 1 : 0;
  return AFMM_OK;
}

afmm_status afmm_set_profiling(afmm_handle* h, int on) {
  if (!h || on < 0 || on > 2) return AFMM_BAD_ARG;
  h->profiling = on != 0;
  h->timer.serial = on == 2;
  return AFMM_OK;
}

afmm_status afmm_get_stage_times(afmm_handle* h, int cap, const char** names, double* ms, int* n) {
  if (!h || !n) return AFMM_BAD_ARG;
  *n = (int)h->stage_ms.size();
  for (int i = 0; i < *n && i < cap; ++i) {
    if (names) names[i] = h->stage_ms[i].first.c_str();
    if (ms) ms[i] = h->stage_ms[i].second;
  }
  return AFMM_OK;
}

afmm_status afmm_get_setup_times(afmm_handle* h, double* t2) {
  if (!h || !t2) return AFMM_BAD_ARG;
  t2[0] = h->t_create;
  t2[1] = h->t_assemble;
  return AFMM_OK;
}

afmm_status afmm_get_setup_phases(afmm_handle* h, int cap, const char** names, double* secs, int* n) {
  if (!h || !n) return AFMM_BAD_ARG;
  *n = (int)h->setup_phase.size();
  for (int i = 0; i < *n && i < cap; ++i) {
    if (names) names[i] = h->setup_phase[i].first.c_str();
    if (secs) secs[i] = h->setup_phase[i].second;
  }
  return AFMM_OK;
}

afmm_status afmm_get_counts(afmm_handle* h, int64_t* c7) {
  if (!h || !c7) return AFMM_BAD_ARG;
  std::copy(h->counts, h->counts + 7, c7);
  return AFMM_OK;
}

afmm_status afmm_get_launch_count(afmm_handle* h, int64_t* n) {
  if (!h || !n) return AFMM_BAD_ARG;
  *n = h->launches;
  return AFMM_OK;
}

afmm_status afmm_get_stream(afmm_handle* h, void** stream) {
  if (!h || !stream) return AFMM_BAD_ARG;
  *stream = (void*)h->stream;
  return AFMM_OK;
}

afmm_status afmm_kernel_eval(int kernel_id, double a, double param, int64_t n, const double* xy1, const double* xy2,
                             double* out, int mode) {
  if (!xy1 || !xy2 || !out || n < 0 || mode < 0 || mode > 2 || !kernel_known(kernel_id)) return AFMM_BAD_ARG;
  if (n == 0) return AFMM_OK;
  return guard(nullptr, [&] {
    check_device();
    DevArena tmp;
    double2* da = tmp.alloc<double2>(n);
    double2* db = tmp.alloc<double2>(n);
    double* dout = tmp.alloc<double>(n);
    AFMM_CUDA(cudaMemcpy(da, xy1, sizeof(double2) * n, cudaMemcpyHostToDevice));
    AFMM_CUDA(cudaMemcpy(db, xy2, sizeof(double2) * n, cudaMemcpyHostToDevice));
    kernel_table(kernel_id).kernel_pairs(da, db, (long)n, make_kernel_params(kernel_id, a, param), mode, dout);
    AFMM_CUDA(cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost));
  });
}

afmm_status afmm_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops) return AFMM_BAD_ARG;
  return guard(nullptr, [&] {
    check_device();
    *fp64_tflops = fma_peak_tflops<double>();
    *fp32_tflops = fma_peak_tflops<float>();
  });
}

afmm_status afmm_measure_fp64_pipes(double* dmma_tflops, double* dfma_tflops, double* both_tflops) {
  if (!dmma_tflops || !dfma_tflops || !both_tflops) return AFMM_BAD_ARG;
  return guard(nullptr, [&] {
    check_device();
    *dmma_tflops = fp64_pipes_tflops<0>().first;
    *dfma_tflops = fp64_pipes_tflops<1>().second;
    const auto b = fp64_pipes_tflops<2>();
    *both_tflops = b.first + b.second;
  });
}

afmm_status afmm_kd_permutation_noalloc(int N, int min_particles_in_leaf, const double* xy, int64_t* perm,
                                        double* xy_sorted, void* stream) {
  if (!xy || !perm) {
    g_err = "xy and perm must be device pointers";
    return AFMM_BAD_ARG;
  }
  return guard(nullptr, [&] {
    int L = n_levels(N, min_particles_in_leaf);
    if (L < 2) throw Error{AFMM_BAD_ARG, "N/MinParticlesInLeaf gives nLevels = " + std::to_string(L) + " < 2"};
    check_device();
    kd_sort_noalloc(xy, N, L, perm, xy_sorted, (cudaStream_t)stream);
  });
}

afmm_status afmm_register_kernel(int kernel_id, const void* table, size_t table_bytes, int abi_version) {
  if (kernel_id < AFMM_KERNEL_USER_FIRST || kernel_id >= AFMM_KERNEL_USER_FIRST + AFMM_KERNEL_USER_COUNT) {
    g_err = "user kernel ids are " + std::to_string(AFMM_KERNEL_USER_FIRST) + " .. " +
            std::to_string(AFMM_KERNEL_USER_FIRST + AFMM_KERNEL_USER_COUNT - 1);
    return AFMM_BAD_ARG;
  }
  if (!table || table_bytes != sizeof(KernelTable) || abi_version != kKernelTableAbi ||
      ((const KernelTable*)table)->abi != kKernelTableAbi || ((const KernelTable*)table)->layout != kArgLayout) {
    g_err = "kernel table built against other library headers (size, ABI version or argument layouts differ)";
    return AFMM_BAD_ARG;
  }
  std::lock_guard<std::mutex> lock(g_kernel_mu);
  const KernelTable*& slot = g_user_kernels[kernel_id - AFMM_KERNEL_USER_FIRST];
  if (slot && slot != table) {
    g_err = "kernel id " + std::to_string(kernel_id) + " is already registered";
    return AFMM_BAD_ARG;
  }
  slot = (const KernelTable*)table;
  return AFMM_OK;
}

afmm_status afmm_kernel_name(int kernel_id, const char** name) {
  if (!name) return AFMM_BAD_ARG;
  return guard(nullptr, [&] { *name = kernel_table(kernel_id).name; });
}

afmm_status afmm_autotune(afmm_handle* h, int what, const char* cache_path, int* from_cache) {
  if (!h) return AFMM_BAD_ARG;
  return guard(h, [&] {
    if (!h->assembled) throw Error{AFMM_NOT_ASSEMBLED, "afmm_autotune before afmm_assemble"};
    if (what < 0 || what > 31)
      throw Error{AFMM_BAD_ARG,
                  "what: bit 0 windows, bit 1 M2L forms, bit 2 host passes, bit 3 M2L tile shape, bit 4 near field"};
    const std::string key = tuning_key(h);
    Tuning t;
    if (cache_lookup(cache_path, key, t)) {
      h->plan.tune = t;
      if (from_cache) *from_cache = 1;
      return;
    }
    if (from_cache) *from_cache = 0;
    do_autotune(h, what == 0 ? 31 : what);
    cache_store(cache_path, key, h->plan.tune);
  });
}

afmm_status afmm_get_tuning(afmm_handle* h, int64_t* v, int n) {
  if (!h || !v || n < kTuningValuesMin) return AFMM_BAD_ARG;
  int64_t w[kTuningValues];
  tuning_to(h->plan.tune, w);
  std::copy(w, w + std::min(n, kTuningValues), v);
  return AFMM_OK;
}

afmm_status afmm_set_tuning(afmm_handle* h, const int64_t* v, int n) {
  if (!h || !v || n < kTuningValuesMin) return AFMM_BAD_ARG;
  return guard(h, [&] {
    int64_t w[kTuningValues];
    tuning_to(h->plan.tune, w);  // values the caller does not pass stay as they are
    std::copy(v, v + std::min(n, kTuningValues), w);
    h->plan.tune = tuning_from(w);
  });
}

afmm_status afmm_get_device_alloc_count(int64_t* n) {
  if (!n) return AFMM_BAD_ARG;
  *n = device_alloc_counter().load();
  return AFMM_OK;
}

afmm_status afmm_destroy(afmm_handle* h) {
  if (!h) return AFMM_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaStream_t s = h->stream;
  delete h;
  if (s) cudaStreamDestroy(s);
  return AFMM_OK;
}

afmm_status afmm_set_create(afmm_handle* const* handles, int n, afmm_set** out) {
  if (!out) return AFMM_BAD_ARG;
  *out = nullptr;
  afmm_set* st = nullptr;
  afmm_status rc = guard(nullptr, [&] {
    check_device();
    if (!handles || n < 1) throw Error{AFMM_BAD_ARG, "afmm_set_create: need n >= 1 handles"};
    std::vector<SetProblem> probs;
    int dev = -1;
    AFMM_CUDA(cudaGetDevice(&dev));
    for (int p = 0; p < n; ++p) {
      afmm_handle* h = handles[p];
      if (!h) throw Error{AFMM_BAD_ARG, "afmm_set_create: null handle"};
      if (!h->assembled) throw Error{AFMM_NOT_ASSEMBLED, "afmm_set_create: handle not assembled"};
      if (h->kernel_id != handles[0]->kernel_id) throw Error{AFMM_BAD_ARG, "afmm_set_create: mixed kernel ids"};
      if (!h->m2l_stored) throw Error{AFMM_BAD_ARG, "afmm_set_create: a handle has no stored M2L blocks"};
      if (h->shard_count > 1) throw Error{AFMM_BAD_ARG, "afmm_set_create: a handle is sharded"};
      if (h->device != dev) throw Error{AFMM_BAD_ARG, "afmm_set_create: handle on another device"};
      probs.push_back({&h->plan, p2p_shape(h->plan.near.nmax)});
    }
    st = new afmm_set();
    AFMM_CUDA(cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking));
    for (int p = 0; p < n; ++p) AFMM_CUDA(cudaStreamSynchronize(handles[p]->stream));
    st->plan.kernel_id = handles[0]->kernel_id;
    set_build(st->plan, probs, st->arena, st->stream);
    st->offsets.resize(n + 1, 0);
    for (int p = 0; p < n; ++p) st->offsets[p + 1] = st->offsets[p] + handles[p]->N;
  });
  if (rc != AFMM_OK) {
    if (st) afmm_set_destroy(st);
    return rc;
  }
  *out = st;
  return AFMM_OK;
}

afmm_status afmm_set_matvec(afmm_set* st, const double* q, double* y, int mem_device) {
  if (!st) return AFMM_BAD_ARG;
  try {
    if (!q || !y) throw Error{AFMM_BAD_ARG, "afmm_set_matvec: null q/y"};
    cudaStream_t s = st->stream;
    const size_t bytes = sizeof(double) * (size_t)st->plan.total_points;
    AFMM_CUDA(cudaMemcpyAsync(st->plan.q, q, bytes, mem_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    set_matvec(st->plan, s);
    ++st->graph_launches;
    AFMM_CUDA(cudaMemcpyAsync(y, st->plan.y, bytes, mem_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    AFMM_CUDA(cudaStreamSynchronize(s));
    if (*st->plan.h_err)
      throw Error{AFMM_TIMEOUT, "afmm_set_matvec: a sweep's wait for the level below gave up (output incomplete)"};
    return AFMM_OK;
  } catch (const Error& e) {
    st->err = e.msg;
    return e.status;
  }
}

afmm_status afmm_set_get_offsets(afmm_set* st, int64_t* offsets) {
  if (!st || !offsets) return AFMM_BAD_ARG;
  std::copy(st->offsets.begin(), st->offsets.end(), offsets);
  return AFMM_OK;
}

afmm_status afmm_set_get_launches(afmm_set* st, int* per_matvec, int64_t* graph_launches) {
  if (!st) return AFMM_BAD_ARG;
  if (per_matvec) *per_matvec = st->plan.launches_per_matvec;
  if (graph_launches) *graph_launches = st->graph_launches;
  return AFMM_OK;
}

afmm_status afmm_set_get_stage_times(afmm_set* st, int cap, const char** names, double* ms, int* n) {
  if (!st || !n) return AFMM_BAD_ARG;
  try {
    if (st->stream) AFMM_CUDA(cudaStreamSynchronize(st->stream));
    if (st->graph_launches == 0) throw Error{AFMM_BAD_ARG, "afmm_set_get_stage_times before afmm_set_matvec"};
    set_stage_times(st->plan, st->stage_ms);
    *n = (int)st->stage_ms.size();
    for (int i = 0; i < *n && i < cap; ++i) {
      if (names) names[i] = st->stage_ms[i].first.c_str();
      if (ms) ms[i] = st->stage_ms[i].second;
    }
    return AFMM_OK;
  } catch (const Error& e) {
    st->err = e.msg;
    return e.status;
  }
}

afmm_status afmm_set_get_stream(afmm_set* st, void** stream) {
  if (!st || !stream) return AFMM_BAD_ARG;
  *stream = (void*)st->stream;
  return AFMM_OK;
}

afmm_status afmm_set_sweep_wait_margin(afmm_set* st, int margin) {
  if (!st) return AFMM_BAD_ARG;
  try {
    if (margin < 0) throw Error{AFMM_BAD_ARG, "afmm_set_sweep_wait_margin: margin >= 0"};
    AFMM_CUDA(cudaStreamSynchronize(st->stream));
    st->plan.up.margin = margin;
    st->plan.down.margin = margin;
    set_recapture(st->plan, st->stream);
    return AFMM_OK;
  } catch (const Error& e) {
    st->err = e.msg;
    return e.status;
  }
}

afmm_status afmm_set_destroy(afmm_set* st) {
  if (!st) return AFMM_OK;
  if (st->stream) cudaStreamSynchronize(st->stream);
  set_release(st->plan);
  cudaStream_t s = st->stream;
  delete st;
  if (s) cudaStreamDestroy(s);
  return AFMM_OK;
}

const char* afmm_set_last_error(afmm_set* st) { return st ? st->err.c_str() : g_err.c_str(); }

const char* afmm_status_string(afmm_status s) {
  switch (s) {
    case AFMM_OK: return "ok";
    case AFMM_BAD_ARG: return "bad argument";
    case AFMM_OOM: return "out of device memory";
    case AFMM_CUDA_ERR: return "CUDA error";
    case AFMM_TIMEOUT: return "device wait timed out";
    case AFMM_NUMERIC: return "non-finite values";
    case AFMM_NOT_ASSEMBLED: return "not assembled";
    case AFMM_NO_DEVICE: return "no sm_100 device";
  }
  return "unknown status";
}

const char* afmm_last_error(afmm_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

const char* afmm_version(void) { return "afmm2d-b200 0.1"; }
}
