// K2 (interaction lists), K5 (M2L blocks) and the FP64 matvec sweeps
// K6-K10 (gather, M2M, M2L, L2L, near field, scatter).
#include <algorithm>

#include "afmm_internal.cuh"
#include "fmm.cuh"

namespace afmm {

// ----------------------------------------------------------------- lists
// Closed form of the reference's parent-to-child recurrence
// (src/AFMM2DTree.cpp:65-967).  Box k at level j sits at grid cell (ix, iy)
// whose bits are the base-4 digits of k read as child offsets
// 0:(0,0) 1:(1,0) 2:(1,1) 3:(0,1) (src/AFMM2DTree.cpp:978-986).  Slot s of
// ring m (m = 1 neighbours N0..N7, 2 inner I0..I15, 3 outer O0..O23) is the
// cell at the s-th offset counter-clockwise around the ring starting at
// (-m,-m).  It is set when the cell is inside the domain and, for ring 3,
// when its parent neighbours the box's parent (the recurrence only visits the
// children of the parent's neighbours).
__device__ __forceinline__ void ring_offset(int m, int s, int& dx, int& dy) {
  const int side = 2 * m, seg = s / side, t = s % side;
  if (seg == 0) { dx = -m + t; dy = -m; }
  else if (seg == 1) { dx = m; dy = -m + t; }
  else if (seg == 2) { dx = m - t; dy = m; }
  else { dx = -m; dy = m - t; }
}

__device__ __forceinline__ void cell_of(long k, int j, int& ix, int& iy) {
  int x = 0, y = 0;
  for (int l = j - 1; l >= 0; --l) {
    int d = (int)((k >> (2 * l)) & 3);
    x = 2 * x + (d == 1 || d == 2);
    y = 2 * y + (d >= 2);
  }
  ix = x;
  iy = y;
}

__device__ __forceinline__ long box_of(int ix, int iy, int j) {
  long k = 0;
  for (int l = j - 1; l >= 0; --l) {
    int bx = (ix >> l) & 1, by = (iy >> l) & 1;
    k = 4 * k + (by ? (bx ? 2 : 3) : (bx ? 1 : 0));
  }
  return k;
}

// One thread per (box, slot of the 48 ring slots).
__global__ void k_lists(int j, long nbox, int32_t* nbr, int32_t* il) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbox * 48) return;
  long k = t / 48;
  int s = (int)(t % 48);
  int m = s < 8 ? 1 : (s < 24 ? 2 : 3);
  int ss = s < 8 ? s : (s < 24 ? s - 8 : s - 24);
  int ix, iy, dx, dy;
  cell_of(k, j, ix, iy);
  ring_offset(m, ss, dx, dy);
  const int side = 1 << j;
  int cx = ix + dx, cy = iy + dy;
  bool ok = cx >= 0 && cy >= 0 && cx < side && cy < side;
  if (ok && m == 3) ok = abs((cx >> 1) - (ix >> 1)) <= 1 && abs((cy >> 1) - (iy >> 1)) <= 1;
  int32_t v = ok ? (int32_t)box_of(cx, cy, j) : -1;
  if (m == 1) nbr[k * 8 + ss] = v;
  else il[k * 40 + (s - 8)] = v;  // inner 0..15 then outer 0..23
}

void build_lists(int j, long nbox, int32_t* nbr, int32_t* il, cudaStream_t s) {
  long n = nbox * 48;
  k_lists<<<(int)((n + 255) / 256), 256, 0, s>>>(j, nbox, nbr, il);
  AFMM_LAUNCH_CHECK();
}

// ------------------------------------------------------------ M2L blocks
// M2L[b][c] = K(R_b, R_c) for every valid inner/outer slot of b, in slot
// order (src/AFMM2DTree.cpp:1070-1097), stored column-major r_b x r_c.
template <class K>
__global__ void k_m2l_assemble(LevelView v, KernelParams kp) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  if (r == 0) return;
  double* out = v.m2l + v.m2l_off[b];
  const double2* xb = v.skel_xy + v.skel_off[b];
  long off = 0;
  for (int s = 0; s < 40; ++s) {
    int c = v.il[b * 40 + s];
    if (c < 0) continue;
    const int rc = v.rank[c];
    const double2* xc = v.skel_xy + v.skel_off[c];
    for (int e = threadIdx.x; e < r * rc; e += blockDim.x) {
      int cc = e / r, i = e - cc * r;
      out[off + e] = K::eval_exact(r2_exact(xb[i].x, xb[i].y, xc[cc].x, xc[cc].y), kp);
    }
    off += (long)r * rc;
  }
}

template <class K>
struct M2lAssembleRun {
  static void run(const LevelView& v, const KernelParams& kp, cudaStream_t s) {
    k_m2l_assemble<K><<<(int)v.nbox, 128, 0, s>>>(v, kp);
    AFMM_LAUNCH_CHECK();
  }
};

void m2l_assemble(const LevelView& v, const KernelParams& kp, cudaStream_t s) {
  dispatch_kernel<M2lAssembleRun>(kp.id, v, kp, s);
}

// ---------------------------------------------------------------- sweeps
// qs[i] = q[perm[i]]  (src/AFMM2D.cpp:49-51)
__global__ void k_gather(const double* __restrict__ q, const int64_t* __restrict__ perm, int n, double* qs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) qs[i] = q[perm[i]];
}

// y[perm[i]] = ys[i]  (src/AFMM2D.cpp:61-63)
__global__ void k_scatter(const double* __restrict__ ys, const int64_t* __restrict__ perm, int n, double* y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[perm[i]] = ys[i];
}

// M2M (src/AFMM2DTree.cpp:1129-1154): qhat_b = L2P_b^T src_b.  One CTA per
// box: the rows are split into SW_WARPS contiguous ranges, one per warp, lanes
// run over the outputs c on the row-major copy of L2P (coalesced); the warps'
// partial sums are added in warp order.  src_b = leaf charges, or the
// concatenated outgoing charges of children 0..3.
__global__ void __launch_bounds__(SW_T) k_m2m(LevelView v, const double* __restrict__ src_all, int leaf) {
  extern __shared__ double part[];  // SW_WARPS x r
  const long b = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = v.rank[b];
  if (r == 0) return;
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (leaf ? v.leaf_start[b] : v.node_off[b]);
  const double* P = v.l2p_rm + v.l2p_off[b];  // n x r, row-major
  const int i0 = (int)((long)n * warp / SW_WARPS), i1 = (int)((long)n * (warp + 1) / SW_WARPS);
  for (int c0 = 0; c0 < r; c0 += 32) {
    const int c = c0 + lane;
    if (c < r) {
      double s = 0.0;
#pragma unroll 4
      for (int i = i0; i < i1; ++i) s += P[(long)i * r + c] * src[i];
      part[warp * r + c] = s;
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < r; c += SW_T) {
    double s = 0.0;
    for (int w = 0; w < SW_WARPS; ++w) s += part[w * r + c];
    v.qhat[v.skel_off[b] + c] = s;
  }
}

// Row-major copy of L2P (per box, r fastest) for the M2M sweep.
template <class T>
__global__ void k_l2p_transpose(LevelView v, const T* __restrict__ cm, T* rm) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  if (r == 0) return;
  const int n = v.node_off[b + 1] - v.node_off[b];
  const long o = v.l2p_off[b];
  for (int e = threadIdx.x; e < n * r; e += blockDim.x) {
    int i = e / r, c = e - i * r;
    rm[o + e] = cm[o + (long)c * n + i];
  }
}

void l2p_transpose(const LevelView& v, const double* cm, double* rm, cudaStream_t s) {
  k_l2p_transpose<double><<<(int)v.nbox, 256, 0, s>>>(v, cm, rm);
  AFMM_LAUNCH_CHECK();
}

// M2L (src/AFMM2DTree.cpp:1156-1178) for every level in one launch.  One CTA
// per box (upper levels first, so the large boxes start early): warp w takes
// the box's valid interaction-list slots w, w + SW_WARPS, ... in slot order,
// lanes run over the box's skeleton rows on column-major blocks (coalesced);
// the warps' partial sums are added in warp order.
__global__ void __launch_bounds__(SW_T) k_m2l_apply(LevelSet ls) {
  extern __shared__ double part[];  // SW_WARPS x r
  __shared__ int s_slot[40], s_nvalid;
  __shared__ long s_off[41];
  long gb = blockIdx.x;
  int j = 0;
  while (j < ls.nlev && gb >= ls.lv[j].nbox) gb -= ls.lv[j++].nbox;
  if (j >= ls.nlev) return;
  const LevelView& v = ls.lv[j];
  const long b = gb;
  const int r = v.rank[b];
  if (r == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    int m = 0;
    long off = 0;
    for (int s = 0; s < 40; ++s) {
      int c = v.il[b * 40 + s];
      if (c < 0) continue;
      s_slot[m] = c;
      s_off[m] = off;
      off += (long)r * v.rank[c];
      ++m;
    }
    s_nvalid = m;
  }
  __syncthreads();
  const double* M0 = v.m2l + v.m2l_off[b];
  for (int i0 = 0; i0 < r; i0 += 32) {
    const int i = i0 + lane;
    double acc = 0.0;
    if (i < r)
      for (int t = warp; t < s_nvalid; t += SW_WARPS) {
        const int c = s_slot[t];
        const int rc = v.rank[c];
        const double* qc = v.qhat + v.skel_off[c];
        const double* M = M0 + s_off[t];
#pragma unroll 8
        for (int cc = 0; cc < rc; ++cc) acc += M[(long)cc * r + i] * qc[cc];
      }
    if (i < r) part[warp * r + i] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < r; i += SW_T) {
    double s = 0.0;
    for (int w = 0; w < SW_WARPS; ++w) s += part[w * r + i];
    v.yhat[v.skel_off[b] + i] = s;
  }
}

// L2L (src/AFMM2DTree.cpp:1180-1197): t = L2P_b yhat_b; added to the children's
// incoming potentials, or written as the leaf potential.  One CTA per box,
// threads over rows (column-major L2P: coalesced).
__global__ void __launch_bounds__(SW_T) k_l2l(LevelView v, double* __restrict__ child_yhat, double* __restrict__ ys,
                                              int leaf) {
  const long b = blockIdx.x;
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* P = v.l2p + v.l2p_off[b];
  const double* yb = v.yhat + v.skel_off[b];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double t = 0.0;
#pragma unroll 8
    for (int c = 0; c < r; ++c) t += P[(long)c * n + i] * yb[c];
    if (leaf) ys[v.leaf_start[b] + i] = t;
    else child_yhat[v.node_off[b] + i] += t;
  }
}

// Near field (src/AFMM2DTree.cpp:1199-1213): per leaf, neighbours 0..7 then
// the leaf itself, kernel evaluated on the fly from shared-memory tiles.
template <class K>
__global__ void k_p2p64(NearView nv, KernelParams kp, const double* __restrict__ qs, double* __restrict__ ys) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* sx = (double2*)smem;
  double* sq = (double*)(sx + nv.nmax);
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  const int T = blockDim.x;
  constexpr int MAXT = 4;
  double2 xi[MAXT];
  double pot[MAXT];
  for (int u = 0; u < MAXT; ++u) {
    int i = threadIdx.x + u * T;
    if (i < n) {
      xi[u] = nv.pts[s0 + i];
      pot[u] = ys[s0 + i];
    }
  }
  for (int slot = 0; slot < 9; ++slot) {
    const long c = slot < 8 ? nv.nbr[b * 8 + slot] : b;
    if (c < 0) continue;
    const int nc = nv.leaf_cnt[c];
    const int c0 = nv.leaf_start[c];
    __syncthreads();
    for (int t = threadIdx.x; t < nc; t += T) {
      sx[t] = nv.pts[c0 + t];
      sq[t] = qs[c0 + t];
    }
    __syncthreads();
    for (int u = 0; u < MAXT; ++u) {
      int i = threadIdx.x + u * T;
      if (i < n) {
        double acc = 0.0;
        for (int t = 0; t < nc; ++t) {
          double dx = xi[u].x - sx[t].x, dy = xi[u].y - sx[t].y;
          acc += K::eval(dx * dx + dy * dy, kp) * sq[t];
        }
        pot[u] += acc;
      }
    }
  }
  for (int u = 0; u < MAXT; ++u) {
    int i = threadIdx.x + u * T;
    if (i < n) ys[s0 + i] = pot[u];
  }
}

template <class K>
struct P2p64Run {
  static void run(const NearView& nv, const KernelParams& kp, const double* qs, double* ys, cudaStream_t s) {
    int T = std::min(256, ((nv.nmax + 3) / 4 + 31) / 32 * 32);
    T = std::max(T, 64);
    size_t smem = (size_t)nv.nmax * (sizeof(double2) + sizeof(double));
    if (smem > 48 * 1024) AFMM_CUDA(cudaFuncSetAttribute(k_p2p64<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_p2p64<K><<<(int)nv.nleaf, T, smem, s>>>(nv, kp, qs, ys);
    AFMM_LAUNCH_CHECK();
  }
};

void sweep_m2m(const MatvecPlan& p, const double* qs, cudaStream_t s, int64_t* launches) {
  for (int j = p.L; j >= 2; --j) {
    const LevelView& v = p.lv[j];
    size_t sm = sizeof(double) * SW_WARPS * std::max(p.rmax[j], 1);
    allow_smem(k_m2m, sm);
    k_m2m<<<(int)v.nbox, SW_T, sm, s>>>(v, j == p.L ? qs : p.lv[j + 1].qhat, j == p.L);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

void sweep_l2l(const MatvecPlan& p, double* ys, cudaStream_t s, int64_t* launches) {
  for (int j = 2; j <= p.L; ++j) {
    const LevelView& v = p.lv[j];
    k_l2l<<<(int)v.nbox, sweep_threads(p.n1max[j]), 0, s>>>(v, j < p.L ? p.lv[j + 1].yhat : nullptr, ys, j == p.L);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

void matvec_fp64(const MatvecPlan& p, const double* q, double* y, cudaStream_t s, StageTimer* tm, int64_t* launches) {
  const int N = p.N;
  const int gb = (N + 255) / 256;
  if (tm) tm->mark(s, "gather");
  k_gather<<<gb, 256, 0, s>>>(q, p.perm, N, p.qs);
  AFMM_LAUNCH_CHECK();
  ++*launches;
  if (tm) tm->mark(s, "m2m");
  sweep_m2m(p, p.qs, s, launches);
  if (tm) tm->mark(s, "m2l");
  {
    long boxes = 0;
    int rm = 1;
    for (int j = 0; j < p.levels.nlev; ++j) boxes += p.levels.lv[j].nbox;
    for (int j = 2; j <= p.L; ++j) rm = std::max(rm, p.rmax[j]);
    size_t sm = sizeof(double) * SW_WARPS * rm;
    allow_smem(k_m2l_apply, sm);
    k_m2l_apply<<<(int)boxes, SW_T, sm, s>>>(p.levels);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
  if (tm) tm->mark(s, "l2l");
  sweep_l2l(p, p.ys, s, launches);
  if (tm) tm->mark(s, "p2p");
  dispatch_kernel<P2p64Run>(p.kp.id, p.near, p.kp, p.qs, p.ys, s);
  ++*launches;
  if (tm) tm->mark(s, "scatter");
  k_scatter<<<gb, 256, 0, s>>>(p.ys, p.perm, N, y);
  AFMM_LAUNCH_CHECK();
  ++*launches;
  if (tm) tm->mark(s, "end");
}

}  // namespace afmm
