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

__global__ void k_fill_box_map(const int32_t* __restrict__ off, long nbox, int32_t* map) {
  long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  for (int32_t t = off[b]; t < off[b + 1]; ++t) map[t] = (int32_t)b;
}

__global__ void k_invert_perm(const int64_t* __restrict__ perm, int n, int32_t* iperm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) iperm[perm[i]] = i;
}

void invert_permutation(const int64_t* perm, int n, int32_t* iperm, cudaStream_t s) {
  k_invert_perm<<<(n + 255) / 256, 256, 0, s>>>(perm, n, iperm);
  AFMM_LAUNCH_CHECK();
}

void fill_box_map(const int32_t* off, long nbox, int32_t* map, cudaStream_t s) {
  k_fill_box_map<<<(int)((nbox + 255) / 256), 256, 0, s>>>(off, nbox, map);
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

// M2M (src/AFMM2DTree.cpp:1129-1154): qhat_b = L2P_b^T src_b.  One thread per
// output (skeleton row of the level), summing over the box's node rows on
// the row-major copy of L2P (a warp's consecutive outputs read contiguously).
// src_b = leaf charges, or the concatenated outgoing charges of children 0..3.
__global__ void k_m2m(LevelView v, const double* __restrict__ src_all, int leaf) {
  const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= v.nrows) return;
  const int b = v.skel_box[row];
  const int r = v.rank[b];
  const int c = (int)(row - v.skel_off[b]);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (leaf ? v.leaf_start[b] : v.node_off[b]);
  const double* P = v.l2p_rm + v.l2p_off[b] + c;  // (i, c) at i*r + c
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int i = 0;
  for (; i + 3 < n; i += 4) {
    a0 += P[(long)i * r] * src[i];
    a1 += P[(long)(i + 1) * r] * src[i + 1];
    a2 += P[(long)(i + 2) * r] * src[i + 2];
    a3 += P[(long)(i + 3) * r] * src[i + 3];
  }
  for (; i < n; ++i) a0 += P[(long)i * r] * src[i];
  v.qhat[row] = (a0 + a1) + (a2 + a3);
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

// Level of flat row g of a LevelSet (row0 is its prefix of row counts).
__device__ __forceinline__ int level_of_row(const LevelSet& ls, long g) {
  int j = 0;
  while (j + 1 < ls.nlev && g >= ls.row0[j + 1]) ++j;
  return j;
}

// M2L (src/AFMM2DTree.cpp:1156-1178) for every level in one launch, one thread
// per skeleton row (upper levels first): row i of box b sums, slot by slot in
// the reference's order (inner 0..15, outer 0..23), row i of the stored block
// M2L[b][c] (column-major: a warp's consecutive rows read contiguously) times
// the outgoing charges of c.
__global__ void k_m2l_apply(LevelSet ls) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ls.row0[ls.nlev]) return;
  const LevelView& v = ls.lv[level_of_row(ls, g)];
  const long row = g - ls.row0[level_of_row(ls, g)];
  const int b = v.skel_box[row];
  const int r = v.rank[b];
  const int i = (int)(row - v.skel_off[b]);
  const double* M = v.m2l + v.m2l_off[b] + i;
  double acc = 0.0;
  for (int s = 0; s < 40; ++s) {
    const int c = v.il[(long)b * 40 + s];
    if (c < 0) continue;
    const int rc = v.rank[c];
    const double* qc = v.qhat + v.skel_off[c];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int cc = 0;
    for (; cc + 3 < rc; cc += 4) {
      a0 += M[(long)cc * r] * qc[cc];
      a1 += M[(long)(cc + 1) * r] * qc[cc + 1];
      a2 += M[(long)(cc + 2) * r] * qc[cc + 2];
      a3 += M[(long)(cc + 3) * r] * qc[cc + 3];
    }
    for (; cc < rc; ++cc) a0 += M[(long)cc * r] * qc[cc];
    acc += (a0 + a1) + (a2 + a3);
    M += (long)r * rc;
  }
  v.yhat[row] = acc;
}

// L2L (src/AFMM2DTree.cpp:1180-1197): t = L2P_b yhat_b, one thread per node
// row of the level (column-major L2P: a warp's consecutive rows read
// contiguously); added to the child's incoming potential (node row g of
// level j is skeleton row g of level j+1), or written as the leaf potential.
__global__ void k_l2l(LevelView v, double* __restrict__ child_yhat, double* __restrict__ ys, int leaf) {
  const long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= v.nnodes) return;
  const int b = v.node_box[g];
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int i = (int)(g - v.node_off[b]);
  const double* P = v.l2p + v.l2p_off[b] + i;  // (i, c) at c*n + i
  const double* yb = v.yhat + v.skel_off[b];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int c = 0;
  for (; c + 3 < r; c += 4) {
    a0 += P[(long)c * n] * yb[c];
    a1 += P[(long)(c + 1) * n] * yb[c + 1];
    a2 += P[(long)(c + 2) * n] * yb[c + 2];
    a3 += P[(long)(c + 3) * n] * yb[c + 3];
  }
  for (; c < r; ++c) a0 += P[(long)c * n] * yb[c];
  const double t = (a0 + a1) + (a2 + a3);
  if (leaf) ys[v.leaf_start[b] + i] = t;
  else child_yhat[g] += t;
}

// Near field (src/AFMM2DTree.cpp:1199-1213): per leaf, neighbours 0..7 and
// the leaf itself, kernel evaluated on the fly.  One CTA per leaf; all source
// leaves are staged in shared memory at once; G groups of NT threads split
// the source leaves (group g takes leaves g, g+G, ...), each thread owns one
// target, and the groups' sums are added in group order.
template <class K>
__global__ void k_p2p64(NearView nv, KernelParams kp, const double* __restrict__ qs, double* __restrict__ ys, int NT,
                        int G) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_src[9], s_cnt[9], s_off[10], s_ns;
  const long b = blockIdx.x;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  if (threadIdx.x == 0) {
    int m = 0, off = 0;
    for (int slot = 0; slot < 9; ++slot) {
      const long c = slot < 8 ? nv.nbr[b * 8 + slot] : b;
      if (c < 0) continue;
      s_src[m] = nv.leaf_start[c];
      s_cnt[m] = nv.leaf_cnt[c];
      s_off[m] = off;
      off += nv.leaf_cnt[c];
      ++m;
    }
    s_off[m] = off;
    s_ns = m;
  }
  __syncthreads();
  const int ns = s_ns, tot = s_off[ns];
  double2* sx = (double2*)smem;
  double* sq = (double*)(sx + 9 * nv.nmax);
  double* red = sq + 9 * nv.nmax;  // G x NT
  for (int m = 0; m < ns; ++m)
    for (int t = threadIdx.x; t < s_cnt[m]; t += blockDim.x) {
      sx[s_off[m] + t] = nv.pts[s_src[m] + t];
      sq[s_off[m] + t] = qs[s_src[m] + t];
    }
  __syncthreads();
  (void)tot;
  const int i = threadIdx.x % NT, g = threadIdx.x / NT;
  double acc = 0.0;
  if (i < n) {
    const double2 xi = nv.pts[s0 + i];
    for (int m = g; m < ns; m += G) {
      const int o = s_off[m], nc = s_cnt[m];
      double a0 = 0.0, a1 = 0.0;
      int t = 0;
      for (; t + 1 < nc; t += 2) {
        const double2 p0 = sx[o + t], p1 = sx[o + t + 1];
        const double dx0 = xi.x - p0.x, dy0 = xi.y - p0.y, dx1 = xi.x - p1.x, dy1 = xi.y - p1.y;
        a0 += K::eval(dx0 * dx0 + dy0 * dy0, kp) * sq[o + t];
        a1 += K::eval(dx1 * dx1 + dy1 * dy1, kp) * sq[o + t + 1];
      }
      if (t < nc) {
        const double2 p0 = sx[o + t];
        const double dx0 = xi.x - p0.x, dy0 = xi.y - p0.y;
        a0 += K::eval(dx0 * dx0 + dy0 * dy0, kp) * sq[o + t];
      }
      acc += a0 + a1;
    }
  }
  red[g * NT + i] = acc;
  __syncthreads();
  if (g == 0 && i < n) {
    double s = ys[s0 + i];
    for (int h = 0; h < G; ++h) s += red[h * NT + i];
    ys[s0 + i] = s;
  }
}

template <class K>
struct P2p64Run {
  static void run(const NearView& nv, const KernelParams& kp, const double* qs, double* ys, cudaStream_t s) {
    P2pShape sh = p2p_shape(nv.nmax);
    size_t smem = (size_t)9 * nv.nmax * (sizeof(double2) + sizeof(double)) + sizeof(double) * sh.threads;
    allow_smem(k_p2p64<K>, smem);
    k_p2p64<K><<<(int)nv.nleaf, sh.threads, smem, s>>>(nv, kp, qs, ys, sh.nt, sh.g);
    AFMM_LAUNCH_CHECK();
  }
};

void sweep_m2m(const MatvecPlan& p, const double* qs, cudaStream_t s, int64_t* launches) {
  for (int j = p.L; j >= 2; --j) {
    const LevelView& v = p.lv[j];
    if (v.nrows == 0) continue;
    k_m2m<<<(int)((v.nrows + 127) / 128), 128, 0, s>>>(v, j == p.L ? qs : p.lv[j + 1].qhat, j == p.L);
    AFMM_LAUNCH_CHECK();
    ++*launches;
  }
}

void sweep_l2l(const MatvecPlan& p, double* ys, cudaStream_t s, int64_t* launches) {
  for (int j = 2; j <= p.L; ++j) {
    const LevelView& v = p.lv[j];
    if (v.nnodes == 0) continue;
    k_l2l<<<(int)((v.nnodes + 127) / 128), 128, 0, s>>>(v, j < p.L ? p.lv[j + 1].yhat : nullptr, ys, j == p.L);
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
    const long rows = p.levels.row0[p.levels.nlev];
    k_m2l_apply<<<(int)((rows + 127) / 128), 128, 0, s>>>(p.levels);
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
