// Kernel-templated part of K3/K4 (ACA skeletonisation and L2P), instantiated
// once per kernel functor by the kernel tables (kernel_table.cuh); the level
// planner that launches them through a table is aca.cu.
//
// K3/K4: ACA skeletonisation and L2P of every box of a level.
//
// Reference: FMM2DTree::getNodes_incoming_box (src/AFMM2DTree.cpp:1009-1061)
// and LowRank::ACA_only_nodes (src/ACA.cpp:27-133).  For box b the rows are
// the box's nodes (leaf points, or the concatenated skeletons of children
// 0..3), the columns the concatenated nodes of its interaction list (inner
// slots 0..15, then outer 0..23).  Partially pivoted ACA picks pivot rows
// (the skeleton) and columns; L2P = Ac * K(R,C)^-1 with Ac the raw pivot
// columns (src/AFMM2DTree.cpp:1057-1059).
//
// B200 mapping: one thread-block cluster of C CTAs per box.  CTA c owns the
// column slice [c*chunk, (c+1)*chunk) and keeps its slice of the ACA factors
// V (rank x chunk, FP64) in shared memory; ranks beyond the shared-memory
// capacity spill to a per-cluster global slot.  The row side (U, n1 x rank)
// is small and replicated in every CTA.  Each ACA step exchanges partial
// results through distributed shared memory: the column argmax, then the
// partial dot products V_l . v; everything else is computed redundantly and
// identically in every CTA, so all CTAs take the same control flow.
//
// Arithmetic follows the reference operation by operation (no FMA, IEEE
// division), and the dot products of the stopping test are correctly rounded
// (double-double accumulation), so residuals, pivots, ranks and L2P equal the
// reference's wherever the kernel entries are equal.
#pragma once
#include <cooperative_groups.h>

#include <cfloat>

#include "aca.cuh"
#include "afmm_internal.cuh"

namespace afmm {

namespace aca_detail {

namespace cg = cooperative_groups;

// Argmax of |v| over an allowed index set with the semantics of
// LowRank::maxAbsVector (src/ACA.cpp:12-25): the scan starts at the first
// allowed index and moves only on a strictly larger |v|, so ties keep the
// lowest index, NaNs never win, and a NaN at the first allowed index wins.
// (a, v, i) is the argmax over non-NaN entries, (fi, fv) the first allowed
// entry; finish() applies the NaN rule.
constexpr int NONE = 0x7fffffff;
struct ArgMax {
  double a;   // |value| (-1 when no non-NaN entry)
  double v;   // signed value
  int i;      // index
  int fi;     // first allowed index
  double fv;  // value at fi
};

__device__ __forceinline__ ArgMax am_empty() { return ArgMax{-1.0, 0.0, NONE, NONE, 0.0}; }

__device__ __forceinline__ void am_add(ArgMax& m, double v, int i) {
  if (i < m.fi) {
    m.fi = i;
    m.fv = v;
  }
  double a = fabs(v);
  if (a > m.a || (a == m.a && i < m.i)) {
    m.a = a;
    m.v = v;
    m.i = i;
  }
}

__device__ __forceinline__ void am_merge(ArgMax& m, const ArgMax& t) {
  if (t.a > m.a || (t.a == m.a && t.i < m.i)) {
    m.a = t.a;
    m.v = t.v;
    m.i = t.i;
  }
  if (t.fi < m.fi) {
    m.fi = t.fi;
    m.fv = t.fv;
  }
}

__device__ __forceinline__ ArgMax am_finish(ArgMax m) {
  if (m.fi != NONE && isnan(m.fv)) {
    m.a = fabs(m.fv);
    m.v = m.fv;
    m.i = m.fi;
  }
  return m;
}

__device__ __forceinline__ ArgMax warp_argmax(ArgMax m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ArgMax t;
    t.a = __shfl_down_sync(0xffffffffu, m.a, o);
    t.v = __shfl_down_sync(0xffffffffu, m.v, o);
    t.i = __shfl_down_sync(0xffffffffu, m.i, o);
    t.fi = __shfl_down_sync(0xffffffffu, m.fi, o);
    t.fv = __shfl_down_sync(0xffffffffu, m.fv, o);
    am_merge(m, t);
  }
  return m;
}

// Block argmax (not finished); result valid in all threads after return.
__device__ inline ArgMax block_argmax(ArgMax m, ArgMax* red) {
  m = warp_argmax(m);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = m;
  __syncthreads();
  if (w == 0) {
    m = l < ACA_WARPS ? red[l] : am_empty();
    m = warp_argmax(m);
    if (l == 0) red[0] = m;
  }
  __syncthreads();
  ArgMax r = red[0];
  __syncthreads();
  return r;
}

// Cluster-wide argmax through distributed shared memory: each CTA publishes
// its block result in xb[0..4]; after the cluster barrier every CTA combines
// all of them in rank order.  Returns the finished result.
__device__ inline ArgMax cluster_argmax(cg::cluster_group& cluster, ArgMax m, double* xb, ArgMax* s_out) {
  if (threadIdx.x == 0) {
    xb[0] = m.a;
    xb[1] = m.v;
    xb[2] = (double)m.i;
    xb[3] = (double)m.fi;
    xb[4] = m.fv;
  }
  cluster.sync();
  if (threadIdx.x == 0) {
    ArgMax g = am_empty();
    const int C = (int)cluster.num_blocks();
    for (int c = 0; c < C; ++c) {
      double* rb = cluster.map_shared_rank(xb, c);
      am_merge(g, ArgMax{rb[0], rb[1], (int)rb[2], (int)rb[3], rb[4]});
    }
    *s_out = am_finish(g);
  }
  __syncthreads();
  return *s_out;
}

template <class K>
__global__ void __launch_bounds__(ACA_T, 2) k_aca(AcaArgs A) {
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int cid = blockIdx.x / C;
  const int ncl = gridDim.x / C;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* gbase = A.gscr ? A.gscr + ((size_t)cid * C + crank) * A.gslot : nullptr;
  auto place = [&](int a) -> unsigned char* { return A.in_smem[a] ? smem + A.off[a] : gbase + A.off[a]; };
  double2* rows_xy = (double2*)place(AR_ROWS);           // n1max
  double2* cols_xy = (double2*)place(AR_COLS);           // chunk
  double* V = (double*)place(AR_V);                      // vcap * chunk (shared memory)
  double* U = (double*)place(AR_U);                      // ucap * n1max (shared memory)
  double* xdot = (double*)place(AR_XDOT);                // 2 parities x 2 x (rcap + 8): V-dot exchange (hi, lo)
  double* vcol = (double*)place(AR_SMALL);               // rcap
  double* udot = vcol + A.rcap;                          // rcap
  double* vdot = udot + A.rcap;                          // rcap
  double* uri = vdot + A.rcap;                           // rcap: U_l(ri)
  double* vdlo = uri + A.rcap;                           // rcap: low part of this CTA's V-dots
  unsigned char* row_ok = place(AR_OK);                  // n1max
  unsigned char* col_ok = row_ok + A.n1max;              // chunk
  double* xarg = (double*)place(AR_XARG);                // 2 * 8: argmax exchange (shared memory)
  // the V-dot exchange of CTA c of this cluster (shared or global memory)
  auto xdot_of = [&](int c) -> double* {
    if (A.in_smem[AR_XDOT]) return cluster.map_shared_rank(xdot, c);
    return (double*)(A.gscr + ((size_t)cid * C + c) * A.gslot + A.off[AR_XDOT]);
  };
  __shared__ int s_pref[41];
  __shared__ int s_box[40];
  __shared__ ArgMax s_red[ACA_WARPS];
  __shared__ ArgMax s_piv;
  __shared__ double s_colxy[2];

  const int vsp = A.rcap - A.vcap, usp = A.rcap - A.ucap;
  double* my_vspill = A.vspill + ((size_t)cid * C + crank) * (size_t)max(vsp, 0) * A.chunk;
  double* my_uspill = A.uspill + ((size_t)cid * C + crank) * (size_t)max(usp, 0) * A.n1max;
  auto Vrow = [&](int l) -> double* { return l < A.vcap ? V + (size_t)l * A.chunk : my_vspill + (size_t)(l - A.vcap) * A.chunk; };
  auto Urow = [&](int l) -> double* { return l < A.ucap ? U + (size_t)l * A.n1max : my_uspill + (size_t)(l - A.ucap) * A.n1max; };
  int xpar = 0;  // exchange parity

  for (int b = cid; b < A.nbox; b += ncl) {
    const int nb0 = A.node_off[b];
    const int n1 = A.node_off[b + 1] - nb0;
    if (tid == 0) {
      int acc = 0;
      for (int s = 0; s < 40; ++s) {
        int c = A.il[(size_t)b * 40 + s];
        s_pref[s] = acc;
        s_box[s] = c;
        if (c >= 0) acc += A.node_off[c + 1] - A.node_off[c];
      }
      s_pref[40] = acc;
    }
    __syncthreads();
    const int n2 = s_pref[40];
    const int lo = min(n2, crank * A.chunk), hi = min(n2, lo + A.chunk);
    const int nloc = hi - lo;
    for (int i = tid; i < n1; i += ACA_T) {
      rows_xy[i] = A.pts[A.node_ids[nb0 + i]];
      row_ok[i] = 1;
    }
    for (int j = tid; j < nloc; j += ACA_T) {
      int g = lo + j, s = 0;
      while (s_pref[s + 1] <= g) ++s;
      int c = s_box[s];
      cols_xy[j] = A.pts[A.node_ids[A.node_off[c] + (g - s_pref[s])]];
      col_ok[j] = 1;
    }
    __syncthreads();
    const int mn = min(n1, n2);
    int rank = 0;
    if (mn > 0) {
      // ---- first pivot: first row whose largest |entry| exceeds tol (src/ACA.cpp:56-68)
      int ri = 0;
      ArgMax piv = am_empty();
      bool found = false;
      for (int l = 0; l < n1; ++l) {
        ri = l;
        double* V0 = Vrow(0);
        const double2 r = rows_xy[ri];
        ArgMax m = am_empty();
        for (int j = tid; j < nloc; j += ACA_T) {
          double2 c = cols_xy[j];
          double v = K::eval_exact(r2_exact(r.x, r.y, c.x, c.y), A.kp);
          V0[j] = v;
          am_add(m, v, lo + j);
        }
        m = block_argmax(m, s_red);
        piv = cluster_argmax(cluster, m, xarg + xpar * 8, &s_piv);
        xpar ^= 1;
        if (piv.i < 0 || piv.i >= n2) break;  // cannot happen: every column is allowed here
        if (piv.a > A.tol) {
          found = true;
          break;
        }
      }
      if (found) {
        // v = row / row(col), u = raw column (src/ACA.cpp:69-80)
        double* V0 = Vrow(0);
        for (int j = tid; j < nloc; j += ACA_T) V0[j] = __ddiv_rn(V0[j], piv.v);
        const int cj = piv.i;
        const int own = cj / A.chunk, jo = cj - own * A.chunk;
        if (tid == 0) {
          int s = 0;
          while (s_pref[s + 1] <= cj) ++s;
          int pid = A.node_ids[A.node_off[s_box[s]] + (cj - s_pref[s])];
          double2 p = A.pts[pid];
          s_colxy[0] = p.x;
          s_colxy[1] = p.y;
          if (crank == 0) {
            A.rowpiv[(size_t)b * A.rcap] = ri;
            A.colpiv[(size_t)b * A.rcap] = pid;
          }
        }
        __syncthreads();
        double* U0 = Urow(0);
        ArgMax m = am_empty();
        if (crank == own && tid == 0) col_ok[jo] = 0;
        if (tid == 0) row_ok[ri] = 0;
        __syncthreads();
        for (int i = tid; i < n1; i += ACA_T) {
          double2 r = rows_xy[i];
          double u = K::eval_exact(r2_exact(r.x, r.y, s_colxy[0], s_colxy[1]), A.kp);
          U0[i] = u;
          if (row_ok[i]) am_add(m, u, i);
        }
        rank = 1;
        m = am_finish(block_argmax(m, s_red));
        ri = (m.i == NONE) ? 0 : m.i;  // src/ACA.cpp:84 (an empty set yields index 0)
        double normS = 0.0, prev = DBL_MAX;
        // ---- main loop (src/ACA.cpp:86-130)
        while (fabs(prev - normS) >= A.tol * prev && rank < mn) {
          const int k = rank;
          const double2 rr = rows_xy[ri];
          double* Vk = Vrow(k);
          for (int l = tid; l < k; l += ACA_T) uri[l] = Urow(l)[ri];
          __syncthreads();
          // residual row over this CTA's columns
          ArgMax mm = am_empty();
          for (int j = tid; j < nloc; j += ACA_T) {
            double2 c = cols_xy[j];
            double v = K::eval_exact(r2_exact(rr.x, rr.y, c.x, c.y), A.kp);
            // the reference's order of subtractions; sixteen V loads issued ahead
            int l = 0;
            for (; l + 16 <= k; l += 16) {
              double w[16];
#pragma unroll
              for (int t = 0; t < 16; ++t) w[t] = Vrow(l + t)[j];
#pragma unroll
              for (int t = 0; t < 16; ++t) v = __dsub_rn(v, __dmul_rn(uri[l + t], w[t]));
            }
            for (; l + 4 <= k; l += 4) {
              double w[4];
#pragma unroll
              for (int t = 0; t < 4; ++t) w[t] = Vrow(l + t)[j];
#pragma unroll
              for (int t = 0; t < 4; ++t) v = __dsub_rn(v, __dmul_rn(uri[l + t], w[t]));
            }
            for (; l < k; ++l) v = __dsub_rn(v, __dmul_rn(uri[l], Vrow(l)[j]));
            Vk[j] = v;
            if (col_ok[j]) am_add(mm, v, lo + j);
          }
          mm = block_argmax(mm, s_red);
          const ArgMax pv = cluster_argmax(cluster, mm, xarg + xpar * 8, &s_piv);
          xpar ^= 1;
          // Every CTA sees the same pv; an empty allowed set cannot occur
          // while rank < min(n1, n2), but stop rather than index out of range.
          if (pv.i < 0 || pv.i >= n2) break;
          const int cjk = pv.i;
          const int ownk = cjk / A.chunk, jok = cjk - ownk * A.chunk;
          // v = residual / pivot
          for (int j = tid; j < nloc; j += ACA_T) Vk[j] = __ddiv_rn(Vk[j], pv.v);
          // V_l(col) for l < k from the owning CTA
          for (int l = tid; l < k; l += ACA_T) {
            double val;
            if (l < A.vcap) {
              double* rv = cluster.map_shared_rank(V, ownk);
              val = rv[(size_t)l * A.chunk + jok];
            } else {
              double* sp = A.vspill + ((size_t)cid * C + ownk) * (size_t)vsp * A.chunk;
              val = sp[(size_t)(l - A.vcap) * A.chunk + jok];
            }
            vcol[l] = val;
          }
          if (tid == 0) {
            int s = 0;
            while (s_pref[s + 1] <= cjk) ++s;
            int pid = A.node_ids[A.node_off[s_box[s]] + (cjk - s_pref[s])];
            double2 p = A.pts[pid];
            s_colxy[0] = p.x;
            s_colxy[1] = p.y;
            if (crank == 0) {
              A.rowpiv[(size_t)b * A.rcap + k] = ri;
              A.colpiv[(size_t)b * A.rcap + k] = pid;
            }
          }
          __syncthreads();
          // residual column u (all rows, every CTA)
          double* Uk = Urow(k);
          for (int i = tid; i < n1; i += ACA_T) {
            double2 r = rows_xy[i];
            double u = K::eval_exact(r2_exact(r.x, r.y, s_colxy[0], s_colxy[1]), A.kp);
            int l = 0;
            for (; l + 4 <= k; l += 4) {
              const double w0 = Urow(l)[i], w1 = Urow(l + 1)[i], w2 = Urow(l + 2)[i], w3 = Urow(l + 3)[i];
              u = __dsub_rn(u, __dmul_rn(vcol[l], w0));
              u = __dsub_rn(u, __dmul_rn(vcol[l + 1], w1));
              u = __dsub_rn(u, __dmul_rn(vcol[l + 2], w2));
              u = __dsub_rn(u, __dmul_rn(vcol[l + 3], w3));
            }
            for (; l < k; ++l) u = __dsub_rn(u, __dmul_rn(vcol[l], Urow(l)[i]));
            Uk[i] = u;
          }
          __syncthreads();
          // Partial V_l . v over this CTA's columns and U_l . u (redundant in every
          // CTA), accumulated in double-double: the cluster-wide sums are then
          // rounded once, so they are the correctly rounded dot products
          // whatever the summation order (the stopping test depends on them).
          for (int l = warp; l <= k; l += ACA_WARPS) {
            const double* Vl = Vrow(l);
            dd sv{0.0, 0.0};
            int j = lane;
            for (; j + 480 < nloc; j += 512) {  // same order of additions, loads issued ahead
              double a[16], c[16];
#pragma unroll
              for (int t = 0; t < 16; ++t) {
                a[t] = Vl[j + 32 * t];
                c[t] = Vk[j + 32 * t];
              }
#pragma unroll
              for (int t = 0; t < 16; ++t) {
                const double p = __dmul_rn(a[t], c[t]);
                sv = dd_add(sv, dd{p, __fma_rn(a[t], c[t], -p)});
              }
            }
            for (; j < nloc; j += 32) {
              const double a = Vl[j], c = Vk[j];
              const double p = __dmul_rn(a, c);
              sv = dd_add(sv, dd{p, __fma_rn(a, c, -p)});
            }
            for (int o = 16; o > 0; o >>= 1)
              sv = dd_add(sv, dd{__shfl_down_sync(0xffffffffu, sv.hi, o), __shfl_down_sync(0xffffffffu, sv.lo, o)});
            if (lane == 0) {
              vdot[l] = sv.hi;
              vdlo[l] = sv.lo;
            }
            const double* Ul = Urow(l);
            dd su{0.0, 0.0};
            for (int i = lane; i < n1; i += 32) {
              const double a = Ul[i], c = Uk[i];
              const double p = __dmul_rn(a, c);
              su = dd_add(su, dd{p, __fma_rn(a, c, -p)});
            }
            for (int o = 16; o > 0; o >>= 1)
              su = dd_add(su, dd{__shfl_down_sync(0xffffffffu, su.hi, o), __shfl_down_sync(0xffffffffu, su.lo, o)});
            if (lane == 0) udot[l] = __dadd_rn(su.hi, su.lo);
          }
          __syncthreads();
          const size_t xo = (size_t)xpar * 2 * (A.rcap + 8);
          for (int l = tid; l <= k; l += ACA_T) {
            xdot[xo + 2 * l] = vdot[l];
            xdot[xo + 2 * l + 1] = vdlo[l];
          }
          if (tid == 0) {
            if (ownk == crank) col_ok[jok] = 0;
            row_ok[ri] = 0;
          }
          cluster.sync();
          for (int l = tid; l <= k; l += ACA_T) {
            dd s{0.0, 0.0};
            for (int c = 0; c < C; ++c) {
              const double* xc = xdot_of(c) + xo;
              s = dd_add(s, dd{xc[2 * l], xc[2 * l + 1]});
            }
            vdot[l] = __dadd_rn(s.hi, s.lo);
          }
          xpar ^= 1;
          __syncthreads();
          rank = k + 1;
          // norm update (src/ACA.cpp:122-128), identical in every thread
          if (rank != 2) prev = normS;
          double un = sqrt(udot[k]), vn = sqrt(vdot[k]);
          double t = un * vn;
          double ns = __dadd_rn(__dmul_rn(normS, normS), __dmul_rn(t, t));
          for (int l = 0; l <= k; ++l) ns = __dadd_rn(ns, __dmul_rn(2.0, fabs(__dmul_rn(udot[l], vdot[l]))));
          normS = sqrt(ns);
          // next pivot row: largest |u| over remaining rows (src/ACA.cpp:129)
          ArgMax mr = am_empty();
          for (int i = tid; i < n1; i += ACA_T)
            if (row_ok[i]) am_add(mr, Uk[i], i);
          mr = am_finish(block_argmax(mr, s_red));
          ri = (mr.i == NONE) ? 0 : mr.i;
        }
      }
    }
    if (crank == 0 && tid == 0) A.rank_out[b] = rank;
    cluster.sync();
  }
}

template <class K>
struct AcaLaunch {
  static void run(const AcaArgs& a, int C, int ncl, size_t smem, cudaStream_t s) {
    auto fn = k_aca<K>;
    AFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (C > 8) AFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ncl * C);
    cfg.blockDim = dim3(ACA_T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    AFMM_CUDA(cudaLaunchKernelEx(&cfg, fn, a));
  }
  static void occupancy(int C, size_t smem, int* ncl) {
    auto fn = k_aca<K>;
    AFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (C > 8) AFMM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(ACA_T);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    AFMM_CUDA(cudaOccupancyMaxActiveClusters(ncl, fn, &cfg));
  }
};

template <class K>
struct AcaOcc {
  static void run(int C, size_t smem, int* ncl) { AcaLaunch<K>::occupancy(C, smem, ncl); }
};
template <class K>
struct AcaRun {
  static void run(const AcaArgs& a, int C, int ncl, size_t smem, cudaStream_t s) { AcaLaunch<K>::run(a, C, ncl, smem, s); }
};

// GA = true keeps the r x r factor in a per-CTA global scratch slot (ranks
// whose factor does not fit in shared memory); the CTA then loops over boxes.
template <class K, bool GA>
__global__ void __launch_bounds__(L2P_T) k_l2p(L2pArgs P) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_piv;
  for (int b = blockIdx.x; b < P.nbox; b += gridDim.x) {
    const int r = P.rank[b];
    if (r == 0) continue;
    const int nb0 = P.node_off[b];
    const int n = P.node_off[b + 1] - nb0;
    const int rr2 = GA ? 0 : ((r * r + 1) & ~1);  // keep the double2 array 16-byte aligned
    double* Am = GA ? P.gscratch + (size_t)blockIdx.x * P.rmax * P.rmax : (double*)smem;  // r x r, row-major
    double2* cxy = (double2*)((double*)smem + rr2);  // r pivot-column points
    // r x xs scratch, one column per solving thread: shared memory, or with the
    // factor in global memory (large ranks) a per-CTA global slot, so that every
    // thread solves and the CTA's small shared footprint lets several CTAs share an SM
    double* X = GA ? P.gx + (size_t)blockIdx.x * P.rmax * P.xs : (double*)(cxy + r);
    int* perm = GA ? (int*)(cxy + r) : (int*)(X + (size_t)r * P.xs);  // r
    const int so = P.skel_off[b];
    __syncthreads();
    for (int l = threadIdx.x; l < r; l += L2P_T) {
      int rid = P.node_ids[nb0 + P.rowpiv[(size_t)b * P.rcap + l]];
      int cid = P.colpiv[(size_t)b * P.rcap + l];
      P.skel_ids[so + l] = rid;
      P.cpiv_ids[so + l] = cid;
      P.skel_xy[so + l] = P.pts[rid];
      cxy[l] = P.pts[cid];
      perm[l] = l;
    }
    __syncthreads();
    // A(i,j) = D(j,i) = K(R_j, C_i)
    for (int e = threadIdx.x; e < r * r; e += L2P_T) {
      int i = e / r, j = e % r;
      double2 rp = P.pts[P.node_ids[nb0 + P.rowpiv[(size_t)b * P.rcap + j]]];
      Am[e] = K::eval_exact(r2_exact(rp.x, rp.y, cxy[i].x, cxy[i].y), P.kp);
    }
    __syncthreads();
    for (int kk = 0; kk < r; ++kk) {
      if (threadIdx.x < 32) {
        double best = -1.0;
        int bi = kk;
        for (int i = kk + threadIdx.x; i < r; i += 32) {
          double a = fabs(Am[(size_t)i * r + kk]);
          if (a > best) { best = a; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
          double ob = __shfl_down_sync(0xffffffffu, best, o);
          int oi = __shfl_down_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (threadIdx.x == 0) s_piv = bi;
      }
      __syncthreads();
      const int pv = s_piv;
      if (pv != kk) {
        for (int j = threadIdx.x; j < r; j += L2P_T) {
          double t = Am[(size_t)kk * r + j];
          Am[(size_t)kk * r + j] = Am[(size_t)pv * r + j];
          Am[(size_t)pv * r + j] = t;
        }
        if (threadIdx.x == 0) {
          int t = perm[kk];
          perm[kk] = perm[pv];
          perm[pv] = t;
        }
      }
      __syncthreads();
      const double d = Am[(size_t)kk * r + kk];
      if (d != 0.0) {
        for (int i = kk + 1 + threadIdx.x; i < r; i += L2P_T) Am[(size_t)i * r + kk] = __ddiv_rn(Am[(size_t)i * r + kk], d);
        __syncthreads();
        const int m = r - kk - 1;
        for (int e = threadIdx.x; e < m * m; e += L2P_T) {
          int i = kk + 1 + e / m, j = kk + 1 + e % m;
          Am[(size_t)i * r + j] = __dsub_rn(Am[(size_t)i * r + j], __dmul_rn(Am[(size_t)i * r + kk], Am[(size_t)kk * r + j]));
        }
      }
      __syncthreads();
    }
    double* out = P.l2p + P.l2p_off[b];  // n x r column-major: (i, l) at l*n + i
    const int xs = P.xs;
    for (int i0 = 0; i0 < n; i0 += xs) {
      const int i = i0 + threadIdx.x;
      if (threadIdx.x < xs && i < n) {
        double* x = X + threadIdx.x;  // x[l * xs]
        double2 rp = P.pts[P.node_ids[nb0 + i]];
        for (int l = 0; l < r; ++l) {
          double2 c = cxy[perm[l]];
          double s = K::eval_exact(r2_exact(rp.x, rp.y, c.x, c.y), P.kp);
          for (int m = 0; m < l; ++m) s -= Am[(size_t)l * r + m] * x[m * xs];
          x[l * xs] = s;
        }
        for (int l = r - 1; l >= 0; --l) {
          double s = x[l * xs];
          for (int m = l + 1; m < r; ++m) s -= Am[(size_t)l * r + m] * x[m * xs];
          x[l * xs] = s / Am[(size_t)l * r + l];
        }
        for (int l = 0; l < r; ++l) out[(size_t)l * n + i] = x[l * xs];
      }
    }
    __syncthreads();
  }
}

template <class K>
struct L2pRun {
  static void run(const L2pArgs& a, size_t smem, bool global_factor, int grid, cudaStream_t s) {
    if (global_factor) {
      AFMM_CUDA(cudaFuncSetAttribute(k_l2p<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_l2p<K, true><<<grid, L2P_T, smem, s>>>(a);
    } else {
      AFMM_CUDA(cudaFuncSetAttribute(k_l2p<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_l2p<K, false><<<grid, L2P_T, smem, s>>>(a);
    }
    AFMM_LAUNCH_CHECK();
  }
};

}  // namespace aca_detail

}  // namespace afmm
