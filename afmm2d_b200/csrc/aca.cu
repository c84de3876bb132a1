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
#include <algorithm>
#include <chrono>
#include <cfloat>

#include "afmm_internal.cuh"
#include "aca.cuh"
#include "kernel_table.cuh"

namespace afmm {

void aca_level(const AcaLevelIn& in, AcaLevelOut& out, DevArena& arena, AcaScratch& scratch, cudaStream_t s,
               int64_t* launches) {
  const int n1max = std::max(in.n1max, 1);
  const int n2max = std::max(in.n2max, 1);
  const int rcap = std::max(1, std::min(n1max, n2max));
  // Cluster size: smallest power of two (<= 16) whose column slice keeps at
  // least min(rcap, 48) ranks of V in shared memory -- unless the level has
  // enough boxes to fill the GPU with smaller clusters (boxes x C >= two CTAs
  // per SM), in which case boxes run side by side and the V ranks beyond the
  // shared-memory capacity live in L2-resident global slots.  Many-box levels
  // use half the shared-memory budget, so two CTAs share an SM.  The small
  // per-CTA arrays go to shared memory first (argmax exchange, column and row
  // coordinates, flags, per-rank vectors, V-dot exchange) while they fit in a
  // quarter of the budget; whatever does not fit lives in a per-CTA slot of
  // global memory.  U then takes up to a quarter and V the rest.
  int dev = 0, nsm = 148;
  AFMM_CUDA(cudaGetDevice(&dev));
  AFMM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  long want_ctas = 2L * nsm;
  size_t budget = in.nbox >= want_ctas ? 100 * 1024 : 200 * 1024;
  if (in.ctas_per_sm == 1 || in.ctas_per_sm == 2) {  // set-up tuning overrides
    budget = in.ctas_per_sm == 1 ? 200 * 1024 : 100 * 1024;
    want_ctas = (long)in.ctas_per_sm * nsm;
  }
  if (in.cluster != 0 && (in.cluster < 1 || in.cluster > 16 || (in.cluster & (in.cluster - 1))))
    throw Error{AFMM_BAD_ARG, "ACA cluster size must be a power of two up to 16"};
  int C = 1, chunk = 0, vcap = 0, ucap = 0;
  size_t smem = 0, gslot = 0;
  size_t off[AR_N] = {0};
  int in_smem[AR_N] = {0};
  for (C = 1;; C *= 2) {
    chunk = (n2max + C - 1) / C;
    size_t sz[AR_N];
    sz[AR_ROWS] = sizeof(double2) * (size_t)n1max;
    sz[AR_COLS] = sizeof(double2) * (size_t)chunk;
    sz[AR_XDOT] = sizeof(double) * 4 * (size_t)(rcap + 8);
    sz[AR_SMALL] = sizeof(double) * 5 * (size_t)rcap;
    sz[AR_OK] = (size_t)n1max + chunk;
    sz[AR_XARG] = sizeof(double) * 16;
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    size_t used = 0, gused = 0;
    const int order[] = {AR_XARG, AR_COLS, AR_ROWS, AR_SMALL, AR_XDOT, AR_OK};
    for (int a : order) {
      if (a == AR_XARG || used + al(sz[a]) <= budget / 4) {
        in_smem[a] = 1;
        off[a] = used;
        used += al(sz[a]);
      } else {
        in_smem[a] = 0;
        off[a] = gused;
        gused += al(sz[a]);
      }
    }
    ucap = std::min<long>(rcap, (long)((budget / 4) / (sizeof(double) * n1max)));
    in_smem[AR_U] = 1;
    off[AR_U] = used;
    used += al(sizeof(double) * (size_t)ucap * n1max);
    size_t left = budget > used ? budget - used : 0;
    vcap = std::min<long>(rcap, (long)(left / (sizeof(double) * chunk)));
    const bool pick = in.cluster ? C == in.cluster : (vcap >= std::min(rcap, 48) || C == 16 || in.nbox * C >= want_ctas);
    if (pick) {
      in_smem[AR_V] = 1;
      off[AR_V] = used;
      used += al(sizeof(double) * (size_t)vcap * chunk);
      smem = used;
      gslot = gused;
      break;
    }
  }
  int ncl = 0;
  kernel_table(in.kp.id).aca_occupancy(C, smem, &ncl);
  if (ncl <= 0) throw Error{AFMM_CUDA_ERR, "ACA kernel cannot be resident (cluster occupancy 0)"};
  ncl = (int)std::min<long>(ncl, std::max<long>(1, in.nbox));
  const int vsp = rcap - vcap, usp = rcap - ucap;
  // The spill slots are sized for the worst-case rank min(n1, n2) of every
  // cluster in flight, which on levels of large ranks (e.g. rank ~900 boxes
  // of a 16M-point spiral) exceeds the device: keep them within half of the
  // memory that is free (counting the pool's buffer, released before it
  // grows) by running fewer clusters; each cluster then takes more boxes in
  // turn, and the results do not change.
  {
    size_t free_b = 0, total_b = 0;
    AFMM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t have = (free_b + scratch.work.cap) / 2;
    const size_t per_cl = (size_t)C * (gslot + sizeof(double) * ((size_t)std::max(vsp, 0) * chunk +
                                                                 (size_t)std::max(usp, 0) * n1max));
    const size_t fixed = 2 * sizeof(int32_t) * (size_t)in.nbox * rcap + 4096;
    if (per_cl > 0) {
      const long fit = have > fixed ? (long)((have - fixed) / per_cl) : 0;
      if (fit < 1)
        throw Error{AFMM_OOM, "ACA working memory of one cluster (" + std::to_string(per_cl) +
                                  " bytes) exceeds half of the free device memory"};
      ncl = (int)std::min<long>(ncl, fit);
    }
  }
  AcaArgs a;
  a.nbox = (int)in.nbox;
  a.pts = in.pts;
  a.node_off = in.node_off;
  a.node_ids = in.node_ids;
  a.il = in.il;
  a.tol = in.tol;
  a.kp = in.kp;
  a.rcap = rcap;
  a.n1max = n1max;
  a.chunk = chunk;
  a.vcap = vcap;
  a.ucap = ucap;
  for (int t = 0; t < AR_N; ++t) {
    a.off[t] = off[t];
    a.in_smem[t] = in_smem[t];
  }
  a.gslot = gslot;
  const size_t n_gscr = gslot > 0 ? (size_t)ncl * C * gslot : 0;
  const size_t n_vsp = vsp > 0 ? (size_t)ncl * C * vsp * chunk : 0;
  const size_t n_usp = usp > 0 ? (size_t)ncl * C * usp * n1max : 0;
  const size_t n_piv = (size_t)in.nbox * rcap;
  DevScratch& w = scratch.work;
  const auto t_res = std::chrono::steady_clock::now();
  const size_t need = DevScratch::need({n_gscr, sizeof(double) * n_vsp, sizeof(double) * n_usp,
                                        sizeof(int32_t) * n_piv, sizeof(int32_t) * n_piv});
  w.reserve(need);
  out.scratch_bytes = need;
  out.scratch_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_res).count();
  a.gscr = n_gscr ? w.take<unsigned char>(n_gscr) : nullptr;
  a.vspill = n_vsp ? w.take<double>(n_vsp) : nullptr;
  a.uspill = n_usp ? w.take<double>(n_usp) : nullptr;
  out.rcap = rcap;
  out.rank = in.rank_out;
  a.rank_out = in.rank_out;
  int32_t* rowpiv = w.take<int32_t>(n_piv);
  int32_t* colpiv = w.take<int32_t>(n_piv);
  a.rowpiv = rowpiv;
  a.colpiv = colpiv;
  const auto t0 = std::chrono::steady_clock::now();
  kernel_table(in.kp.id).aca_run(a, C, ncl, smem, s);
  *launches += 1;
  out.cluster = C;
  out.clusters = ncl;
  // ranks -> offsets (host), then L2P with exact offsets
  std::vector<int32_t> h_rank(in.nbox);
  AFMM_CUDA(cudaMemcpyAsync(h_rank.data(), in.rank_out, sizeof(int32_t) * in.nbox, cudaMemcpyDeviceToHost, s));
  AFMM_CUDA(cudaStreamSynchronize(s));
  const auto t1 = std::chrono::steady_clock::now();
  out.aca_s = std::chrono::duration<double>(t1 - t0).count();
  out.h_rank = h_rank;
  out.h_skel_off.assign(in.nbox + 1, 0);
  out.h_l2p_off.assign(in.nbox + 1, 0);
  int rmax = 0;
  for (long b = 0; b < in.nbox; ++b) {
    int n = in.h_node_off[b + 1] - in.h_node_off[b];
    out.h_skel_off[b + 1] = out.h_skel_off[b] + h_rank[b];
    out.h_l2p_off[b + 1] = out.h_l2p_off[b] + (int64_t)n * h_rank[b];
    rmax = std::max(rmax, h_rank[b]);
  }
  out.rmax = rmax;
  const long tr = out.h_skel_off[in.nbox];
  out.skel_off = arena.alloc<int32_t>(in.nbox + 1);
  out.l2p_off = arena.alloc<int64_t>(in.nbox + 1);
  out.skel_ids = arena.alloc<int32_t>(tr);
  out.cpiv_ids = arena.alloc<int32_t>(tr);
  out.skel_xy = arena.alloc<double2>(tr);
  out.l2p = arena.alloc<double>(out.h_l2p_off[in.nbox] + 4);  // + 32 B for whole-piece L2 prefetches
  AFMM_CUDA(cudaMemcpyAsync(out.skel_off, out.h_skel_off.data(), sizeof(int32_t) * (in.nbox + 1), cudaMemcpyHostToDevice, s));
  AFMM_CUDA(cudaMemcpyAsync(out.l2p_off, out.h_l2p_off.data(), sizeof(int64_t) * (in.nbox + 1), cudaMemcpyHostToDevice, s));
  if (rmax > 0) {
    L2pArgs p;
    p.nbox = (int)in.nbox;
    p.pts = in.pts;
    p.node_off = in.node_off;
    p.node_ids = in.node_ids;
    p.rank = in.rank_out;
    p.rowpiv = rowpiv;
    p.colpiv = colpiv;
    p.rcap = rcap;
    p.kp = in.kp;
    p.skel_off = out.skel_off;
    p.l2p_off = out.l2p_off;
    p.skel_ids = out.skel_ids;
    p.cpiv_ids = out.cpiv_ids;
    p.skel_xy = out.skel_xy;
    p.l2p = out.l2p;
    const size_t budget2 = 200 * 1024;
    // factor in shared memory when it leaves room for >= 32 solving threads
    size_t fa = sizeof(double) * (size_t)((rmax * rmax + 1) & ~1);
    size_t rest = sizeof(double2) * rmax + sizeof(int) * rmax + 64;
    bool global_factor = fa + rest + sizeof(double) * (size_t)rmax * 32 > budget2;
    size_t base = (global_factor ? 0 : fa) + rest;
    // with the factor in global memory the solve columns go there too: all
    // L2P_T threads solve (shared memory would hold only ~26 columns at rank
    // ~900) and the CTA's shared footprint stays small
    p.xs = global_factor ? L2P_T : (int)std::min<size_t>(L2P_T, (budget2 - base) / (sizeof(double) * rmax));
    if (p.xs < 1) throw Error{AFMM_BAD_ARG, "box rank " + std::to_string(rmax) + " too large for the L2P solve"};
    size_t sm = base + (global_factor ? 0 : sizeof(double) * (size_t)rmax * p.xs);
    p.rmax = rmax;
    int grid = (int)in.nbox;
    p.gscratch = nullptr;
    p.gx = nullptr;
    if (global_factor) {
      grid = (int)std::min<long>(in.nbox, 148 * 8);
      const size_t n_fac = (size_t)grid * rmax * rmax;
      const size_t n_x = (size_t)grid * rmax * p.xs;
      scratch.factors.reserve(DevScratch::need({sizeof(double) * n_fac, sizeof(double) * n_x}));
      p.gscratch = scratch.factors.take<double>(n_fac);
      p.gx = scratch.factors.take<double>(n_x);
    }
    kernel_table(in.kp.id).l2p_run(p, sm, global_factor, grid, s);
    *launches += 1;
  }
  AFMM_CUDA(cudaStreamSynchronize(s));
  out.l2p_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
}

}  // namespace afmm
