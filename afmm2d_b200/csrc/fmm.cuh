// Tree views handed to the sweep kernels (see fmm.cu, mixed.cu).
#pragma once
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "afmm_internal.cuh"

namespace afmm {

constexpr int kMaxLevels = 16;

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
  const int32_t* wgrp_box = nullptr;  // row chunk (<= 32 skeleton rows of one box) -> box
  const int32_t* wgrp_row = nullptr;  // row chunk -> first skeleton row
  long nwgroups = 0;
  const int32_t* nwgrp_box = nullptr;  // node-row chunk (<= 32 node rows of one box) -> box
  const int32_t* nwgrp_row = nullptr;  // node-row chunk -> first node row
  long nnwgroups = 0;
  const int32_t* ptile_par = nullptr;  // parent row tile (<= 128 rows of 4 children) -> parent box
  const int32_t* ptile_row = nullptr;  // parent row tile -> first row of the children's concatenated rows
  long nptiles = 0;
  const int32_t* tile_box = nullptr;  // row tile (<= 128 skeleton rows of one box) -> box
  const int32_t* tile_row = nullptr;  // row tile -> first row within the box (a multiple of 8)
  long ntiles = 0;
  unsigned char* m2l_s = nullptr;      // byte-plane blocks (m2l_i8_k.cuh; null when not stored)
  const int64_t* m2l_s_off = nullptr;
  unsigned char* qs8 = nullptr;        // charges' byte planes of the current pass
  const int32_t* qs8_off = nullptr;
  int32_t* qs_exp = nullptr;
  int64_t* qs_sum = nullptr;
  uint32_t* m2l_q = nullptr;          // 32-bit fixed-point blocks (null when not stored)
  double2* m2l_dec = nullptr;         // per (box, slot) decode constants
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
  long wgrp0[kMaxLevels + 1] = {0};  // prefix of warp row-chunk counts
  long pt0[kMaxLevels + 1] = {0};    // prefix of parent row-tile counts
  long t0[kMaxLevels + 1] = {0};     // prefix of 128-row tile counts
  long b0[kMaxLevels + 1] = {0};     // prefix of box counts
  int src[kMaxLevels] = {0};         // index of entry j among levels 2..L (per-level device tables)
  uint32_t pf_ahead = 12 * 1024;     // L2 prefetch window of the stored-block M2L kernels (bytes)
};

// The levels of `ls` whose bit in `mask` (bit t = entry t) equals `keep`,
// with their prefixes rebuilt and their original indices kept in src.
inline LevelSet level_subset(const LevelSet& ls, uint32_t mask, bool keep) {
  LevelSet o;
  o.pf_ahead = ls.pf_ahead;
  for (int t = 0; t < ls.nlev; ++t) {
    if ((((mask >> t) & 1u) != 0) != keep) continue;
    const int n = o.nlev;
    o.lv[n] = ls.lv[t];
    o.src[n] = ls.src[t];
    o.row0[n + 1] = o.row0[n] + (ls.row0[t + 1] - ls.row0[t]);
    o.grp0[n + 1] = o.grp0[n] + (ls.grp0[t + 1] - ls.grp0[t]);
    o.cgrp0[n + 1] = o.cgrp0[n] + (ls.cgrp0[t + 1] - ls.cgrp0[t]);
    o.wgrp0[n + 1] = o.wgrp0[n] + (ls.wgrp0[t + 1] - ls.wgrp0[t]);
    o.pt0[n + 1] = o.pt0[n] + (ls.pt0[t + 1] - ls.pt0[t]);
    o.t0[n + 1] = o.t0[n] + (ls.t0[t + 1] - ls.t0[t]);
    o.b0[n + 1] = o.b0[n] + (ls.b0[t + 1] - ls.b0[t]);
    ++o.nlev;
  }
  return o;
}

// Tunable launch parameters of a handle (afmm_autotune / afmm_set_tuning);
// none of them changes the FP64 path's arithmetic.
struct Tuning {
  uint32_t pf_fp64 = 12 * 1024;     // L2 prefetch window of the one-column FP64 / mixed M2L (bytes)
  uint32_t pf_batched = 12 * 1024;  // L2 prefetch window of the batched stored-block M2L (bytes)
  uint32_t otf_mixed = 0;           // bit t: level t + 2 evaluated on the fly in the one-column mixed path
  uint32_t otf_batched = 0;         // bit t: level t + 2 evaluated on the fly in batched mixed passes
  int host_pass_cols = 0;           // columns per pass of host-pointer batched calls (0: automatic)
  int m2l_t16 = 0;                  // 16-column stored M2L on transposed m16n8k4 tiles (else 8x8x4 tiles)
  int p2p_tc = 0;                   // 16-column mixed near field on tcgen05 tiles (else mma.sync tiles)
  int m2l_tc = 0;  // 16-column mixed stored M2L on tcgen05: 2 exact integer products from the byte
                   // planes; 1 TF32 tiles, an FP32 far field outside the mixed tolerance on deep trees,
                   // never chosen by the autotuner; 0 FP64 tiles
};

// Grid cell (ix, iy) of box k at level j: the base-4 digits of k read as
// child offsets 0:(0,0) 1:(1,0) 2:(1,1) 3:(0,1) (src/AFMM2DTree.cpp:978-986),
// and the inverse.
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

// L2 prefetch of a global range: cp.async.bulk.prefetch.L2 (16-byte aligned
// start, size a multiple of 16).  Issued by one lane.
__device__ __forceinline__ void prefetch_l2_bulk(uintptr_t p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Streams a box's contiguous M2L region into L2 ahead of the warp that
// consumes it in order: `advance(pos)` keeps the prefetched front `ahead`
// bytes beyond `pos` (0: no prefetch), in kStep pieces (the last piece may
// extend < 16 bytes past the region; the block allocations are padded for
// that).
struct L2Stream {
  static constexpr uintptr_t kStep = 4096;
  uintptr_t front, end, ahead;
  __device__ __forceinline__ L2Stream(const void* begin, const void* stop, uintptr_t window)
      : front((uintptr_t)begin & ~(uintptr_t)15), end((uintptr_t)stop), ahead(window) {}
  __device__ __forceinline__ void advance(const void* pos, int lane) {
    uintptr_t upto = (uintptr_t)pos + ahead;
    if (upto > end) upto = end;
    while (front < upto) {  // warp-uniform
      if (lane == 0) {
        const uintptr_t left = (end - front + 15) & ~(uintptr_t)15;
        prefetch_l2_bulk(front, (uint32_t)(left < kStep ? left : kStep));
      }
      front += kStep;
    }
  }
};

// Prefetches [begin, end) into L2 in 4 KB pieces spread over the warp's
// lanes (start rounded down to 16 bytes, end up to 16 bytes: the arrays are
// allocated with that much padding).
__device__ __forceinline__ void prefetch_l2_region(const void* begin, const void* end, int lane) {
  const uintptr_t a = (uintptr_t)begin & ~(uintptr_t)15;
  const uintptr_t e = ((uintptr_t)end + 15) & ~(uintptr_t)15;
  for (uintptr_t p = a + (uintptr_t)lane * 4096; p < e; p += 32 * 4096) {
    const uintptr_t left = e - p;
    prefetch_l2_bulk(p, (uint32_t)(left < 4096 ? left : 4096));
  }
}

// Value of a 32-bit fixed-point M2L entry: the double with high word
// 0x43300000 and low word u is 2^52 + u exactly, so one FMA with the block's
// decode constants (2^k, -(2^52 + 2^31) 2^k) gives (u - 2^31) 2^k exactly.
__device__ __forceinline__ double decode_q32(uint32_t u, double2 dec) {
  return fma(__hiloint2double(0x43300000, (int)u), dec.x, dec.y);
}

// Leaf-level data for the near field.
struct NearView {
  long nleaf = 0;  // leaves of the launch: leaf0 .. leaf0 + nleaf - 1 (a shard's range, else all)
  long leaf0 = 0;
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
  // stages run one after another on the launching stream (no near field
  // beside the far field), so every stage is its kernels' own duration
  bool serial = false;
  // spans timed on another stream (a stage that overlaps the marked ones)
  struct Span {
    std::string name;
    cudaEvent_t b, e;
  };
  std::vector<Span> spans;
  size_t nspans = 0;
  void reset() {
    used = 0;
    nspans = 0;
  }
  int span_begin(cudaStream_t s, const char* name) {
    if (nspans == spans.size()) {
      Span sp{name, nullptr, nullptr};
      cudaEventCreate(&sp.b);
      cudaEventCreate(&sp.e);
      spans.push_back(sp);
    }
    spans[nspans].name = name;
    cudaEventRecord(spans[nspans].b, s);
    return (int)nspans++;
  }
  void span_end(cudaStream_t s, int i) { cudaEventRecord(spans[(size_t)i].e, s); }
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
    for (size_t i = 0; i < nspans; ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, spans[i].b, spans[i].e);
      bool found = false;
      for (auto& o : out)
        if (o.first == spans[i].name) {
          o.second += ms;
          found = true;
        }
      if (!found) out.push_back({spans[i].name, ms});
    }
  }
  ~StageTimer() {
    for (auto& m : marks) cudaEventDestroy(m.second);
    for (auto& sp : spans) {
      cudaEventDestroy(sp.b);
      cudaEventDestroy(sp.e);
    }
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
  Tuning tune;
  // A shard of one problem (afmm_set_shard): the stored-block M2L and the
  // L2L of the levels at and below shard_level, and the near field, run only
  // over the shard's subtrees (contiguous box ranges); the gather, the M2M,
  // the on-the-fly M2L and the upper levels run whole on every shard, and the
  // potentials of points outside the shard come out as zeros.  Unsharded,
  // these equal levels / lv / near.
  int shard_index = 0, shard_count = 1, shard_level = 0;
  LevelSet levels_m2l;
  LevelView lv_down[kMaxLevels];
  NearView near_own;
};

// Level and box range [k0, k1) of shard `index` of `count` on a tree of
// levels 2..L: the shallowest level with at least four boxes per shard (the
// deepest level when none has), boxes split evenly (a KD tree's boxes of one
// level hold equal point counts).  Returns false when the tree has fewer
// leaves than shards.
inline bool shard_range(int L, int index, int count, int& level, long& k0, long& k1) {
  if (count < 1 || index < 0 || index >= count || L < 2) return false;
  level = L;
  for (int j = 2; j <= L; ++j)
    if ((1L << (2 * j)) >= 4L * count) {
      level = j;
      break;
    }
  const long nb = 1L << (2 * level);
  if (nb < count) return false;
  k0 = nb * index / count;
  k1 = nb * (index + 1) / count;
  return true;
}

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

// ------------------------------------------------ FP64 sweep rows
// The arithmetic of one output of each FP64 sweep, shared by the
// single-problem kernels (fmm.cu) and the fused many-problem kernels (set.cu)
// so both give the same bits.

// Loads of values that may have been written earlier in the same launch (the
// persistent many-problem sweeps): kL2 reads them through L2 (ld.global.cg),
// which other SMs' published stores reach; otherwise an ordinary load.
template <bool kL2>
__device__ __forceinline__ double ld_src(const double* p) {
  if constexpr (kL2) return __ldcg(p);
  else return *p;
}

// M2M (src/AFMM2DTree.cpp:1129-1154): qhat[row] = (L2P_b^T src_b)[row] over
// the row-major L2P copy; src_b = leaf charges, or the concatenated outgoing
// charges of children 0..3.
template <bool kL2 = false>
__device__ __forceinline__ void m2m_row(const LevelView& v, const double* __restrict__ src_all, int leaf, long row) {
  const int b = v.skel_box[row];
  const int r = v.rank[b];
  const int c = (int)(row - v.skel_off[b]);
  const int n = v.node_off[b + 1] - v.node_off[b];
  const double* src = src_all + (leaf ? v.leaf_start[b] : v.node_off[b]);
  const double* P = v.l2p_rm + v.l2p_off[b] + c;  // (i, c) at i*r + c
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int i = 0;
  // (unrolled: more loads in flight; each partial sum keeps its order)
#pragma unroll 4
  for (; i + 3 < n; i += 4) {
    a0 += P[(long)i * r] * ld_src<kL2>(src + i);
    a1 += P[(long)(i + 1) * r] * ld_src<kL2>(src + i + 1);
    a2 += P[(long)(i + 2) * r] * ld_src<kL2>(src + i + 2);
    a3 += P[(long)(i + 3) * r] * ld_src<kL2>(src + i + 3);
  }
  for (; i < n; ++i) a0 += P[(long)i * r] * ld_src<kL2>(src + i);
  v.qhat[row] = (a0 + a1) + (a2 + a3);
}

// M2L (src/AFMM2DTree.cpp:1156-1178): row i of box b sums, slot by slot in
// the reference's order (inner 0..15, outer 0..23), row i of the stored block
// M2L[b][c] (column-major) times the outgoing charges of c.
__device__ __forceinline__ void m2l_row(const LevelView& v, long row) {
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

// L2L (src/AFMM2DTree.cpp:1180-1197): t = (L2P_b yhat_b)[node row g] over the
// column-major L2P, added to the child's incoming potential (node row g of
// level j is skeleton row g of level j+1), or written as the leaf potential.
template <bool kL2 = false>
__device__ __forceinline__ void l2l_row(const LevelView& v, double* __restrict__ child_yhat, double* __restrict__ ys,
                                        int leaf, long g) {
  const int b = v.node_box[g];
  const int r = v.rank[b];
  const int n = v.node_off[b + 1] - v.node_off[b];
  const int i = (int)(g - v.node_off[b]);
  const double* P = v.l2p + v.l2p_off[b] + i;  // (i, c) at c*n + i
  const double* yb = v.yhat + v.skel_off[b];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int c = 0;
#pragma unroll 4
  for (; c + 3 < r; c += 4) {
    a0 += P[(long)c * n] * ld_src<kL2>(yb + c);
    a1 += P[(long)(c + 1) * n] * ld_src<kL2>(yb + c + 1);
    a2 += P[(long)(c + 2) * n] * ld_src<kL2>(yb + c + 2);
    a3 += P[(long)(c + 3) * n] * ld_src<kL2>(yb + c + 3);
  }
  for (; c < r; ++c) a0 += P[(long)c * n] * ld_src<kL2>(yb + c);
  const double t = (a0 + a1) + (a2 + a3);
  if (leaf) ys[v.leaf_start[b] + i] = t;
  else child_yhat[g] += t;
}

// Source slots of leaf b's near field (neighbours 0..7, then the leaf itself),
// fetched by warp 0 in one round of loads instead of a walk by one thread
// (nine dependent neighbour -> leaf lookups): lane s < 9 reads slot s, the
// existing slots keep their order (compacted by a ballot), and a slot's
// offset is the sum of units(count) = ceil(count / UNIT) over the existing
// slots before it.  In lane s: the source leaf c (-1: no neighbour), its
// compacted index m (-1 if none), start, count, offset; in every lane the
// number of existing slots ns and the total of their units.  Warp 0, all 32
// lanes, only.
struct NearSlots {
  long c;
  int m, start, cnt, off, total, ns;
};

template <int UNIT>
__device__ __forceinline__ NearSlots near_slots(const NearView& nv, long b, int lane) {
  NearSlots r;
  r.c = -1;
  r.start = 0;
  r.cnt = 0;
  if (lane < 9) {
    r.c = lane < 8 ? (long)nv.nbr[b * 8 + lane] : b;
    if (r.c >= 0) {
      r.start = nv.leaf_start[r.c];
      r.cnt = nv.leaf_cnt[r.c];
    }
  }
  const bool ok = lane < 9 && r.c >= 0;
  const unsigned valid = __ballot_sync(0xffffffffu, ok);
  const int u = ok ? (r.cnt + UNIT - 1) / UNIT : 0;
  int pre = u;  // inclusive prefix over lanes 0..lane
#pragma unroll
  for (int o = 1; o < 16; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += t;
  }
  r.off = pre - u;
  r.total = __shfl_sync(0xffffffffu, pre, 8);
  r.ns = __popc(valid);
  r.m = ok ? __popc(valid & ((1u << lane) - 1u)) : -1;
  return r;
}

// Near field (src/AFMM2DTree.cpp:1199-1213) of leaf b: neighbours 0..7 and the
// leaf itself, kernel evaluated on the fly.  Run by one CTA of at least
// NT * G threads: all source leaves are staged in shared memory (`smem`:
// 9 * nmax double2 + 9 * nmax double + NT * G double); G groups of NT
// threads split the source leaves (group g takes leaves g, g+G, ...), each
// thread owns one target, and the groups' sums are added in group order.
template <class K>
__device__ __forceinline__ void p2p64_leaf(const NearView& nv, const KernelParams& kp, const double* __restrict__ qs,
                                           double* __restrict__ ys, int NT, int G, long b, unsigned char* smem) {
  __shared__ int s_src[9], s_cnt[9], s_off[10], s_ns;
  const int n = nv.leaf_cnt[b];
  const int s0 = nv.leaf_start[b];
  if (threadIdx.x < 32) {
    const NearSlots sl = near_slots<1>(nv, b, threadIdx.x);
    if (sl.m >= 0) {
      s_src[sl.m] = sl.start;
      s_cnt[sl.m] = sl.cnt;
      s_off[sl.m] = sl.off;
    }
    if (threadIdx.x == 0) {
      s_off[sl.ns] = sl.total;
      s_ns = sl.ns;
    }
  }
  __syncthreads();
  const int ns = s_ns;
  double2* sx = (double2*)smem;
  double* sq = (double*)(sx + 9 * nv.nmax);
  double* red = sq + 9 * nv.nmax;  // G x NT
  for (int m = 0; m < ns; ++m)
    for (int t = threadIdx.x; t < s_cnt[m]; t += blockDim.x) {
      sx[s_off[m] + t] = nv.pts[s_src[m] + t];
      sq[s_off[m] + t] = qs[s_src[m] + t];
    }
  __syncthreads();
  const bool active = (int)threadIdx.x < NT * G;
  const int i = threadIdx.x % NT, g = threadIdx.x / NT;
  double acc = 0.0;
  if (active && i < n) {
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
  if (active) red[g * NT + i] = acc;
  __syncthreads();
  if (active && g == 0 && i < n) {
    double s = ys[s0 + i];
    for (int h = 0; h < G; ++h) s += red[h * NT + i];
    ys[s0 + i] = s;
  }
}

void build_lists(int j, long nbox, int32_t* nbr, int32_t* il, cudaStream_t s);
// map[off[b] + l] = b for l < off[b+1] - off[b]
void fill_box_map(const int32_t* off, long nbox, int32_t* map, cudaStream_t s);
// iperm[perm[i]] = i
void invert_permutation(const int64_t* perm, int n, int32_t* iperm, cudaStream_t s);
// out[t] = pts[ids[t]]
void gather_points(const double2* pts, const int32_t* ids, long n, double2* out, cudaStream_t s);
void m2l_assemble(const LevelView& v, const KernelParams& kp, cudaStream_t s);
// 32-bit fixed-point copy of the stored FP64 blocks (m2l_q, m2l_dec).
void m2l_compress(const LevelView& v, cudaStream_t s);
void l2p_transpose(const LevelView& v, const double* cm, double* rm, cudaStream_t s);
void matvec_fp64(const MatvecPlan& p, const double* q, double* y, cudaStream_t s, StageTimer* tm, int64_t* launches);
// M2L of every level in FP64: the stored blocks (one thread per skeleton row),
// or m2l_apply_otf when no blocks are stored.
void m2l_apply(const MatvecPlan& p, cudaStream_t s);
// M2L of the given levels from the stored blocks, 32-bit fixed point (q32)
// or FP64, FP64 arithmetic, one warp per row chunk.
void m2l_apply_stored(const MatvecPlan& p, const LevelSet& levels, bool q32, cudaStream_t s);
// M2L of the given levels with the entries evaluated on the fly in FP64 (mixed.cu).
void m2l_apply_otf(const MatvecPlan& p, const LevelSet& levels, cudaStream_t s);
// The FP64 sweeps shared by both precisions (leaf charges qs in FP64).
void sweep_m2m(const MatvecPlan& p, const double* qs, cudaStream_t s, int64_t* launches);
void sweep_l2l(const MatvecPlan& p, double* ys, cudaStream_t s, int64_t* launches);

}  // namespace afmm
