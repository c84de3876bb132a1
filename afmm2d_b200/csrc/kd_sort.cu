// K1: KD-tree permutation on the GPU, bit-exact with the reference.
//
// The reference (src/KDTree.cpp:37-142) recursively merge-sorts each segment
// by x, splits it at n/2, merge-sorts each half by y, splits each at half/2,
// and recurses into the four quarters (LB, LT, RB, RT) down to level L; the
// leaf-level call still sorts by x and then each half by y.  Its merge takes
// the right element on ties (src/KDTree.cpp:47), so a sort orders equal keys
// by descending position in the previous order.  Unrolling that tie rule
// through the alternating x/y sorts gives a fixed total order per sort:
//   level-0 x-sort:        (x asc, original index desc)
//   x-sort at level >= 1:  (x asc, y desc, original index desc)
//   every y-sort:          (y asc, x desc, original index asc)
// (with -0.0 == +0.0, as '<' treats them).  Only the membership of each half
// depends on these orders until the last level, so the GPU
//   1. ranks every point once under the three total orders (stable LSD radix
//      sorts of 64-bit order-preserving keys),
//   2. splits the large top-level segments with stable radix multi-splits by
//      segment id over the rank-ordered point sequence, and
//   3. finishes segments of <= kSmallSeg points inside one CTA (bitonic sorts
//      of (sub-segment, rank) keys in shared memory), levels down to L.
#include <algorithm>

#include "afmm_internal.cuh"
#include "kd_sort.cuh"

namespace afmm {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;                     // per lane
constexpr int RS_WARP_TILE = RS_ITEMS * 32;      // 512 consecutive elements per warp
constexpr int RS_TILE = RS_WARPS * RS_WARP_TILE; // 4096 per block

__device__ __forceinline__ uint64_t orderable_key(double d) {
  uint64_t u = (uint64_t)__double_as_longlong(d);
  if (d == 0.0) u = 0;  // -0.0 and +0.0 compare equal
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__global__ void k_make_keys(const double* __restrict__ xy, int n, uint64_t* kx, uint64_t* ky) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    kx[i] = orderable_key(xy[2 * i]);
    ky[i] = orderable_key(xy[2 * i + 1]);
  }
}

// vals[i] = descending ? n-1-i : i
__global__ void k_iota(int32_t* v, int n, int descending) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = descending ? n - 1 - i : i;
}

// keys[i] = (complement ? ~src[vals[i]] : src[vals[i]])
__global__ void k_gather_key64(const uint64_t* __restrict__ src, const int32_t* __restrict__ vals, int n,
                               int complement, uint64_t* keys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    uint64_t k = src[vals[i]];
    keys[i] = complement ? ~k : k;
  }
}

__global__ void k_gather_key32(const int32_t* __restrict__ src, const int32_t* __restrict__ vals, int n,
                               uint64_t* keys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = (uint64_t)(uint32_t)src[vals[i]];
}

// rank[vals[i]] = i
__global__ void k_invert(const int32_t* __restrict__ vals, int n, int32_t* rank) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rank[vals[i]] = i;
}

// Per-block digit histogram; counts laid out digit-major: counts[d*nblk + b].
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t* __restrict__ keys, int n, int shift,
                                                        int bits, uint32_t* counts, int nblk) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += RS_THREADS) h[i] = 0;
  __syncthreads();
  uint64_t mask = (1ull << bits) - 1;
  long base = (long)blockIdx.x * RS_TILE;
  for (int i = threadIdx.x; i < RS_TILE; i += RS_THREADS) {
    long idx = base + i;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & mask], 1u);
  }
  __syncthreads();
  int nd = 1 << bits;
  for (int d = threadIdx.x; d < nd; d += RS_THREADS) counts[(long)d * nblk + blockIdx.x] = h[d];
}

// In-place exclusive scan of m uint32 values with one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_single(uint32_t* a, long m) {
  __shared__ uint32_t part[1024];
  long per = (m + 1023) / 1024;
  long lo = threadIdx.x * per, hi = min(m, lo + per);
  uint32_t s = 0;
  for (long i = lo; i < hi; ++i) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - s;
  for (long i = lo; i < hi; ++i) {
    uint32_t t = a[i];
    a[i] = run;
    run += t;
  }
}

// Stable scatter of one radix pass.  Warp w of a block owns the block's
// elements [w*512, (w+1)*512) and walks them in rounds of 32 consecutive
// elements, so the order (warp, round, lane) is the input order.
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                           const int32_t* __restrict__ vin, uint64_t* kout,
                                                           int32_t* vout, int n, int shift, int bits,
                                                           const uint32_t* __restrict__ offsets, int nblk) {
  __shared__ uint32_t wcnt[RS_WARPS][256];
  __shared__ uint32_t boff[256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t mask = (1ull << bits) - 1;
  for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
  const long base = (long)blockIdx.x * RS_TILE + (long)warp * RS_WARP_TILE;
  uint64_t key[RS_ITEMS];
  int32_t val[RS_ITEMS];
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    long idx = base + r * 32 + lane;
    key[r] = idx < n ? kin[idx] : 0;
    val[r] = idx < n ? vin[idx] : 0;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    long idx = base + r * 32 + lane;
    bool ok = idx < n;
    unsigned vm = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      unsigned d = (unsigned)((key[r] >> shift) & mask);
      unsigned peers = __match_any_sync(vm, d);
      if (lane == __ffs(peers) - 1) wcnt[warp][d] += __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  int nd = 1 << bits;
  for (int d = threadIdx.x; d < nd; d += RS_THREADS) {
    uint32_t run = 0;
    for (int w = 0; w < RS_WARPS; ++w) {
      uint32_t c = wcnt[w][d];
      wcnt[w][d] = run;
      run += c;
    }
    boff[d] = offsets[(long)d * nblk + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ITEMS; ++r) {
    long idx = base + r * 32 + lane;
    bool ok = idx < n;
    unsigned vm = __ballot_sync(0xffffffffu, ok);
    unsigned d = 0, peers = 0, pos = 0;
    if (ok) {
      d = (unsigned)((key[r] >> shift) & mask);
      peers = __match_any_sync(vm, d);
      pos = boff[d] + wcnt[warp][d] + __popc(peers & lt);
    }
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] += __popc(peers);
    __syncwarp();
    if (ok) {
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
  }
}

// After grouping the sequence by segment (keys = segment id), split each
// segment at floor(n_s/2): out_id[p] = 2*s + (position in segment >= floor(n_s/2)).
__global__ void k_split_assign(const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals, int n,
                               const int64_t* __restrict__ seg_start, int32_t* out_id) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = (int)keys[i];
  int64_t st = seg_start[s], len = seg_start[s + 1] - st;
  int side = (i - st) >= len / 2;
  out_id[vals[i]] = 2 * s + side;
}

// ---------------------------------------------------------------- bottom
// One CTA per level-lb segment (<= kSmallSeg points).  Repeats, for levels
// lb..L, the x-split and y-split inside shared memory with bitonic sorts of
// keys (sub-segment << 40 | rank << 12 | slot).
constexpr int BT_THREADS = 1024;

__device__ void bitonic_sort(uint64_t* K, int P) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < P / 2; t += BT_THREADS) {
        int i = 2 * j * (t / j) + (t % j);
        int l = i + j;
        bool up = ((i & k) == 0);
        uint64_t a = K[i], b = K[l];
        if ((a > b) == up) {
          K[i] = b;
          K[l] = a;
        }
      }
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(BT_THREADS) k_kd_bottom(const int32_t* __restrict__ seq,
                                                          const int64_t* __restrict__ seg_start, int lb, int L,
                                                          const int32_t* __restrict__ rank_x0,
                                                          const int32_t* __restrict__ rank_x,
                                                          const int32_t* __restrict__ rank_y, int32_t* perm_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int64_t s0 = seg_start[blockIdx.x];
  const int n = (int)(seg_start[blockIdx.x + 1] - s0);
  int P = 1;
  while (P < n) P <<= 1;
  uint64_t* K = (uint64_t*)smem;                   // P
  int32_t* id = (int32_t*)(K + kSmallSeg);         // n
  int32_t* rx = id + kSmallSeg;                    // n
  int32_t* ry = rx + kSmallSeg;                    // n
  int32_t* sub = ry + kSmallSeg;                   // sub-segment starts, kSmallSeg + 1
  int32_t* half = sub + kSmallSeg + 1;             // half starts, 2*kSmallSeg + 1
  __shared__ int nsub;
  for (int i = threadIdx.x; i < n; i += BT_THREADS) {
    int p = seq[s0 + i];
    id[i] = p;
    rx[i] = (lb == 0) ? rank_x0[p] : rank_x[p];
    ry[i] = rank_y[p];
  }
  if (threadIdx.x == 0) {
    nsub = 1;
    sub[0] = 0;
    sub[1] = n;
  }
  __syncthreads();
  for (int lev = lb; lev <= L; ++lev) {
    const int ns = nsub;
    // x-sort inside each sub-segment
    for (int pos = threadIdx.x; pos < P; pos += BT_THREADS) {
      if (pos < n) {
        int lo = 0, hi = ns;  // largest s with sub[s] <= pos
        while (hi - lo > 1) {
          int mid = (lo + hi) >> 1;
          if (sub[mid] <= pos) lo = mid; else hi = mid;
        }
        // first pass: slots are in input order
        int slot = (lev == lb) ? pos : (int)(K[pos] & 0xFFF);
        K[pos] = ((uint64_t)lo << 40) | ((uint64_t)(uint32_t)rx[slot] << 12) | (uint64_t)slot;
      } else {
        K[pos] = ~0ull;
      }
    }
    __syncthreads();
    bitonic_sort(K, P);
    // halves: sub-segment s of length m splits at floor(m/2)
    for (int s = threadIdx.x; s < ns; s += BT_THREADS) {
      int st = sub[s], m = sub[s + 1] - st;
      half[2 * s] = st;
      half[2 * s + 1] = st + m / 2;
    }
    if (threadIdx.x == 0) half[2 * ns] = n;
    __syncthreads();
    // y-sort inside each half
    for (int pos = threadIdx.x; pos < P; pos += BT_THREADS) {
      if (pos < n) {
        int lo = 0, hi = 2 * ns;  // largest h with half[h] <= pos (empty halves skipped)
        while (hi - lo > 1) {
          int mid = (lo + hi) >> 1;
          if (half[mid] <= pos) lo = mid; else hi = mid;
        }
        int slot = (int)(K[pos] & 0xFFF);
        K[pos] = ((uint64_t)lo << 40) | ((uint64_t)(uint32_t)ry[slot] << 12) | (uint64_t)slot;
      }
    }
    __syncthreads();
    bitonic_sort(K, P);
    if (lev == L) break;
    // quarters: half h of length m splits at floor(m/2)
    for (int h = threadIdx.x; h < 2 * ns; h += BT_THREADS) {
      int st = half[h], m = half[h + 1] - st;
      sub[2 * h] = st;
      sub[2 * h + 1] = st + m / 2;
    }
    if (threadIdx.x == 0) {
      sub[4 * ns] = n;
      nsub = 4 * ns;
      // the level-0 x-key is only used by the first level
    }
    __syncthreads();
    if (lev == lb && lb == 0) {
      for (int i = threadIdx.x; i < n; i += BT_THREADS) rx[i] = rank_x[id[i]];
      __syncthreads();
    }
  }
  for (int pos = threadIdx.x; pos < n; pos += BT_THREADS) perm_out[s0 + pos] = id[(int)(K[pos] & 0xFFF)];
}

__global__ void k_finish_perm(const int32_t* __restrict__ perm32, const double* __restrict__ xy, int n,
                              int64_t* perm, double* xy_sorted) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    int p = perm32[i];
    perm[i] = p;
    if (xy_sorted) {
      xy_sorted[2 * i] = xy[2 * p];
      xy_sorted[2 * i + 1] = xy[2 * p + 1];
    }
  }
}

inline int nblocks(long n, int t) { return (int)((n + t - 1) / t); }

struct RadixCtx {
  uint64_t *k0, *k1;
  int32_t *v0, *v1;
  uint32_t* counts;
  int n;
  cudaStream_t s;
  int64_t* launches;
  // Stable sort of (k0, v0) by key bits [lo, hi); result left in (k0, v0).
  void sort(int lo, int hi) {
    int nblk = nblocks(n, RS_TILE);
    for (int shift = lo; shift < hi; shift += 8) {
      int bits = std::min(8, hi - shift);
      k_rs_hist<<<nblk, RS_THREADS, 0, s>>>(k0, n, shift, bits, counts, nblk);
      k_scan_single<<<1, 1024, 0, s>>>(counts, (long)(1 << bits) * nblk);
      k_rs_scatter<<<nblk, RS_THREADS, 0, s>>>(k0, v0, k1, v1, n, shift, bits, counts, nblk);
      AFMM_LAUNCH_CHECK();
      *launches += 3;
      std::swap(k0, k1);
      std::swap(v0, v1);
    }
  }
};

}  // namespace

// Segment sizes of the KD recursion: level l has 4^l segments in DFS order;
// a segment of n points splits into halves floor(n/2), n - floor(n/2) and
// each half h into floor(h/2), h - floor(h/2) (src/KDTree.cpp:96-114).
std::vector<std::vector<int64_t>> kd_segment_sizes(int64_t N, int L) {
  std::vector<std::vector<int64_t>> sz(L + 1);
  sz[0] = {N};
  for (int l = 0; l < L; ++l) {
    sz[l + 1].reserve(sz[l].size() * 4);
    for (int64_t n : sz[l]) {
      int64_t ln = n / 2, rn = n - ln;
      sz[l + 1].push_back(ln / 2);
      sz[l + 1].push_back(ln - ln / 2);
      sz[l + 1].push_back(rn / 2);
      sz[l + 1].push_back(rn - rn / 2);
    }
  }
  return sz;
}

namespace {

// Device scratch of one KD sort of n points: key and id arrays of n entries
// each, the radix-pass counts (256 per radix tile) and the segment starts
// (starts_cap int64).  kd_sort_device takes it from a DevArena,
// kd_sort_noalloc from the static array below; both run kd_sort_run.
struct KdScratch {
  uint64_t *kx = nullptr, *ky = nullptr, *k0 = nullptr, *k1 = nullptr;
  int32_t *v0 = nullptr, *v1 = nullptr;
  int32_t *rank_x0 = nullptr, *rank_x = nullptr, *rank_y = nullptr;
  int32_t *perm_x0 = nullptr, *perm_x = nullptr, *perm_y = nullptr, *perm32 = nullptr;
  int32_t *seg_of = nullptr, *half_of = nullptr;
  uint32_t* counts = nullptr;
  int64_t* starts = nullptr;
  size_t starts_cap = 0;
};

// Level below which every segment has at most kSmallSeg points (the top
// levels split by radix multi-splits, the rest finish inside one CTA).
int kd_bottom_level(const std::vector<std::vector<int64_t>>& sizes, int L) {
  int lb = 0;
  while (lb < L && *std::max_element(sizes[lb].begin(), sizes[lb].end()) > kSmallSeg) ++lb;
  if (*std::max_element(sizes[lb].begin(), sizes[lb].end()) > kSmallSeg)
    throw Error{AFMM_BAD_ARG, "leaf segments larger than " + std::to_string(kSmallSeg) + " points"};
  return lb;
}

// The KD permutation (src/KDTree.cpp:37-243) with the scratch of `sc`:
// ranks under the three total orders, radix splits of the top levels, CTA
// sorts of the small segments.  Synchronises `s` before returning.
void kd_sort_run(const KdScratch& sc, const double* d_xy, int N, int L, int64_t* d_perm, double* d_xy_sorted,
                 cudaStream_t s, int64_t* launches) {
  const int T = 256;
  RadixCtx rc;
  rc.k0 = sc.k0;
  rc.k1 = sc.k1;
  rc.v0 = sc.v0;
  rc.v1 = sc.v1;
  rc.counts = sc.counts;
  rc.n = N;
  rc.s = s;
  rc.launches = launches;
  const int gb = nblocks(N, T);

  k_make_keys<<<gb, T, 0, s>>>(d_xy, N, sc.kx, sc.ky);
  // (x asc, index desc)
  k_iota<<<gb, T, 0, s>>>(rc.v0, N, 1);
  k_gather_key64<<<gb, T, 0, s>>>(sc.kx, rc.v0, N, 0, rc.k0);
  *launches += 3;
  rc.sort(0, 64);
  AFMM_CUDA(cudaMemcpyAsync(sc.perm_x0, rc.v0, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, s));
  // (x asc, y desc, index desc)
  k_iota<<<gb, T, 0, s>>>(rc.v0, N, 1);
  k_gather_key64<<<gb, T, 0, s>>>(sc.ky, rc.v0, N, 1, rc.k0);
  *launches += 2;
  rc.sort(0, 64);
  k_gather_key64<<<gb, T, 0, s>>>(sc.kx, rc.v0, N, 0, rc.k0);
  *launches += 1;
  rc.sort(0, 64);
  AFMM_CUDA(cudaMemcpyAsync(sc.perm_x, rc.v0, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, s));
  // (y asc, x desc, index asc)
  k_iota<<<gb, T, 0, s>>>(rc.v0, N, 0);
  k_gather_key64<<<gb, T, 0, s>>>(sc.kx, rc.v0, N, 1, rc.k0);
  *launches += 2;
  rc.sort(0, 64);
  k_gather_key64<<<gb, T, 0, s>>>(sc.ky, rc.v0, N, 0, rc.k0);
  *launches += 1;
  rc.sort(0, 64);
  AFMM_CUDA(cudaMemcpyAsync(sc.perm_y, rc.v0, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, s));
  k_invert<<<gb, T, 0, s>>>(sc.perm_x0, N, sc.rank_x0);
  k_invert<<<gb, T, 0, s>>>(sc.perm_x, N, sc.rank_x);
  k_invert<<<gb, T, 0, s>>>(sc.perm_y, N, sc.rank_y);
  *launches += 3;
  AFMM_LAUNCH_CHECK();

  // Top levels: split while segments are larger than kSmallSeg.
  auto sizes = kd_segment_sizes(N, L);
  const int lb = kd_bottom_level(sizes, L);
  if (2 * sizes[lb].size() + 2 > sc.starts_cap) throw Error{AFMM_BAD_ARG, "too many top-level segments"};
  const int32_t* seq = nullptr;  // point ids grouped by level-lb segment
  if (lb == 0) {
    k_iota<<<gb, T, 0, s>>>(sc.perm32, N, 0);
    *launches += 1;
    seq = sc.perm32;
  }
  std::vector<int64_t> h_starts;
  for (int l = 0; l < lb; ++l) {
    size_t ns = sizes[l].size();
    // x-split: group perm_x (perm_x0 at level 0) by segment, split each at n/2.
    AFMM_CUDA(cudaMemcpyAsync(rc.v0, l == 0 ? sc.perm_x0 : sc.perm_x, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice,
                              s));
    if (l == 0) {
      AFMM_CUDA(cudaMemsetAsync(rc.k0, 0, sizeof(uint64_t) * N, s));
    } else {
      k_gather_key32<<<gb, T, 0, s>>>(sc.seg_of, rc.v0, N, rc.k0);
      *launches += 1;
      rc.sort(0, 2 * l);
    }
    h_starts.assign(ns + 1, 0);
    for (size_t i = 0; i < ns; ++i) h_starts[i + 1] = h_starts[i] + sizes[l][i];
    AFMM_CUDA(cudaMemcpyAsync(sc.starts, h_starts.data(), sizeof(int64_t) * (ns + 1), cudaMemcpyHostToDevice, s));
    k_split_assign<<<gb, T, 0, s>>>(rc.k0, rc.v0, N, sc.starts, sc.half_of);
    *launches += 1;
    // y-split: group perm_y by half, split each half at h/2.
    AFMM_CUDA(cudaMemcpyAsync(rc.v0, sc.perm_y, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, s));
    k_gather_key32<<<gb, T, 0, s>>>(sc.half_of, rc.v0, N, rc.k0);
    *launches += 1;
    rc.sort(0, 2 * l + 1);
    h_starts.assign(2 * ns + 1, 0);
    for (size_t i = 0; i < ns; ++i) {
      int64_t ln = sizes[l][i] / 2;
      h_starts[2 * i + 1] = h_starts[2 * i] + ln;
      h_starts[2 * i + 2] = h_starts[2 * i + 1] + (sizes[l][i] - ln);
    }
    AFMM_CUDA(cudaMemcpyAsync(sc.starts, h_starts.data(), sizeof(int64_t) * (2 * ns + 1), cudaMemcpyHostToDevice, s));
    k_split_assign<<<gb, T, 0, s>>>(rc.k0, rc.v0, N, sc.starts, sc.seg_of);
    *launches += 1;
    AFMM_CUDA(cudaStreamSynchronize(s));  // h_starts is reused
    AFMM_LAUNCH_CHECK();
  }
  if (lb > 0) seq = rc.v0;  // grouped by half => grouped by level-lb segment
  size_t nseg = sizes[lb].size();
  h_starts.assign(nseg + 1, 0);
  for (size_t i = 0; i < nseg; ++i) h_starts[i + 1] = h_starts[i] + sizes[lb][i];
  AFMM_CUDA(cudaMemcpyAsync(sc.starts, h_starts.data(), sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice, s));
  size_t smem = (size_t)kSmallSeg * 8 + (size_t)kSmallSeg * 4 * 3 + (size_t)(kSmallSeg + 1) * 4 +
                (size_t)(2 * kSmallSeg + 1) * 4;
  AFMM_CUDA(cudaFuncSetAttribute(k_kd_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int32_t* out32 = (seq == sc.perm32) ? sc.perm_y : sc.perm32;  // perm_y is no longer needed
  k_kd_bottom<<<(int)nseg, BT_THREADS, smem, s>>>(seq, sc.starts, lb, L, sc.rank_x0, sc.rank_x, sc.rank_y, out32);
  k_finish_perm<<<gb, T, 0, s>>>(out32, d_xy, N, d_perm, d_xy_sorted);
  *launches += 2;
  AFMM_LAUNCH_CHECK();
  AFMM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void kd_sort_device(const double* d_xy, int N, int L, int64_t* d_perm, double* d_xy_sorted, cudaStream_t s,
                    int64_t* launches) {
  if ((int64_t)N >= (1LL << 28)) throw Error{AFMM_BAD_ARG, "N must be below 2^28"};
  DevArena tmp;
  KdScratch sc;
  sc.kx = tmp.alloc<uint64_t>(N);
  sc.ky = tmp.alloc<uint64_t>(N);
  sc.k0 = tmp.alloc<uint64_t>(N);
  sc.k1 = tmp.alloc<uint64_t>(N);
  for (int32_t** p : {&sc.v0, &sc.v1, &sc.rank_x0, &sc.rank_x, &sc.rank_y, &sc.perm_x0, &sc.perm_x, &sc.perm_y,
                      &sc.perm32, &sc.seg_of, &sc.half_of})
    *p = tmp.alloc<int32_t>(N);
  sc.counts = tmp.alloc<uint32_t>((size_t)256 * nblocks(N, RS_TILE));
  auto sizes = kd_segment_sizes(N, L);
  sc.starts_cap = 2 * sizes[kd_bottom_level(sizes, L)].size() + 2;
  sc.starts = tmp.alloc<int64_t>(sc.starts_cap);
  kd_sort_run(sc, d_xy, N, L, d_perm, d_xy_sorted, s, launches);
}

// ------------------------------------------------- allocation-free variant
// The KD permutation for callers that cannot allocate device memory.  All
// scratch lives in one file-scope device array (kNoAllocScratchBytes, held by
// every GPU that loads this library until exit); inputs and outputs are the
// caller's.  The kernel sequence is kd_sort_run's; only the scratch comes
// from the array instead of cudaMalloc.
namespace {

// Layout of the scratch for up to kNoAllocMaxPoints points (each part 256-byte
// aligned): 4 x 8-byte keys and 11 x 4-byte ids/ranks per point, the radix
// pass counts, segment starts and the non-finite flag.
constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaPts = (size_t)kNoAllocMaxPoints;
constexpr size_t kNaCountBlocks = (kNaPts + RS_TILE - 1) / RS_TILE;
constexpr size_t kNaStarts = 1024;  // int64 segment starts (needs 2*4^lb + 2 <= 34 here)
constexpr size_t kNaNeed = 4 * al256(kNaPts * 8) + 11 * al256(kNaPts * 4) + al256(256 * kNaCountBlocks * 4) +
                           al256(kNaStarts * 8) + al256(sizeof(int));
static_assert(kNaNeed <= kNoAllocScratchBytes, "scratch array too small for its layout");

static __device__ __align__(256) unsigned char g_kd_scratch[kNoAllocScratchBytes];

// Device address of g_kd_scratch in the current context.  In host code the
// symbol is only a host-side stand-in, so the address is looked up on every
// call with the caller's device current (cheap, and never stale after a
// context is torn down and recreated).
unsigned char* scratch_address() {
  void* p = nullptr;
  AFMM_CUDA(cudaGetSymbolAddress(&p, g_kd_scratch));
  return (unsigned char*)p;
}

__global__ void k_check_finite(const double* __restrict__ xy, int n, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(isfinite(xy[2 * i]) && isfinite(xy[2 * i + 1]))) atomicExch(flag, 1);
}

}  // namespace

void kd_sort_noalloc(const double* d_xy, int N, int L, int64_t* d_perm, double* d_xy_sorted, cudaStream_t s) {
  if (N < 1 || N > kNoAllocMaxPoints)
    throw Error{AFMM_BAD_ARG, "N = " + std::to_string(N) + " outside 1.." + std::to_string(kNoAllocMaxPoints) +
                                  " for the allocation-free permutation"};
  unsigned char* base = scratch_address();
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    unsigned char* p = base + off;
    off += al256(bytes);
    return p;
  };
  KdScratch sc;
  sc.kx = (uint64_t*)carve(kNaPts * 8);
  sc.ky = (uint64_t*)carve(kNaPts * 8);
  sc.k0 = (uint64_t*)carve(kNaPts * 8);
  sc.k1 = (uint64_t*)carve(kNaPts * 8);
  for (int32_t** p : {&sc.v0, &sc.v1, &sc.rank_x0, &sc.rank_x, &sc.rank_y, &sc.perm_x0, &sc.perm_x, &sc.perm_y,
                      &sc.perm32, &sc.seg_of, &sc.half_of})
    *p = (int32_t*)carve(kNaPts * 4);
  sc.counts = (uint32_t*)carve(256 * kNaCountBlocks * 4);
  sc.starts = (int64_t*)carve(kNaStarts * 8);
  sc.starts_cap = kNaStarts;
  int* flag = (int*)carve(sizeof(int));
  const int T = 256, gb = nblocks(N, T);
  // the array keeps the previous call's contents: clear the flag
  AFMM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
  k_check_finite<<<gb, T, 0, s>>>(d_xy, N, flag);
  AFMM_LAUNCH_CHECK();
  int h_flag = 0;
  AFMM_CUDA(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  AFMM_CUDA(cudaStreamSynchronize(s));
  if (h_flag) throw Error{AFMM_BAD_ARG, "a point has a non-finite coordinate"};
  int64_t launches = 0;
  kd_sort_run(sc, d_xy, N, L, d_perm, d_xy_sorted, s, &launches);
}

}  // namespace afmm
