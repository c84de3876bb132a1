// K1: KD-tree permutation (see kd_sort.cu).
#pragma once
#include <stdint.h>

#include <vector>

#include <cuda_runtime.h>

namespace afmm {

// Segments of at most this many points finish inside one CTA.
constexpr int kSmallSeg = 4096;

// Sizes of the KD recursion's segments, level by level, in DFS order.
std::vector<std::vector<int64_t>> kd_segment_sizes(int64_t N, int L);

// d_perm[i] = original index of the i-th sorted point; d_xy_sorted = gathered
// coordinates (interleaved).  Synchronises `s` before returning.
void kd_sort_device(const double* d_xy, int N, int L, int64_t* d_perm, double* d_xy_sorted, cudaStream_t s,
                    int64_t* launches);

// Allocation-free variant for N <= kNoAllocMaxPoints: all scratch lives in a
// file-scope device array of kNoAllocScratchBytes (see kd_sort.cu).
constexpr int kNoAllocMaxPoints = 65536;
constexpr size_t kNoAllocScratchBytes = (size_t)5 << 20;
void kd_sort_noalloc(const double* d_xy, int N, int L, int64_t* d_perm, double* d_xy_sorted, cudaStream_t s);

}  // namespace afmm
