/*
 * afmm2d.h -- C ABI of the B200 (sm_100a) AFMM2D engine.
 *
 * Drop-in replacement for the matvec path of the reference AFMM2D library
 * (vaishna77/AFMM2D): y = K q for an N x N kernel matrix K(i,j) over 2-D
 * points, through a uniform KD-tree, ACA skeletonisation of every
 * interaction list, and M2M / M2L / L2L / near-field sweeps.  All compute
 * runs on one GPU; there is no CPU fallback.  Plain pointers and sizes only.
 *
 * Reference interface each entry point replaces:
 *   afmm_create           AFMM::AFMM(int N, int MinParticlesInLeaf, int TOL_POW,
 *                         Eigen::MatrixXd& loc)       include/AFMM2D.hpp:28,
 *                         src/AFMM2D.cpp:3-39 (KD sort, tree, lists)
 *   afmm_assemble         AFMM::assemble()            include/AFMM2D.hpp:29,
 *                         src/AFMM2D.cpp:41-44 (getNodes + assemble_M2L)
 *   afmm_matvec           AFMM::computeMatVecProduct(Eigen::VectorXd)
 *                         include/AFMM2D.hpp:30, src/AFMM2D.cpp:46-65
 *   afmm_eval_error       AFMM::evaluateError()       include/AFMM2D.hpp:31,
 *                         src/AFMM2D.cpp:67-74, src/AFMM2DTree.cpp:1227-1236
 *   afmm_get_permutation  AFMM::sorted_Properties     include/AFMM2D.hpp:25
 *   afmm_get_sorted_locations  AFMM::sorted_Locations include/AFMM2D.hpp:24
 *   afmm_get_nlevels      AFMM::nLevels               include/AFMM2D.hpp:19
 *   afmm_get_leaves       FMM2DTree::NumberOfParticlesInLeaves / boxNumbers
 *                         include/AFMM2DTree.hpp:34-35
 *   afmm_get_lists        FMM2DBox::neighborNumbers / innerNumbers /
 *                         outerNumbers               include/AFMM2DBox.hpp:17-19
 *   afmm_get_ranks, afmm_get_skeletons, afmm_get_charge_points, afmm_get_l2p
 *                         FMM2DBox::incoming_checkPoints / incoming_chargePoints
 *                         / L2P                      include/AFMM2DBox.hpp:25-35
 *   afmm_destroy          AFMM::~AFMM()               include/AFMM2D.hpp:32
 * The user kernel userkernel::getMatrixEntry (include/kernel.hpp:58) is
 * selected by `kernel_id` (see afmm_kernel_id); new kernels are added as
 * device functors.
 *
 * Errors: every call returns an afmm_status; afmm_last_error() gives a
 * message.  Where the reference aborts or has undefined behaviour the engine
 * returns an error instead (nLevels < 2, non-finite coordinates), and a box
 * whose ACA rank is 0 contributes no far field (the reference crashes there).
 *
 * Threading: a handle owns one CUDA stream; calls on one handle must not
 * overlap; distinct handles are independent.
 */
#ifndef AFMM2D_B200_H
#define AFMM2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AFMM_OK = 0,
  AFMM_BAD_ARG = 1,       /* invalid argument, e.g. N/M giving fewer than 2 levels */
  AFMM_OOM = 2,           /* device allocation failed */
  AFMM_CUDA_ERR = 3,      /* a CUDA call failed */
  AFMM_TIMEOUT = 4,       /* a bounded device wait gave up */
  AFMM_NUMERIC = 5,       /* non-finite values where finite ones are required */
  AFMM_NOT_ASSEMBLED = 6, /* matvec before assemble */
  AFMM_NO_DEVICE = 7      /* no CUDA device of compute capability 10.x */
} afmm_status;

/* Kernels (userkernel::getMatrixEntry, include/kernel.hpp:58).  Ids 0..3 are
 * built in; ids AFMM_KERNEL_USER_FIRST .. + AFMM_KERNEL_USER_COUNT - 1 are
 * user kernels registered with afmm_register_kernel. */
#define AFMM_KERNEL_USER_FIRST 16
#define AFMM_KERNEL_USER_COUNT 64
typedef enum {
  AFMM_KERNEL_ONE_OVER_R_SCALED = 0, /* R<a ? R/a : a/R  (examples/testAFMM2D.cpp:9-20) */
  AFMM_KERNEL_LOG = 1,               /* log r with diagonal convention (examples/tutorial.cpp:22-35) */
  AFMM_KERNEL_ONE_OVER_R = 2,        /* 1/r, 0 at r=0 */
  AFMM_KERNEL_GAUSSIAN = 3           /* exp(-r^2/p), p = kparams[0] (default 0.01) */
} afmm_kernel_id;

typedef enum {
  AFMM_PREC_FP64 = 0,        /* plain FP64 apply (stored operators), column by column */
  AFMM_PREC_MIXED = 1,       /* FP32 near field (FP64 for close pairs), far field in FP64
                                arithmetic on 32-bit fixed-point M2L blocks */
  AFMM_PREC_FP64_BATCHED = 2 /* FP64 throughout, 8 or 16 columns per pass on the FP64 tensor
                                cores; agrees with AFMM_PREC_FP64 to FP64 rounding (the
                                summation order differs) */
} afmm_precision;

/* Storage of the M2L blocks K(R_b, R_c) (src/AFMM2DTree.cpp:1070-1097). */
typedef enum {
  AFMM_M2L_AUTO = 0,      /* store them when they fit in device memory (default) */
  AFMM_M2L_STORE = 1,     /* always store them (AFMM_OOM if they do not fit) */
  AFMM_M2L_ON_THE_FLY = 2 /* never store them: every matvec evaluates the entries in FP64 */
} afmm_m2l_storage;

/* Layout of the `loc` array given to afmm_create. */
typedef enum {
  AFMM_LOC_COLMAJOR = 0,   /* N x 2 column-major, as Eigen::MatrixXd loc(N,2) */
  AFMM_LOC_INTERLEAVED = 1 /* x0,y0,x1,y1,... */
} afmm_loc_layout;

typedef struct afmm_handle afmm_handle;

/* Builds the KD-tree permutation, leaf layout and interaction lists on the GPU.
 * nLevels = (unsigned)(log(N/M)/log(4)) with integer N/M (src/AFMM2D.cpp:7);
 * nLevels < 2 is rejected with AFMM_BAD_ARG.  kparams may be NULL. */
afmm_status afmm_create(int N, int min_particles_in_leaf, int tol_pow, const double* loc, int loc_layout,
                        int kernel_id, const double* kparams, int nkparams, afmm_handle** out);

/* ACA skeletonisation of every box (levels L..2), L2P, and M2L blocks. */
afmm_status afmm_assemble(afmm_handle* h);

/* Setup files.  No reference counterpart: the reference keeps the setup only
 * in memory, per box (FMM2DBox members, include/AFMM2DBox.hpp:25-35, filled
 * by src/AFMM2DTree.cpp:1009-1097), so every process repeats the ACA.
 * afmm_save writes an assembled handle's KD permutation, sorted points and,
 * per level, ranks, skeletons, pivot columns and L2P operators to a
 * versioned binary file with a digest; afmm_load rebuilds an assembled
 * handle from it on the current device (lists, row tables and M2L blocks are
 * recomputed from the file's contents), skipping the KD sort and the ACA.
 * The loaded handle's matvecs have the same bits as the saved handle's.  A
 * file that is truncated, corrupted, of another version or inconsistent is
 * rejected with AFMM_BAD_ARG before any device work. */
afmm_status afmm_save(afmm_handle* h, const char* path);
afmm_status afmm_load(const char* path, afmm_handle** out);

/* M2L storage policy (afmm_m2l_storage), before afmm_assemble.  No reference
 * counterpart: the reference always stores the blocks in std::maps
 * (src/AFMM2DTree.cpp:1070-1097), which at 16M points and TOL 12 needs
 * ~190 GB.  Without stored blocks the M2L entries are evaluated on the fly in
 * FP64 (the matvec's fast FP64 kernel form) by every precision; results
 * agree with the stored blocks to FP64 rounding.  Sets need stored blocks. */
afmm_status afmm_set_m2l_storage(afmm_handle* h, int mode);
/* 1 when the assembled handle stores its M2L blocks. */
afmm_status afmm_get_m2l_stored(afmm_handle* h, int* stored);
/* Whether assembly also keeps a 32-bit fixed-point copy of the stored M2L
 * blocks for AFMM_PREC_MIXED (on by default, when it fits in device memory),
 * before afmm_assemble.  No reference counterpart (the reference keeps FP64
 * blocks only, src/AFMM2DTree.cpp:1070-1097).  Each block carries a
 * power-of-two scale; its entries are stored as 32-bit integers of that
 * scale, within 2^-31 of the block's largest entry, and applied in FP64
 * arithmetic: half the bytes of the FP64 blocks.  AFMM_PREC_FP64 and
 * AFMM_PREC_FP64_BATCHED always apply the FP64 blocks.  Mode 2 also keeps
 * the copy as byte planes for the exact integer tcgen05 M2L (tuning value
 * m2l_tc = 2; about 1.3x the fixed-point bytes more). */
afmm_status afmm_set_m2l_fixed_point(afmm_handle* h, int on);
/* Launch plan of the ACA kernel for every level, before afmm_assemble: CTAs
 * per box (a thread-block cluster of 1, 2, 4, 8 or 16; 0 = the planner's
 * choice) and CTAs per SM (1: full shared-memory budget, 2: half; 0 = the
 * planner's choice).  Ranks, skeletons and L2P do not depend on it; only the
 * setup time does (afmm_get_setup_phases reports the time and cluster size
 * of every level).  No reference counterpart. */
afmm_status afmm_set_aca_plan(afmm_handle* h, int cluster, int ctas_per_sm);
/* 1 when the assembled handle keeps the fixed-point copy. */
afmm_status afmm_get_m2l_fixed_point(afmm_handle* h, int* stored);

/* y = K q for nrhs right-hand sides.  q and y are N x nrhs, column j at
 * offset j*ld (ld >= N), in the caller's ORIGINAL point order.
 * mem_device = 0: host pointers (copied in and out); 1: device pointers.
 * precision: afmm_precision. */
afmm_status afmm_matvec(afmm_handle* h, const double* q, double* y, int nrhs, int64_t ld, int precision,
                        int mem_device);

/* Relative 2-norm error of the last FP64 matvec (its last RHS) against a direct FP64
 * evaluation over `nsample` leaf boxes chosen with `seed` (all leaves when
 * nsample <= 0).  Reproducible, unlike src/AFMM2D.cpp:68. */
afmm_status afmm_eval_error(afmm_handle* h, int nsample, uint64_t seed, double* rel_err);

/* perm[i] = original index of the i-th sorted point (sorted_Properties). */
afmm_status afmm_get_permutation(afmm_handle* h, int64_t* perm);
/* Sorted locations, interleaved x,y (sorted_Locations). */
afmm_status afmm_get_sorted_locations(afmm_handle* h, double* xy);
afmm_status afmm_get_nlevels(afmm_handle* h, int* nlevels);
/* The construction parameters: i5 = [N, MinParticlesInLeaf, TOL_POW,
 * nLevels, kernel id]; kparam (may be NULL) = the kernel parameter
 * (AFMM::N, MinParticlesInLeaf, TOL_POW, nLevels, include/AFMM2D.hpp:16-19). */
afmm_status afmm_get_params(afmm_handle* h, int* i5, double* kparam);
/* Leaf counts in KD (DFS) order and the DFS -> quadtree box-number map, 4^L each. */
afmm_status afmm_get_leaves(afmm_handle* h, int32_t* counts, int32_t* box_numbers);
/* Lists of one level (4^level boxes): nbr[8], inner[16], outer[24] per box, -1 = none. */
afmm_status afmm_get_lists(afmm_handle* h, int level, int32_t* nbr, int32_t* inner, int32_t* outer);
/* Ranks of the 4^level boxes of a level (after assemble). */
afmm_status afmm_get_ranks(afmm_handle* h, int level, int32_t* ranks);
/* Skeletons (incoming check points) of all boxes of a level, concatenated in box
 * order; *count receives the total.  ids may be NULL to query the count. */
afmm_status afmm_get_skeletons(afmm_handle* h, int level, int32_t* ids, int64_t* count);
/* Pivot columns (incoming charge points) likewise. */
afmm_status afmm_get_charge_points(afmm_handle* h, int level, int32_t* ids, int64_t* count);
/* L2P of box k at a level: rows x cols, written row-major (out may be NULL). */
afmm_status afmm_get_l2p(afmm_handle* h, int level, int k, int32_t* rows, int32_t* cols, double* out);

/* Per-stage device times (ms) of the last matvec and setup, when profiling is
 * on.  names/values arrays of capacity `cap`; *n receives the count.  Stages
 * on the handle's stream are the intervals between consecutive marks; in a
 * batched pass the near field runs on a second stream beside the far field,
 * so its span is the separate "p2p_kernel" entry and "p2p" is the far
 * field's wait for it.  afmm_set_profiling(h, 2) profiles with the near
 * field run after the far field on the handle's stream (same results), so
 * that "p2p" is the near-field kernel's own duration. */
afmm_status afmm_set_profiling(afmm_handle* h, int on);
afmm_status afmm_get_stage_times(afmm_handle* h, int cap, const char** names, double* ms, int* n);
/* Setup wall times in seconds: [create, assemble]. */
afmm_status afmm_get_setup_times(afmm_handle* h, double* t2);
/* Counts of the assembled structure: [nlevels, N, sum ranks, stored L2P entries,
 * stored M2L entries, near-field kernel evaluations, far-field (M2L) entries]. */
/* Wall-clock seconds of the assemble phases: ACA kernels ("aca"), L2P solves
 * ("l2p"), M2L block evaluation ("m2l_blocks"), row-major L2P copy and mixed
 * setup ("transpose_mixed"), sizes, allocations and row tables
 * ("tables_alloc", of which the M2L block allocation "m2l_cudamalloc"),
 * per-level host preparation ("level_prep"), the rest of the per-level ACA
 * call -- scratch allocation, rank offsets ("aca_alloc_other"), then the ACA
 * time of each level ("aca_levelJ");
 * names stay valid for the handle's lifetime.
 * Replaces the reference's omp_get_wtime prints around assemble
 * (examples/testAFMM2D.cpp:56-84). */
afmm_status afmm_get_setup_phases(afmm_handle* h, int cap, const char** names, double* secs, int* n);
afmm_status afmm_get_counts(afmm_handle* h, int64_t* c7);
/* Number of kernels this library launched since the handle was created. */
afmm_status afmm_get_launch_count(afmm_handle* h, int64_t* n);
/* The CUDA stream (cudaStream_t) the handle launches on. */
afmm_status afmm_get_stream(afmm_handle* h, void** stream);

/* Evaluates the kernel on n point pairs (host arrays, interleaved x,y):
 * out[t] = K(xy1[t], xy2[t]) with box-size parameter a (2^-nLevels) and
 * kernel parameter `param`.  mode 0: the setup arithmetic (operation order of
 * the reference, correctly rounded log/exp); 1: the FP64 matvec form; 2: the
 * FP32 form.  Replaces no reference interface (a diagnostic of
 * userkernel::getMatrixEntry, include/kernel.hpp:58). */
afmm_status afmm_kernel_eval(int kernel_id, double a, double param, int64_t n, const double* xy1, const double* xy2,
                             double* out, int mode);

/* Measures this device's FP64 and FP32 fused-multiply-add throughput (TFLOP/s,
 * 2 flops per FMA) with a register-only kernel of ~50 ms each: the roofline
 * denominators of the compute-bound kernels.  Replaces no reference interface. */
afmm_status afmm_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops);

/* Measures this device's FP64 tensor throughput (mma.sync m8n8k4, the tiles
 * of the batched sweeps, M2L and FP64 near field), its FP64 FMA throughput,
 * and both issued together (TFLOP/s; a total no higher than either alone
 * means one shared FP64 datapath): the denominators of the FP64-tile
 * kernels.  Replaces no reference interface. */
afmm_status afmm_measure_fp64_pipes(double* dmma_tflops, double* dfma_tflops, double* both_tflops);

/* Sharding one problem over several GPUs (or processes): every shard holds
 * the whole assembled problem (each process builds it; setup is
 * deterministic, so the operators are identical), and afmm_set_shard(h,
 * index, count) makes the handle's matvecs compute only the potentials of
 * shard `index`'s points -- the points of its subtrees: the boxes [k0, k1) of
 * the shallowest level with at least four boxes per shard, split evenly
 * (afmm_shard_range) -- and write zeros for every other point, so that the
 * sum of the shards' outputs (an all-reduce) is the whole product, bit for
 * bit.  Per shard the M2L (stored blocks), the L2L at and below that level
 * and the near field run over its subtrees only; the gather, the M2M, the
 * upper levels and the on-the-fly M2L run whole.  After afmm_assemble;
 * count = 1 restores the whole problem.  No reference counterpart (the
 * reference is single-process, src/AFMM2DTree.cpp:1099-1225); handles in a
 * set may not be sharded.  afmm_shard_range needs no device. */
afmm_status afmm_set_shard(afmm_handle* h, int index, int count);
afmm_status afmm_get_shard(afmm_handle* h, int* index, int* count, int* level);
afmm_status afmm_shard_range(int nlevels, int index, int count, int* level, int64_t* k0, int64_t* k1);

/* KD-tree permutation without any device allocation.  It has no counterpart
 * in the reference; it computes the same permutation as afmm_create /
 * afmm_get_permutation.  For callers that cannot allocate GPU memory: a
 * process whose device memory is already reserved by another framework's
 * caching allocator, a service that must hold a fixed, declared footprint, or
 * a loop that cannot afford a cudaMalloc/cudaFree pair per call (cudaFree
 * synchronises the whole device).  xy (N interleaved x,y), perm (N int64) and
 * xy_sorted (2N doubles, may be NULL) are device pointers owned by the caller;
 * stream is a cudaStream_t (NULL: the default stream).  The call is
 * synchronous: it reads a validity flag back from the device and returns
 * after the stream has completed the work.  Limit: 1 <= N <= 65,536 points
 * (AFMM_BAD_ARG beyond).  Scratch is one static device array of 5 MiB that
 * every GPU loading this library keeps until the process exits; each call
 * looks up its address in the current context.  All calls share that array,
 * so calls that overlap on the GPU (other threads or streams) race and must
 * be serialised by the caller. */
afmm_status afmm_kd_permutation_noalloc(int N, int min_particles_in_leaf, const double* xy, int64_t* perm,
                                        double* xy_sorted, void* stream);

/* Autotuner.  No reference counterpart (the reference has no launch
 * parameters; its M2L loop is uniform over levels, src/AFMM2DTree.cpp:1156-1178).
 * afmm_autotune times, on the handle's own problem with CUDA events, the
 * launch parameters `what` selects (bit 0: L2 prefetch windows of the
 * stored-block M2L kernels; bit 1: per level, stored blocks or entries on
 * the fly in the mixed paths; bit 2: pass width of host-pointer batched
 * calls; bit 3: form of the 16-column stored M2L (FP64 tiles or tcgen05
 * integer products); bit 4: tcgen05 or
 * mma.sync near field of 16-column mixed passes; 0 = all) and keeps the
 * fastest in the handle.  With a cache_path
 * (may be NULL), a line keyed by the device name and the problem's structure
 * (N, M, levels, kernel, TOL_POW, storage, sum of ranks, M2L entries) is
 * reused when present (*from_cache = 1) and appended otherwise.  The FP64
 * path's results do not depend on the tuning; the mixed paths' stay within
 * their tolerance.  The handle must be assembled.
 * afmm_get_tuning / afmm_set_tuning read or set the first n (n >= 7) of the 8 values
 * v = [prefetch window of the one-column M2L (bytes), prefetch window of the
 * batched M2L (bytes), on-the-fly level mask of the one-column mixed path
 * (bit t = level t + 2), the same for batched mixed passes, host pass width
 * (0 = automatic), 16-column stored M2L on transposed m16n8k4 tiles (1) or
 * on 8x8x4 tiles (0), 16-column mixed near field on tcgen05 tiles (1) or on
 * mma.sync tiles (0), 16-column mixed stored M2L on tcgen05 with exact
 * integer products from byte planes of the fixed-point blocks (2), on
 * tcgen05 TF32 tiles (1: an FP32 far field, outside the mixed tolerance on
 * deep trees) or on FP64 tiles (0)]; values past n are left
 * unchanged by afmm_set_tuning.  A tcgen05 kernel whose bounded wait gives up
 * makes the matvec return AFMM_TIMEOUT. */
afmm_status afmm_autotune(afmm_handle* h, int what, const char* cache_path, int* from_cache);
afmm_status afmm_get_tuning(afmm_handle* h, int64_t* v, int n);
afmm_status afmm_set_tuning(afmm_handle* h, const int64_t* v, int n);

/* Number of device allocations (cudaMalloc) this library has made in the
 * process so far, over all handles and sets.  No reference counterpart: a
 * diagnostic that lets a caller check that a call allocated nothing. */
afmm_status afmm_get_device_alloc_count(int64_t* n);

/* Registers a user kernel: the reference's plug-in point, a user-defined
 * userkernel::getMatrixEntry (include/kernel.hpp:23,58; defined out of line
 * in examples/testAFMM2D.cpp:9-20), becomes a kernel functor compiled in the
 * user's own CUDA translation unit.  That unit includes afmm2d_kernel.cuh and
 * writes AFMM_REGISTER_KERNEL(id, Functor), which instantiates every stage
 * that evaluates the kernel (ACA, L2P, M2L blocks, near fields, on-the-fly
 * M2L, sets, diagnostics) for the functor and calls this function with the
 * table of their launchers when the unit's library is loaded.  kernel_id in
 * AFMM_KERNEL_USER_FIRST ..; table_bytes and abi_version must match this
 * library's headers.  Afterwards the id is accepted by afmm_create,
 * afmm_kernel_eval and afmm_load like a built-in id. */
afmm_status afmm_register_kernel(int kernel_id, const void* table, size_t table_bytes, int abi_version);
/* Name of a built-in or registered kernel (AFMM_BAD_ARG for unknown ids). */
afmm_status afmm_kernel_name(int kernel_id, const char** name);

afmm_status afmm_destroy(afmm_handle* h);

/* ---- many independent problems in one call -------------------------------
 * No single counterpart in the reference, which applies one problem per AFMM
 * object (AFMM::computeMatVecProduct, include/AFMM2D.hpp:30); a set replaces
 * a loop of that call over many objects.  afmm_set_create takes n assembled
 * handles on the current device with one kernel id (the handles stay owned
 * by the caller and must outlive the set) and records, once, a CUDA graph in
 * which every stage of the FP64 matvec is one fused launch over all problems
 * (gather; the M2M of every level as one persistent up-sweep; M2L of all
 * levels; the L2L of every level as one persistent down-sweep; near field;
 * scatter).  In a sweep, work items wait on the device, each for at most
 * two seconds, until the level they read is complete; a wait that gives up
 * makes afmm_set_matvec return AFMM_TIMEOUT (the output is then incomplete;
 * the set stays usable).  afmm_set_matvec replays it: q and y hold the
 * problems' charges / potentials back to back in handle order (problem p at
 * offsets[p] .. offsets[p+1], each in its own original point order), host or
 * device memory.  Each problem's result has the same bits as its own FP64
 * afmm_matvec.  The set uses the handles' FP64 work buffers: do not run a
 * set and one of its handles concurrently. */
typedef struct afmm_set afmm_set;
afmm_status afmm_set_create(afmm_handle* const* handles, int n, afmm_set** out);
afmm_status afmm_set_matvec(afmm_set* s, const double* q, double* y, int mem_device);
/* offsets: n + 1 entries (prefix of the problems' N). */
afmm_status afmm_set_get_offsets(afmm_set* s, int64_t* offsets);
/* Fused launches recorded in the graph per matvec, and graph launches so far. */
afmm_status afmm_set_get_launches(afmm_set* s, int* launches_per_matvec, int64_t* graph_launches);
/* Device milliseconds per stage of the last afmm_set_matvec (events recorded
 * inside the graph between stages); names stay valid until the next call. */
afmm_status afmm_set_get_stage_times(afmm_set* s, int cap, const char** names, double* ms, int* n);
afmm_status afmm_set_get_stream(afmm_set* s, void** stream);
/* Test hook for the sweeps' time limit: adds `margin` (>= 0) to every row
 * count that a sweep's item waits for, so with margin > 0 no wait can be
 * satisfied and the next afmm_set_matvec returns AFMM_TIMEOUT after the limit;
 * 0 (the default) restores normal operation.  Re-records the graph. */
afmm_status afmm_set_sweep_wait_margin(afmm_set* s, int margin);
afmm_status afmm_set_destroy(afmm_set* s);
const char* afmm_set_last_error(afmm_set* s);

const char* afmm_status_string(afmm_status s);
const char* afmm_last_error(afmm_handle* h);
/* Library version string. */
const char* afmm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* AFMM2D_B200_H */
