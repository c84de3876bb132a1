// Test infrastructure only (never linked into the product).
//
// Driver translation unit for the reference AFMM2D library, compiled from the
// reference's unmodified src/*.cpp against the Eigen-API shim in shim/.  It
// supplies the user-defined kernel (userkernel::getMatrixEntry,
// include/kernel.hpp:58) for the four kernels of this project and exposes the
// reference's public classes (AFMM, FMM2DTree) through a small C API so that
// Python tests and the CPU baseline can drive them with ctypes.
//
// Kernels (same ids as the product's kernel registry):
//   0  one over r, scaled:  R < a ? R/a : a/R        (examples/testAFMM2D.cpp:9-20)
//   1  log with the diagonal convention:             (examples/tutorial.cpp:22-35)
//        R2 < 1e-10 -> 0;  R2 < a^2 -> 0.5*R2*log(R2)/a/a;  else 0.5*log(R2)
//   2  1/r with 0 at r = 0
//   3  Gaussian exp(-R2/p), p = kernel parameter (0.01 by default)
// log and exp are correctly rounded (cr_math.h), so the entries are a
// function of the coordinates alone, as on the device.
//   101  the log kernel exactly as examples/tutorial.cpp:22-35 writes it,
//        with the host libm's log (not correctly rounded): the stock kernel,
//        for measuring how far the reference's own output moves with it.
#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>

#include "AFMM2D.hpp"
#include "cr_math.h"

static int g_kernel_id = 1;
static double g_kparam = 0.01;

double userkernel::getMatrixEntry(const unsigned i, const unsigned j) {
  pts2D r1 = particles_X[i];
  pts2D r2 = particles_X[j];
  double dx = r1.x - r2.x;
  double dy = r1.y - r2.y;
  double R2 = dx * dx + dy * dy;
  switch (g_kernel_id) {
    case 0: {
      double R = sqrt(R2);
      return (R < a) ? R / a : a / R;
    }
    case 1:
      if (R2 < 1e-10) return 0.0;
      if (R2 < a * a) return 0.5 * R2 * crm::log_cr(R2) / a / a;
      return 0.5 * crm::log_cr(R2);
    case 2: {
      if (R2 == 0.0) return 0.0;
      double R = sqrt(R2);
      return 1.0 / R;
    }
    case 101:
      if (R2 < 1e-10) return 0.0;
      if (R2 < a * a) return 0.5 * R2 * log(R2) / a / a;
      return 0.5 * log(R2);
    default:
      return crm::exp_cr(-R2 / g_kparam);
  }
}

namespace {
struct RefHandle {
  AFMM* afmm;
  double t_create, t_assemble;
};
double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

// xy: N points, interleaved (x0,y0,x1,y1,...).
void* ref_create(int N, int M, int tol_pow, const double* xy, int kernel_id, double kparam) {
  g_kernel_id = kernel_id;
  g_kparam = kparam;
  Eigen::MatrixXd loc(N, 2);
  for (int j = 0; j < N; ++j) {
    loc(j, 0) = xy[2 * j];
    loc(j, 1) = xy[2 * j + 1];
  }
  RefHandle* h = new RefHandle();
  double t0 = now();
  // The AFMM object is never deleted: its destructor frees arrays that the
  // reference's sort_KDTree already freed (src/KDTree.cpp:202-203 vs
  // src/AFMM2D.cpp:77-78).
  h->afmm = new AFMM(N, M, tol_pow, loc);
  h->t_create = now() - t0;
  h->t_assemble = 0.0;
  return h;
}

void ref_assemble(void* hv) {
  RefHandle* h = (RefHandle*)hv;
  g_kernel_id = g_kernel_id;  // kernel selection is process-global
  double t0 = now();
  h->afmm->assemble();
  h->t_assemble = now() - t0;
}

void ref_matvec(void* hv, const double* q, double* y) {
  RefHandle* h = (RefHandle*)hv;
  int N = h->afmm->N;
  Eigen::VectorXd b(N);
  for (int i = 0; i < N; ++i) b(i) = q[i];
  Eigen::VectorXd out = h->afmm->computeMatVecProduct(b);
  for (int i = 0; i < N; ++i) y[i] = out(i);
}

int ref_nlevels(void* hv) { return (int)((RefHandle*)hv)->afmm->nLevels; }

void ref_timings(void* hv, double* t) {
  RefHandle* h = (RefHandle*)hv;
  t[0] = h->t_create;
  t[1] = h->t_assemble;
}

// sorted_Properties[i] = original index of the i-th sorted point.
void ref_get_permutation(void* hv, int64_t* perm) {
  AFMM* a = ((RefHandle*)hv)->afmm;
  for (int i = 0; i < a->N; ++i) perm[i] = (int64_t)a->sorted_Properties[i];
}

void ref_get_sorted_locations(void* hv, double* xy) {
  AFMM* a = ((RefHandle*)hv)->afmm;
  std::memcpy(xy, a->sorted_Locations, sizeof(double) * 2 * (size_t)a->N);
}

// Leaf counts in DFS (KD) order and the DFS -> quadtree box-number map.
void ref_get_leaves(void* hv, int32_t* counts, int32_t* box_numbers) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[t->nLevels];
  for (int k = 0; k < n; ++k) {
    counts[k] = t->NumberOfParticlesInLeaves[k];
    box_numbers[k] = t->boxNumbers[k];
  }
}

// Interaction lists of one level: 8 neighbour, 16 inner, 24 outer slots.
void ref_get_lists(void* hv, int level, int32_t* nbr, int32_t* inner, int32_t* outer) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[level];
  for (int k = 0; k < n; ++k) {
    const FMM2DBox& b = t->tree[level][k];
    for (int s = 0; s < 8; ++s) nbr[8 * k + s] = b.neighborNumbers[s];
    for (int s = 0; s < 16; ++s) inner[16 * k + s] = b.innerNumbers[s];
    for (int s = 0; s < 24; ++s) outer[24 * k + s] = b.outerNumbers[s];
  }
}

// Ranks of all boxes at one level (after assemble).
void ref_get_ranks(void* hv, int level, int32_t* ranks) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[level];
  for (int k = 0; k < n; ++k) ranks[k] = (int32_t)t->tree[level][k].incoming_checkPoints.size();
}

// Skeleton (incoming check points, sorted-point ids) of all boxes at a level,
// concatenated in box order; returns the total count.
long ref_get_skeletons(void* hv, int level, int32_t* ids) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[level];
  long c = 0;
  for (int k = 0; k < n; ++k)
    for (int id : t->tree[level][k].incoming_checkPoints) {
      if (ids) ids[c] = id;
      ++c;
    }
  return c;
}

// Pivot columns (incoming charge points) of all boxes at a level.
long ref_get_charge_points(void* hv, int level, int32_t* ids) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[level];
  long c = 0;
  for (int k = 0; k < n; ++k)
    for (int id : t->tree[level][k].incoming_chargePoints) {
      if (ids) ids[c] = id;
      ++c;
    }
  return c;
}

// L2P of one box: rows x cols, written row-major; returns rows*cols.
long ref_get_l2p(void* hv, int level, int k, int32_t* rows, int32_t* cols, double* out) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  const Eigen::MatrixXd& m = t->tree[level][k].L2P;
  *rows = (int32_t)m.rows();
  *cols = (int32_t)m.cols();
  if (out)
    for (long i = 0; i < m.rows(); ++i)
      for (long j = 0; j < m.cols(); ++j) out[i * m.cols() + j] = m(i, j);
  return m.rows() * m.cols();
}

// Per-stage vectors after a matvec: outgoing (M2M) and incoming_potential
// (after M2L + L2L) of every box at a level, concatenated in box order.
long ref_get_stage(void* hv, int level, int which, double* out) {
  FMM2DTree* t = ((RefHandle*)hv)->afmm->afmm2dtree;
  int n = t->nBoxesPerLevel[level];
  long c = 0;
  for (int k = 0; k < n; ++k) {
    const FMM2DBox& b = t->tree[level][k];
    const Eigen::VectorXd& v = (which == 0) ? b.outgoing_charges : b.incoming_potential;
    for (long i = 0; i < v.size(); ++i) {
      if (out) out[c] = v(i);
      ++c;
    }
  }
  return c;
}

int ref_abs_is_double(void) { return abs(0.5) == 0.5 ? 1 : 0; }

int ref_num_threads(void) { return omp_get_max_threads(); }
}
