// afmm2d_compat.hpp -- header-only C++ mirror of the reference's class AFMM
// (include/AFMM2D.hpp:14-33) over the C ABI in afmm2d.h.
//
// The reference's user code
//
//     AFMM* afmm = new AFMM(N, MinParticlesInLeaf, TOL_POW, loc);
//     afmm->assemble();
//     Eigen::VectorXd y = afmm->computeMatVecProduct(b);
//     afmm->evaluateError();
//
// compiles unchanged against this header when Eigen is available (the
// reference's kernel, userkernel::getMatrixEntry, becomes the `kernel`
// argument, default log).  Without Eigen the same members take and return
// std::vector<double>.  Errors throw afmm2d::Error.
#ifndef AFMM2D_COMPAT_HPP
#define AFMM2D_COMPAT_HPP

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "afmm2d.h"

#if defined(__has_include)
#if __has_include(<Eigen/Dense>) && !defined(AFMM2D_COMPAT_NO_EIGEN)
#include <Eigen/Dense>
#define AFMM2D_COMPAT_EIGEN 1
#endif
#endif

namespace afmm2d {

struct Error : std::runtime_error {
  afmm_status status;
  Error(afmm_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(afmm_status s, afmm_handle* h) {
  if (s != AFMM_OK) throw Error(s, std::string(afmm_status_string(s)) + ": " + afmm_last_error(h));
}

}  // namespace afmm2d

class AFMM {
 public:
  int N;
  int MinParticlesInLeaf;
  int TOL_POW;
  unsigned nLevels;
  std::vector<double> sorted_Locations;   // interleaved x, y (include/AFMM2D.hpp:24)
  std::vector<double> sorted_Properties;  // original index of each sorted point (:25)

  // loc: N x 2 column-major (Eigen::MatrixXd layout) unless interleaved.
  AFMM(int N_, int M_, int tol_pow, const double* loc, int kernel = AFMM_KERNEL_LOG,
       bool interleaved = false, double kparam = 0.01)
      : N(N_), MinParticlesInLeaf(M_), TOL_POW(tol_pow) {
    init(loc, interleaved ? AFMM_LOC_INTERLEAVED : AFMM_LOC_COLMAJOR, kernel, kparam);
  }
#ifdef AFMM2D_COMPAT_EIGEN
  AFMM(int N_, int M_, int tol_pow, Eigen::MatrixXd& loc, int kernel = AFMM_KERNEL_LOG,
       double kparam = 0.01)
      : N(N_), MinParticlesInLeaf(M_), TOL_POW(tol_pow) {
    init(loc.data(), AFMM_LOC_COLMAJOR, kernel, kparam);
  }
  Eigen::VectorXd computeMatVecProduct(const Eigen::VectorXd& b, afmm_precision p = AFMM_PREC_FP64) {
    Eigen::VectorXd y(N);
    afmm2d::check(afmm_matvec(h_, b.data(), y.data(), 1, N, p, 0), h_);
    return y;
  }
#endif
  AFMM(const AFMM&) = delete;
  AFMM& operator=(const AFMM&) = delete;
  ~AFMM() { afmm_destroy(h_); }

  void assemble() { afmm2d::check(afmm_assemble(h_), h_); }

  std::vector<double> computeMatVecProduct(const std::vector<double>& b, afmm_precision p = AFMM_PREC_FP64) {
    std::vector<double> y(N);
    afmm2d::check(afmm_matvec(h_, b.data(), y.data(), 1, N, p, 0), h_);
    return y;
  }

  // Seeded error of the last FP64 matvec over `nsample` leaves (the reference
  // prints the error of one random leaf, src/AFMM2D.cpp:67-74).
  double evaluateError(int nsample = 1, uint64_t seed = 0) {
    double e = 0;
    afmm2d::check(afmm_eval_error(h_, nsample, seed, &e), h_);
    std::printf("\nPerforming error calculation in box: \nerr: %g\n", e);
    return e;
  }

  // Setup files (afmm_save / afmm_load): a later process skips the KD sort
  // and the ACA; the loaded object's matvecs have the saved one's bits.
  void save(const std::string& path) { afmm2d::check(afmm_save(h_, path.c_str()), h_); }
  static AFMM* load(const std::string& path) {
    afmm_handle* h = nullptr;
    afmm2d::check(afmm_load(path.c_str(), &h), nullptr);
    return new AFMM(h);
  }
  // Launch parameters timed on this problem (afmm_autotune); cache may be NULL.
  bool autotune(const char* cache = nullptr) {
    int hit = 0;
    afmm2d::check(afmm_autotune(h_, 0, cache, &hit), h_);
    return hit != 0;
  }

  afmm_handle* handle() const { return h_; }

 private:
  afmm_handle* h_ = nullptr;
  explicit AFMM(afmm_handle* h) : h_(h) {
    int v[5] = {0, 0, 0, 0, 0};
    afmm2d::check(afmm_get_params(h_, v, nullptr), h_);
    N = v[0];
    MinParticlesInLeaf = v[1];
    TOL_POW = v[2];
    nLevels = (unsigned)v[3];
    read_sorted();
  }
  void read_sorted() {
    std::vector<int64_t> perm(N);
    afmm2d::check(afmm_get_permutation(h_, perm.data()), h_);
    sorted_Properties.assign(perm.begin(), perm.end());
    sorted_Locations.resize(2 * (size_t)N);
    afmm2d::check(afmm_get_sorted_locations(h_, sorted_Locations.data()), h_);
  }
  void init(const double* loc, int layout, int kernel, double kparam) {
    afmm2d::check(afmm_create(N, MinParticlesInLeaf, TOL_POW, loc, layout, kernel, &kparam, 1, &h_), nullptr);
    int L = 0;
    afmm2d::check(afmm_get_nlevels(h_, &L), h_);
    nLevels = (unsigned)L;
    read_sorted();
  }
};

#endif  // AFMM2D_COMPAT_HPP
