// Correctly rounded (to within one rounding of a ~2^-100-accurate value)
// double-precision log and exp for the setup kernels.
//
// The setup (ACA pivoting, L2P, M2L blocks) must see the same kernel entries
// as the reference's host code, whose libm log/exp return the correctly
// rounded result in all but vanishingly rare cases.  These functions evaluate
// in double-double arithmetic and round once:
//  * error-free transformations: TwoSum (Knuth), TwoProduct via FMA, and
//    double-double add / multiply / divide after Dekker (1971);
//  * log(x) = e*ln2 + 2*atanh(s), s = (m-1)/(m+1), x = m*2^e with
//    m in [1/sqrt2, sqrt2): |s| <= 0.1716, 22 odd terms of the atanh series
//    reach 2^-106;
//  * exp(x) = 2^k * exp(r), x = k*ln2 + r, |r| <= ln2/2 (r formed in
//    double-double), exp(r) by its Taylor series to 2^-106 (27 terms).
// ln 2 is carried as the double-double 0x1.62e42fefa39efp-1 + 0x1.abc9e3b39803fp-56.
#pragma once

namespace afmm {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd dd_two_sum(double a, double b) {
  double s = __dadd_rn(a, b);
  double bb = __dsub_rn(s, a);
  double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return dd{s, e};
}

__device__ __forceinline__ dd dd_fast_two_sum(double a, double b) {  // |a| >= |b|
  double s = __dadd_rn(a, b);
  return dd{s, __dsub_rn(b, __dsub_rn(s, a))};
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = dd_two_sum(a.hi, b.hi);
  dd t = dd_two_sum(a.lo, b.lo);
  s.lo = __dadd_rn(s.lo, t.hi);
  s = dd_fast_two_sum(s.hi, s.lo);
  s.lo = __dadd_rn(s.lo, t.lo);
  return dd_fast_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  double p = __dmul_rn(a.hi, b.hi);
  double e = __fma_rn(a.hi, b.hi, -p);
  e = __fma_rn(a.hi, b.lo, e);
  e = __fma_rn(a.lo, b.hi, e);
  return dd_fast_two_sum(p, e);
}

__device__ __forceinline__ dd dd_mul_d(dd a, double b) {
  double p = __dmul_rn(a.hi, b);
  double e = __fma_rn(a.hi, b, -p);
  e = __fma_rn(a.lo, b, e);
  return dd_fast_two_sum(p, e);
}

__device__ __forceinline__ dd dd_div(dd a, dd b) {
  double q1 = __ddiv_rn(a.hi, b.hi);
  dd r = dd_add(a, dd_mul_d(b, -q1));
  double q2 = __ddiv_rn(r.hi, b.hi);
  r = dd_add(r, dd_mul_d(b, -q2));
  double q3 = __ddiv_rn(r.hi, b.hi);
  dd q = dd_fast_two_sum(q1, q2);
  return dd_add(q, dd{q3, 0.0});
}

__device__ __forceinline__ dd dd_ln2() { return dd{0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56}; }

// 1/n for a small integer n as a double-double: h = rn(1/n), l = (1 - h*n)*h
// (the residual 1 - h*n is exact with FMA; l carries it to ~2^-106).
__device__ __forceinline__ dd dd_inv_int(double n) {
  double h = __drcp_rn(n);
  return dd{h, __dmul_rn(__fma_rn(-h, n, 1.0), h)};
}

// log(x) for finite x > 0.
static __device__ __noinline__ double log_cr(double x) {
  int e;
  double m = frexp(x, &e);  // x = m * 2^e, m in [0.5, 1)
  if (m < 0.70710678118654752440) {
    m = __dmul_rn(m, 2.0);
    e -= 1;
  }
  if (m == 1.0 && e == 0) return 0.0;
  dd num = dd_two_sum(m, -1.0);
  dd den = dd_two_sum(m, 1.0);
  dd s = dd_div(num, den);
  dd s2 = dd_mul(s, s);
  // atanh(s)/s = sum_{k>=0} s^(2k)/(2k+1), Horner from the tail
  dd acc = dd_inv_int(43.0);
  for (int k = 20; k >= 0; --k) acc = dd_add(dd_inv_int((double)(2 * k + 1)), dd_mul(acc, s2));
  dd lm = dd_mul(dd_mul_d(s, 2.0), acc);
  dd r = dd_add(dd_mul_d(dd_ln2(), (double)e), lm);
  return __dadd_rn(r.hi, r.lo);
}

// exp(x) for finite x (results that under/overflow follow 2^k scaling).
static __device__ __noinline__ double exp_cr(double x) {
  if (x == 0.0) return 1.0;
  if (x < -745.2) return 0.0;
  if (x > 709.8) return __longlong_as_double(0x7ff0000000000000LL);
  double kf = rint(x * 1.4426950408889634074);
  int k = (int)kf;
  // r = x - k*ln2 in double-double
  dd r = dd_add(dd{x, 0.0}, dd_mul_d(dd_ln2(), -kf));
  // exp(r) = sum r^n / n!, Horner from n = 27
  dd acc{1.0, 0.0};
  for (int n = 27; n >= 1; --n) acc = dd_add(dd{1.0, 0.0}, dd_mul(dd_mul(acc, r), dd_inv_int((double)n)));
  // scale by 2^k in two steps to stay normal where possible
  int k1 = k / 2, k2 = k - k1;
  double hi = __dadd_rn(acc.hi, acc.lo);
  return ldexp(ldexp(hi, k1), k2);
}

}  // namespace afmm
