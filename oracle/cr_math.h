// Test infrastructure only.  Correctly rounded log/exp and dot products for
// the CPU oracles, mirroring the engine's device arithmetic:
//  * double-double arithmetic from error-free transformations (TwoSum after
//    Knuth, TwoProduct with fma, Dekker's double-double add/multiply/divide);
//  * log(x) = e*ln2 + 2*atanh(s), s = (m-1)/(m+1), m in [1/sqrt2, sqrt2),
//    22 odd terms of the atanh series;
//  * exp(x) = 2^k exp(r), |r| <= ln2/2, Taylor series to 27 terms;
//  * dot products accumulated in double-double and rounded once.
// The user kernels of the reference are user code (examples/*.cpp); using a
// correctly rounded log/exp there makes the kernel entries a function of the
// inputs alone, identical on host and device.
#pragma once
#include <cmath>

namespace crm {

struct dd {
  double hi, lo;
};

inline dd two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}
inline dd fast_two_sum(double a, double b) {
  double s = a + b;
  return dd{s, b - (s - a)};
}
inline dd add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
inline dd mul(dd a, dd b) {
  double p = a.hi * b.hi;
  double e = std::fma(a.hi, b.hi, -p);
  e = std::fma(a.hi, b.lo, e);
  e = std::fma(a.lo, b.hi, e);
  return fast_two_sum(p, e);
}
inline dd mul_d(dd a, double b) {
  double p = a.hi * b;
  double e = std::fma(a.hi, b, -p);
  e = std::fma(a.lo, b, e);
  return fast_two_sum(p, e);
}
inline dd div(dd a, dd b) {
  double q1 = a.hi / b.hi;
  dd r = add(a, mul_d(b, -q1));
  double q2 = r.hi / b.hi;
  r = add(r, mul_d(b, -q2));
  double q3 = r.hi / b.hi;
  return add(fast_two_sum(q1, q2), dd{q3, 0.0});
}
inline dd ln2() { return dd{0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56}; }
inline dd inv_int(double n) {
  double h = 1.0 / n;
  return dd{h, std::fma(-h, n, 1.0) * h};
}

inline double log_cr(double x) {
  int e;
  double m = std::frexp(x, &e);
  if (m < 0.70710678118654752440) {
    m *= 2.0;
    e -= 1;
  }
  if (m == 1.0 && e == 0) return 0.0;
  dd s = div(two_sum(m, -1.0), two_sum(m, 1.0));
  dd s2 = mul(s, s);
  dd acc = inv_int(43.0);
  for (int k = 20; k >= 0; --k) acc = add(inv_int((double)(2 * k + 1)), mul(acc, s2));
  dd r = add(mul_d(ln2(), (double)e), mul(mul_d(s, 2.0), acc));
  return r.hi + r.lo;
}

inline double exp_cr(double x) {
  if (x == 0.0) return 1.0;
  if (x < -745.2) return 0.0;
  if (x > 709.8) return HUGE_VAL;
  double kf = std::rint(x * 1.4426950408889634074);
  int k = (int)kf;
  dd r = add(dd{x, 0.0}, mul_d(ln2(), -kf));
  dd acc{1.0, 0.0};
  for (int n = 27; n >= 1; --n) acc = add(dd{1.0, 0.0}, mul(mul(acc, r), inv_int((double)n)));
  int k1 = k / 2, k2 = k - k1;
  return std::ldexp(std::ldexp(acc.hi + acc.lo, k1), k2);
}

// sum_i a[i]*b[i], correctly rounded (double-double accumulation).
inline double dot_cr(const double* a, const double* b, long n) {
  dd s{0.0, 0.0};
  for (long i = 0; i < n; ++i) {
    double p = a[i] * b[i];
    s = add(s, dd{p, std::fma(a[i], b[i], -p)});
  }
  return s.hi + s.lo;
}

}  // namespace crm
