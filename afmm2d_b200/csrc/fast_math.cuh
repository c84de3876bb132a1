// FP64 natural logarithm and exponential for the matvec's kernel entries
// (near field, FP64 tensor-tile near field, on-the-fly M2L); the setup keeps
// the correctly rounded log_cr / exp_cr of exact_math.cuh.
//
// log_tang:
// Method: P. T. P. Tang, "Table-driven implementation of the logarithm
// function in IEEE floating-point arithmetic", ACM TOMS 16(4), 1990.
// x = 2^k m with m in [1, 2); F = 1 + j/128 is the breakpoint nearest m (j
// from the top mantissa bits, rounded), f = m - F exactly (|f| <= 2^-8), and
//   ln x = (k ln2_hi + lnF_hi) + (u0 + (k ln2_lo + lnF_lo + u1 + p(u0))),
// where u0 + u1 = f/F (u0 = f * (1/F), u1 from its exact FMA residual), and
// p(u) = ln(1 + u) - u = -u^2/2 + u^3/3 - ... - u^6/6 + u^7/7 (truncation
// below 2^-59 relative for |u| <= 2^-8).  ln2_hi and lnF_hi are multiples of
// 2^-42, so the first bracket is exact for every exponent; near x = 1 from
// either side it is exactly zero (j = 0, k = 0, or j = 128, k = -1), so small
// results keep full relative accuracy.  About 16 FP64 operations and two
// table loads (math_tables.cuh, L1-resident).  Error within about one ulp for
// positive normal x (tests compare it with the correctly rounded log); zero,
// subnormal and non-finite inputs give an unspecified value without a trap,
// which the kernel functors select away (their R2 < 1e-10 branch).
#pragma once

#include "math_tables.cuh"

namespace afmm {

__device__ __forceinline__ double log_tang(double x) {
  const int hx = __double2hiint(x), lx = __double2loint(x);
  const int frac_hi = hx & 0x000fffff;
  const int j = (frac_hi + 0x1000) >> 13;  // round(128 (m - 1)), 0..128
  const double m = __hiloint2double(frac_hi | 0x3ff00000, lx);
  const double F = __hiloint2double(0x3ff00000 + (j << 13), 0);  // 1 + j/128 (2 for j = 128)
  // k = biased exponent - 1023, as a double without an integer conversion
  const double kd = __hiloint2double(0x43300000, (hx >> 20) & 0x7ff) - 4503599627371519.0;  // - (2^52 + 1023)
  const double f = m - F;
  const double inv = __ldg(&kLogInvF[j]);
  const double2 lnF = __ldg(&kLogLnF[j]);
  const double hi = fma(kd, kLn2Hi, lnF.x);  // exact
  const double u0 = f * inv;
  const double u1 = fma(-u0, F, f) * inv;    // the residual f - u0 F is exact
  double q = fma(1.0 / 7.0, u0, -1.0 / 6.0);
  q = fma(q, u0, 1.0 / 5.0);
  q = fma(q, u0, -0.25);
  q = fma(q, u0, 1.0 / 3.0);
  q = fma(q, u0, -0.5);
  const double p = q * (u0 * u0);
  const double lo = (fma(kd, kLn2Lo, lnF.y) + u1) + p;
  return hi + (u0 + lo);
}

// exp_tang: P. T. P. Tang, "Table-driven implementation of the exponential
// function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989.
// x = (32 m + j) ln2/32 + r with N = 32 m + j the integer nearest x 32/ln2,
// j = N mod 32, |r| <= ln2/64 (r = x - N L1 - N L2, N L1 exact);
//   exp(x) = 2^m (S_hi + (S_lo + S p(r))),  S = 2^(j/32) = S_hi + S_lo,
// p(r) = exp(r) - 1 by its Taylor polynomial to r^6 (truncation below
// 2^-58).  About 13 FP64 operations and one table load.  Error within about
// one ulp for x in [-708, 709.7] (tests compare it with the correctly rounded
// exp); below -708 it returns 0 (the true value is under 2^-1021).
__device__ __forceinline__ double exp_tang(double x) {
  const double shifter = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
  const double t = fma(x, k32OverLn2, shifter);
  const int N = __double2loint(t);
  const double nd = t - shifter;
  double r = fma(-nd, kLn2Over32Hi, x);  // exact
  r = fma(-nd, kLn2Over32Lo, r);
  const double2 S = __ldg(&kExp2J32[N & 31]);
  double q = fma(1.0 / 720.0, r, 1.0 / 120.0);
  q = fma(q, r, 1.0 / 24.0);
  q = fma(q, r, 1.0 / 6.0);
  q = fma(q, r, 0.5);
  const double p = fma(q * r, r, r);
  const double v = S.x + fma(S.x, p, fma(S.y, p, S.y));
  const double scale = __hiloint2double(((N >> 5) + 1023) << 20, 0);  // 2^m
  return x < -708.0 ? 0.0 : v * scale;
}

}  // namespace afmm
