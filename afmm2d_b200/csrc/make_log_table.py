"""Writes log_table.cuh: the breakpoint table of the FP64 matvec logarithm
(log_tang in fast_math.cuh).

For j = 0..128 and F = 1 + j/128: 1/F rounded to double, and ln F split as
hi + lo with hi a multiple of 2^-42 (so that k*ln2_hi + hi is exact for every
double exponent k) and lo = ln F - hi rounded to double; ln 2 = entry 128.
ln F is computed with 60-digit decimal arithmetic.

Usage: python make_log_table.py  (rewrites log_table.cuh beside this file)
"""
import os
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 60
HERE = os.path.dirname(os.path.abspath(__file__))


def split_ln(F):
    ln = Decimal(F).ln()
    hi = Fraction(round(Fraction(ln) * 2 ** 42), 2 ** 42)
    hi_d = float(hi)
    assert Fraction(hi_d) == hi  # 42 fraction bits, magnitude < 1: exact in a double
    lo_d = float(Decimal(ln) - Decimal(hi.numerator) / Decimal(hi.denominator))
    return hi_d, lo_d


def main():
    inv, lnhi, lnlo = [], [], []
    for j in range(129):
        F = 1.0 + j / 128.0
        inv.append(1.0 / F)  # IEEE division: correctly rounded
        h, lo = split_ln(F)
        lnhi.append(h)
        lnlo.append(lo)
    lines = [
        "// Generated by make_log_table.py: breakpoints F = 1 + j/128 (j = 0..128) of",
        "// log_tang -- 1/F, and ln F as hi (a multiple of 2^-42) + lo.  Do not edit.",
        "#pragma once",
        "",
        "namespace afmm {",
        "",
        "static __device__ const double kLogInvF[129] = {",
    ]
    lines += [f"    {v.hex()}," for v in inv]
    lines += ["};", "", "// {hi, lo} of ln F", "static __device__ const double2 kLogLnF[129] = {"]
    lines += [f"    {{{h.hex()}, {lo.hex()}}}," for h, lo in zip(lnhi, lnlo)]
    lines += ["};", "", f"constexpr double kLn2Hi = {lnhi[128].hex()};", f"constexpr double kLn2Lo = {lnlo[128].hex()};",
              "", "}  // namespace afmm", ""]
    with open(os.path.join(HERE, "log_table.cuh"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
