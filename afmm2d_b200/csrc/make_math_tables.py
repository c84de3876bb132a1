"""Writes math_tables.cuh: the tables of the FP64 matvec logarithm and
exponential (log_tang and exp_tang in fast_math.cuh).

log: for j = 0..128 and F = 1 + j/128: 1/F rounded to double, and ln F split
as hi + lo with hi a multiple of 2^-42 (so that k*ln2_hi + hi is exact for
every double exponent k) and lo = ln F - hi rounded to double; ln 2 = entry
128.
exp: 2^(j/32) for j = 0..31 as hi + lo (hi the correctly rounded double), and
ln2/32 as L1 + L2 with L1 a multiple of 2^-42 (N * L1 exact for |N| < 2^16).
Values are computed with 60-digit decimal arithmetic.

Usage: python make_math_tables.py  (rewrites math_tables.cuh beside this file)
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
        "// Generated by make_math_tables.py.  Do not edit.",
        "// log_tang: breakpoints F = 1 + j/128 (j = 0..128) -- 1/F, and ln F as hi (a",
        "// multiple of 2^-42) + lo.  exp_tang: 2^(j/32) as hi + lo, ln2/32 as L1 + L2.",
        "#pragma once",
        "",
        "namespace afmm {",
        "",
        "static __device__ const double kLogInvF[129] = {",
    ]
    lines += [f"    {v.hex()}," for v in inv]
    lines += ["};", "", "// {hi, lo} of ln F", "static __device__ const double2 kLogLnF[129] = {"]
    lines += [f"    {{{h.hex()}, {lo.hex()}}}," for h, lo in zip(lnhi, lnlo)]
    lines += ["};", "", f"constexpr double kLn2Hi = {lnhi[128].hex()};", f"constexpr double kLn2Lo = {lnlo[128].hex()};"]
    # exp: 2^(j/32) as hi + lo
    lines += ["", "// {hi, lo} of 2^(j/32)", "static __device__ const double2 kExp2J32[32] = {"]
    for j in range(32):
        v = Decimal(2) ** (Decimal(j) / Decimal(32))
        hi = float(v)
        lo = float(v - Decimal(hi))
        lines.append(f"    {{{hi.hex()}, {lo.hex()}}},")
    ln2_32 = Decimal(2).ln() / Decimal(32)
    l1 = Fraction(round(Fraction(ln2_32) * 2 ** 42), 2 ** 42)
    l1_d = float(l1)
    assert Fraction(l1_d) == l1
    l2_d = float(ln2_32 - Decimal(l1.numerator) / Decimal(l1.denominator))
    inv = float(Decimal(32) / Decimal(2).ln())
    lines += ["};", "", f"constexpr double kLn2Over32Hi = {l1_d.hex()};", f"constexpr double kLn2Over32Lo = {l2_d.hex()};",
              f"constexpr double k32OverLn2 = {inv.hex()};", "", "}  // namespace afmm", ""]
    with open(os.path.join(HERE, "math_tables.cuh"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
