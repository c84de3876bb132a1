"""The FP64 matvec logarithm and exponential (log_tang, exp_tang in
afmm2d_b200/csrc/fast_math.cuh): the CPU tests restate their steps in Python
(exact FMA through fractions) with the generated tables (math_tables.cuh) and
check them against the correctly rounded functions; the GPU tests check the
library's own FP64 log and Gaussian kernel entries against the setup's
correctly rounded ones."""
import math
import os
import re
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "afmm2d_b200", "csrc")


def _table():
    s = open(os.path.join(CSRC, "math_tables.cuh")).read()
    inv_block = s[s.index("kLogInvF[129]"):s.index("};")]
    inv = [float.fromhex(v) for v in re.findall(r"(-?0x[0-9a-f.]+p[-+]\d+)", inv_block)]
    ln_block = s[s.index("kLogLnF[129]"):]
    ln_block = ln_block[:ln_block.index("};")]
    pairs = re.findall(r"\{(-?0x[0-9a-f.]+p[-+]\d+), (-?0x[0-9a-f.]+p[-+]\d+)\}", ln_block)
    ln = [(float.fromhex(a), float.fromhex(b)) for a, b in pairs]
    l2h = float.fromhex(re.search(r"kLn2Hi = (\S+);", s).group(1))
    l2l = float.fromhex(re.search(r"kLn2Lo = (\S+);", s).group(1))
    assert len(inv) == 129 and len(ln) == 129
    return inv, ln, l2h, l2l


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def log_tang(x, T):
    """The device function's operations in IEEE double, one rounding each."""
    inv, ln, l2h, l2l = T
    bits = np.float64(x).view(np.uint64).item()
    hx, lx = bits >> 32, bits & 0xffffffff
    frac_hi = hx & 0x000fffff
    j = (frac_hi + 0x1000) >> 13
    m = np.uint64(((frac_hi | 0x3ff00000) << 32) | lx).view(np.float64).item()
    F = np.uint64((0x3ff00000 + (j << 13)) << 32).view(np.float64).item()
    kd = float(((hx >> 20) & 0x7ff) - 1023)
    f = m - F
    hi = _fma(kd, l2h, ln[j][0])
    u0 = f * inv[j]
    u1 = _fma(-u0, F, f) * inv[j]
    q = _fma(1.0 / 7.0, u0, -1.0 / 6.0)
    q = _fma(q, u0, 1.0 / 5.0)
    q = _fma(q, u0, -0.25)
    q = _fma(q, u0, 1.0 / 3.0)
    q = _fma(q, u0, -0.5)
    p = q * (u0 * u0)
    lo = (_fma(kd, l2l, ln[j][1]) + u1) + p
    return hi + (u0 + lo)


def _cr_log(x):
    getcontext().prec = 50
    return float(Decimal(x).ln())


def _ulps(a, b):
    return abs(a - b) / math.ulp(b) if b != 0 else abs(a)


def test_table_is_consistent():
    inv, ln, l2h, l2l = _table()
    getcontext().prec = 50
    assert ln[0] == (0.0, 0.0) and ln[128] == (l2h, l2l)
    for j in range(129):
        F = 1.0 + j / 128.0
        assert inv[j] == 1.0 / F
        assert Fraction(ln[j][0]) * 2 ** 42 == int(Fraction(ln[j][0]) * 2 ** 42)  # multiple of 2^-42
        err = Decimal(ln[j][0]) + Decimal(ln[j][1]) - Decimal(F).ln()
        assert abs(err) < Decimal(2) ** -95


def test_restated_log_within_one_ulp():
    T = _table()
    rng = np.random.default_rng(3)
    xs = list(np.exp(rng.uniform(math.log(1e-10), math.log(8.0), 3000)))   # R2 of the matvec's pairs
    xs += list(np.exp(rng.uniform(-700, 700, 1000)))                       # the whole normal range
    xs += [1.0 + d for d in rng.uniform(-2 ** -7, 2 ** -7, 500)]          # both sides of 1
    xs += [np.nextafter(1.0, 0.0), np.nextafter(1.0, 2.0), 2.0, 0.5, 1e-10, 2.0 ** -1022]
    xs += [1.0 + (j + 0.5) / 128 * (1 + s * 2 ** -40) for j in range(128) for s in (-1, 1)]  # rounding edges of j
    worst = 0.0
    for x in xs:
        x = float(x)
        worst = max(worst, _ulps(log_tang(x, T), _cr_log(x)))
    assert worst <= 1.0, worst


@pytest.mark.gpu
def test_device_log_kernel_entries_within_one_ulp():
    import afmm2d_b200 as A
    rng = np.random.default_rng(8)
    n = 200000
    xy1 = rng.uniform(0, 1, (n, 2))
    # separations along x only: R2 = dx * dx is the same double in both forms
    # (with a y term, the FP64 form's fused multiply-add can round R2
    # differently, which moves log(R2) near R2 = 1 by many of its tiny ulps)
    xy2 = xy1.copy()
    xy2[:, 0] += np.exp(rng.uniform(np.log(1e-4), np.log(1.4), n)) * rng.choice([-1.0, 1.0], n)
    a = 2.0 ** -14  # every pair takes the 0.5 log(R2) branch: the value is half the log, exactly
    fast = A.kernel_eval("log", a, xy1, xy2, mode="fp64")
    exact = A.kernel_eval("log", a, xy1, xy2, mode="exact")
    dx, dy = xy1[:, 0] - xy2[:, 0], xy1[:, 1] - xy2[:, 1]
    far = dx * dx + dy * dy >= a * a
    ul = np.abs(fast[far] - exact[far]) / np.spacing(np.abs(exact[far]))
    assert far.sum() > 0.9 * n
    assert ul.max() <= 1.0


def _exp_table():
    s = open(os.path.join(CSRC, "math_tables.cuh")).read()
    blk = s[s.index("kExp2J32[32]"):]
    blk = blk[:blk.index("};")]
    pairs = re.findall(r"\{(-?0x[0-9a-f.]+p[-+]\d+), (-?0x[0-9a-f.]+p[-+]\d+)\}", blk)
    S = [(float.fromhex(a), float.fromhex(b)) for a, b in pairs]
    c = {k: float.fromhex(re.search(k + r" = (\S+);", s).group(1)) for k in ("kLn2Over32Hi", "kLn2Over32Lo", "k32OverLn2")}
    assert len(S) == 32
    return S, c


def exp_tang(x, T):
    """The device function's operations in IEEE double, one rounding each."""
    S, c = T
    shifter = 6755399441055744.0
    t = _fma(x, c["k32OverLn2"], shifter)
    nd = t - shifter
    N = int(nd)
    r = _fma(-nd, c["kLn2Over32Hi"], x)
    r = _fma(-nd, c["kLn2Over32Lo"], r)
    hi, lo = S[N & 31]
    q = _fma(1.0 / 720.0, r, 1.0 / 120.0)
    q = _fma(q, r, 1.0 / 24.0)
    q = _fma(q, r, 1.0 / 6.0)
    q = _fma(q, r, 0.5)
    p = _fma(q * r, r, r)
    v = hi + _fma(hi, p, _fma(lo, p, lo))
    return 0.0 if x < -708.0 else v * 2.0 ** (N >> 5)


def _cr_exp(x):
    getcontext().prec = 50
    return float(Decimal(x).exp())


def test_exp_table_is_consistent():
    S, c = _exp_table()
    getcontext().prec = 50
    for j in range(32):
        err = Decimal(S[j][0]) + Decimal(S[j][1]) - (Decimal(2) ** (Decimal(j) / 32))
        assert abs(err) < Decimal(2) ** -104
    l1 = Fraction(c["kLn2Over32Hi"])
    assert l1 * 2 ** 42 == int(l1 * 2 ** 42)
    assert abs(Decimal(c["kLn2Over32Hi"]) + Decimal(c["kLn2Over32Lo"]) - Decimal(2).ln() / 32) < Decimal(2) ** -95


def test_restated_exp_within_one_ulp():
    T = _exp_table()
    rng = np.random.default_rng(4)
    xs = list(-np.exp(rng.uniform(math.log(1e-12), math.log(700.0), 3000)))  # the Gaussian's -R2/param
    xs += list(rng.uniform(-708.0, 709.0, 1000))
    xs += [0.0, -0.0, 1e-300, -1e-300, -708.0, 709.0, math.log(2) / 64, -math.log(2) / 64]
    xs += [(n + 0.5) * math.log(2) / 32 * (1 + s * 2 ** -45) for n in range(-40, 40) for s in (-1, 1)]
    worst = 0.0
    for x in xs:
        x = float(x)
        worst = max(worst, _ulps(exp_tang(x, T), _cr_exp(x)))
    assert worst <= 1.0, worst
    assert exp_tang(-708.5, T) == 0.0


@pytest.mark.gpu
def test_device_gaussian_entries_within_bound():
    """FP64 Gaussian entries exp(R2 * (-1/param)) against the setup's correctly
    rounded exp(-R2/param), x = R2/param: the argument carries two roundings
    (of -1/param and of the product), relative 2^-52 at most, which moves
    exp(-x) by at most 2|x| ulps; with the exp's own ulp the bound is
    1 + 2|x| ulps."""
    import afmm2d_b200 as A
    rng = np.random.default_rng(9)
    n = 200000
    xy1 = rng.uniform(0, 1, (n, 2))
    xy2 = xy1.copy()
    xy2[:, 0] += np.exp(rng.uniform(np.log(1e-5), np.log(0.5), n)) * rng.choice([-1.0, 1.0], n)
    param = 0.01
    fast = A.kernel_eval("gaussian", 2.0 ** -7, xy1, xy2, mode="fp64", param=param)
    exact = A.kernel_eval("gaussian", 2.0 ** -7, xy1, xy2, mode="exact", param=param)
    dx = xy1[:, 0] - xy2[:, 0]
    x = dx * dx / param
    ok = exact > 1e-300
    ul = np.abs(fast[ok] - exact[ok]) / np.spacing(exact[ok])
    assert ok.sum() > 0.5 * n
    assert np.all(ul <= 1.0 + 2.0 * x[ok] + 1e-9), float(np.max(ul - 2.0 * x[ok]))
    assert np.median(ul) == 0.0


def test_committed_tables_match_their_generator(tmp_path):
    """math_tables.cuh is exactly what make_math_tables.py writes."""
    import importlib.util
    import shutil
    src = os.path.join(CSRC, "make_math_tables.py")
    shutil.copy(src, tmp_path / "make_math_tables.py")
    spec = importlib.util.spec_from_file_location("make_math_tables_copy", tmp_path / "make_math_tables.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.main()  # writes beside the copy
    assert (tmp_path / "math_tables.cuh").read_text() == open(os.path.join(CSRC, "math_tables.cuh")).read()
