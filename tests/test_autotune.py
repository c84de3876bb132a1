"""The autotuner (afmm_autotune): launch parameters timed on the handle's own
problem, kept in the handle and in a cache file keyed by device and problem
structure.  Tuning never changes the FP64 path's bits and keeps the mixed
paths within their tolerance."""
import ctypes

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads
from test_oracle import assert_rel

MIXED_TOL = 1e-6


def test_autotune_rejects_null_handle():
    assert A.lib().afmm_autotune(None, 0, None, None) == 1
    assert A.lib().afmm_get_tuning(None, None, 7) == 1
    assert A.lib().afmm_set_tuning(None, None, 7) == 1


@pytest.mark.gpu
def test_autotune_results_and_cache(tmp_path):
    pts, _, _ = workloads.make("mixture4m", N=65536)
    Q = np.random.default_rng(2).standard_normal((65536, 16))
    a = A.AFMM(65536, 64, 6, pts, kernel="one_over_r")
    a.assemble()
    default = a.tuning()
    assert default["pf_fp64"] == 12288 and default["otf_mixed"] == 0
    y64 = a.computeMatVecProduct(Q[:, 0])
    cache = tmp_path / "tuning.txt"
    tuned, hit = a.autotune(cache=cache)
    assert not hit
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].startswith("dev=") and "|N=65536|" in lines[0]
    assert all(tuned[k] % 16 == 0 for k in ("pf_fp64", "pf_batched"))
    assert tuned["host_pass_cols"] in (8, 16)
    # the FP64 path does not depend on the tuning
    np.testing.assert_array_equal(a.computeMatVecProduct(Q[:, 0]), y64)
    assert_rel(a.computeMatVecProduct(Q[:, 0], precision="mixed"), y64, MIXED_TOL)
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    for c in (0, 9):
        assert_rel(Ym[:, c], a.computeMatVecProduct(Q[:, c]), MIXED_TOL)
    # a second handle of the same problem takes the cached values without timing
    b = A.AFMM(65536, 64, 6, pts, kernel="one_over_r")
    b.assemble()
    again, hit = b.autotune(cache=cache)
    assert hit and again == tuned
    assert len(cache.read_text().splitlines()) == 1


@pytest.mark.gpu
def test_set_tuning_values_and_forms():
    pts, _, _ = workloads.make("uniform1m", N=32768)
    Q = np.random.default_rng(4).standard_normal((32768, 16))
    a = A.AFMM(32768, 64, 10, pts, kernel="log")
    a.assemble()
    y64 = a.computeMatVecProduct(Q[:, 1])
    # every level on the fly, no prefetch, two host passes of 8
    a.set_tuning(pf_fp64=0, pf_batched=0, otf_mixed=(1 << 16) - 1, otf_batched=(1 << 16) - 1, host_pass_cols=8)
    np.testing.assert_array_equal(a.computeMatVecProduct(Q[:, 1]), y64)
    assert_rel(a.computeMatVecProduct(Q[:, 1], precision="mixed"), y64, MIXED_TOL)
    assert_rel(a.computeMatVecProduct(Q, precision="mixed")[:, 1], y64, MIXED_TOL)
    # alternate levels
    a.set_tuning(otf_mixed=0b1010, otf_batched=0b0101, pf_fp64=8192, pf_batched=24576)
    assert_rel(a.computeMatVecProduct(Q[:, 1], precision="mixed"), y64, MIXED_TOL)
    assert_rel(a.computeMatVecProduct(Q, precision="mixed")[:, 1], y64, MIXED_TOL)
    with pytest.raises(A.AFMMError):
        a.set_tuning(pf_fp64=7)
    with pytest.raises(A.AFMMError):
        a.set_tuning(host_pass_cols=17)
    # the transposed m16n8k4 tiles of the 16-column stored M2L: FP64-batched
    # columns still match the FP64 path to rounding, mixed within tolerance
    a.set_tuning(m2l_t16=1, otf_mixed=0, otf_batched=0)
    assert_rel(a.computeMatVecProduct(Q, precision="fp64_batched")[:, 1], y64, 1e-12)
    assert_rel(a.computeMatVecProduct(Q, precision="mixed")[:, 1], y64, MIXED_TOL)
    # seven values (callers older than the eighth) leave the eighth as it is
    a.set_tuning(m2l_tc=1)
    v = np.array(list(a.tuning().values())[:7], np.int64)
    assert A.lib().afmm_set_tuning(a._h, v.ctypes.data_as(ctypes.c_void_p), 7) == 0
    assert a.tuning()["m2l_tc"] == 1
    with pytest.raises(A.AFMMError):
        a.set_tuning(m2l_tc=3)
