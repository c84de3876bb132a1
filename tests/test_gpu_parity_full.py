"""Parity at the workloads' full sizes and at the configurations the smaller
tests do not reach: the 1,048,576-point log problem at TOL 10 against the
reference's own output (committed fixture), interaction lists of 8- and
9-level trees against the restated recurrence, many-problem sets against the
oracle, the 64-right-hand-side Gaussian workload, the tutorial's stock log
kernel, boxes of ACA rank 0, the fixed-point M2L blocks and the pipelined
host-pointer path.  All calls go through the C ABI (libafmm2d.so)."""
import hashlib
import os

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads
from oracle_lib import Oracle, RefLib, dense_rows, kd_total_order
from test_oracle import assert_rel

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MIXED_TOL = 1e-6  # relative 2-norm of a mixed-precision result vs the FP64 path / the oracle


def sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def test_uniform1m_full_size_vs_reference():
    """N = 1,048,576 uniform, log, M = 64, TOL 10 (L = 7): permutation, leaf
    layout, lists of all levels, ranks, skeletons and pivot columns bit-exact
    against the reference run at full size (fixture from
    tests/golden/make_uniform1m_fixture.py); potentials within 10^-TOL of the
    reference's at 32,768 sampled rows."""
    f = np.load(os.path.join(HERE, "golden", "full_size", "uniform1m_log_tol10.npz"))
    pts, q, p = workloads.make("uniform1m")
    a = A.AFMM(len(pts), p["M"], p["tol"], pts, kernel=p["kernel"])
    assert a.nLevels == int(f["L"]) == 7
    perm = a.permutation()
    assert sha(perm, "<i8") == str(f["perm_sha"])
    np.testing.assert_array_equal(perm, kd_total_order(pts, a.nLevels))
    c, b = a.leaves()
    np.testing.assert_array_equal(c, f["counts"])
    np.testing.assert_array_equal(b, f["boxnum"])
    for lev in range(1, a.nLevels + 1):
        assert sha(np.concatenate(a.lists(lev)), "<i4") == str(f[f"lists_sha{lev}"]), lev
    a.assemble()
    for lev in range(2, a.nLevels + 1):
        np.testing.assert_array_equal(a.ranks(lev), f[f"rank{lev}"])
        assert sha(a.skeletons(lev), "<i4") == str(f[f"skel_sha{lev}"]), lev
        assert sha(a.charge_points(lev), "<i4") == str(f[f"cpiv_sha{lev}"]), lev
    y = a.computeMatVecProduct(q)
    rows = f["rows"]
    assert_rel(y[rows], f["y_rows"], 10.0 ** (-p["tol"]))
    # the FP64 tensor-core path on the same problem, 8 columns (column 0 = q)
    Q = np.random.default_rng(12).standard_normal((len(pts), 8))
    Q[:, 0] = q
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    assert_rel(Yb[rows, 0], f["y_rows"], 10.0 ** (-p["tol"]))


@pytest.mark.parametrize("L", [8, 9])
def test_lists_deep_levels_vs_recurrence(L):
    """Lists of every level of an L-level tree (N = 2 * 4^L points, M = 1)
    against the oracle's restatement of the reference's parent-to-child
    recurrence (src/AFMM2DTree.cpp:65-967), plus the permutation."""
    N = 2 * 4 ** L
    pts = np.random.default_rng(L).uniform(0, 1, (N, 2))
    a = A.AFMM(N, 1, 6, pts, kernel="log")
    assert a.nLevels == L
    o = Oracle(pts, 1, 6, "log")
    assert o.L == L
    np.testing.assert_array_equal(a.permutation(), o.permutation())
    for lev in range(1, L + 1):
        for got, want in zip(a.lists(lev), o.lists(lev)):
            np.testing.assert_array_equal(got, want)


def test_set_problems_vs_oracle():
    """Problems of a many-problem set (log, M = 32, TOL 8), each applied
    through the fused set graph, against the oracle's own matvec."""
    probs, p = workloads.many_problems(count=5, nmax=32768)
    hs = []
    for pts, _ in probs:
        h = A.AFMM(len(pts), p["M"], p["tol"], pts, kernel=p["kernel"])
        h.assemble()
        hs.append(h)
    st = A.AFMMSet(hs)
    ys = st.matvec([qk for _, qk in probs])
    for k in range(len(probs)):
        pts, qk = probs[k]
        o = Oracle(pts, p["M"], p["tol"], p["kernel"])
        o.assemble()
        assert_rel(ys[k], o.matvec(qk), 10.0 ** (-p["tol"]))
    st.close()


def test_gauss_64rhs_vs_oracle_65k():
    """The 64-right-hand-side Gaussian workload (exp(-r^2/0.01), M = 64,
    TOL 8) at N = 65,536: mixed (four 16-column passes) and FP64-batched
    columns against the oracle's FP64 matvec."""
    pts, Q, p = workloads.make("gauss1m", N=65536)
    assert Q.shape == (65536, 64)
    a = A.AFMM(len(pts), p["M"], p["tol"], pts, kernel=p["kernel"])
    a.assemble()
    o = Oracle(pts, p["M"], p["tol"], p["kernel"])
    o.assemble()
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    for c in (0, 15, 16, 40, 63):
        yo = o.matvec(np.ascontiguousarray(Q[:, c]))
        assert_rel(Ym[:, c], yo, MIXED_TOL)
        assert_rel(Yb[:, c], yo, 10.0 ** (-p["tol"]))


def test_gauss_64rhs_full_size():
    """N = 1,048,576, 64 right-hand sides: mixed and FP64-batched columns
    against the plain FP64 path (sampled columns), and linearity."""
    pts, Q, p = workloads.make("gauss1m")
    N = len(pts)
    a = A.AFMM(N, p["M"], p["tol"], pts, kernel=p["kernel"])
    a.assemble()
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    for c in (0, 17, 63):
        y64 = a.computeMatVecProduct(Q[:, c])
        assert_rel(Ym[:, c], y64, MIXED_TOL)
        assert_rel(Yb[:, c], y64, 1e-12)
    y01 = a.computeMatVecProduct(Q[:, 0] + Q[:, 1], precision="mixed")
    assert_rel(y01, Ym[:, 0] + Ym[:, 1], MIXED_TOL)


def test_stock_log_kernel_deviation():
    """The tutorial's log kernel as written calls the host libm's log, which
    is not correctly rounded; this engine (like the oracle) evaluates a
    correctly rounded log.  At N = 65,536, TOL 10 the engine's FP64 result is
    compared with the reference built with the stock kernel: the misrounded
    entries move some ACA pivots, so the two agree to the method's accuracy
    but not to the last bits."""
    if not RefLib.available():
        pytest.skip("reference build (oracle/_ref) not present")
    pts, q, p = workloads.make("uniform1m", N=65536)
    a = A.AFMM(len(pts), 64, 10, pts, kernel="log")
    a.assemble()
    y = a.computeMatVecProduct(q)
    r = RefLib(pts, 64, 10, 101)  # kernel 101: examples/tutorial.cpp:22-35 with libm log
    r.assemble()
    ys = r.matvec(q)
    rel = float(np.linalg.norm(y - ys) / np.linalg.norm(ys))
    print(f"engine (correctly rounded log) vs reference with libm log: {rel:.3e}")
    assert rel <= 1e-8


def test_rank_zero_boxes():
    """A Gaussian so narrow (exp(-r^2/1e-6)) that every far-field entry
    underflows to 0: ACA returns rank 0 for every box (where the reference's
    Eigen asserts fire, src/AFMM2DTree.cpp:1151), the far field contributes
    nothing, and every path equals the direct product."""
    pts = np.random.default_rng(3).uniform(0, 1, (16384, 2))
    q = np.random.default_rng(4).standard_normal(16384)
    a = A.AFMM(16384, 64, 8, pts, kernel="gaussian", kparam=1e-6)
    a.assemble()
    for lev in range(2, a.nLevels + 1):
        assert not a.ranks(lev).any()
    yd = dense_rows(pts, q, "gaussian", a.nLevels, np.arange(16384), kparam=1e-6)
    assert_rel(a.computeMatVecProduct(q), yd, 1e-13)
    assert_rel(a.computeMatVecProduct(q, precision="mixed"), yd, MIXED_TOL)
    Q = np.stack([q, 2 * q, -q, q, q, q, q, q, q], 1)
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    assert_rel(Yb[:, 1], 2 * yd, 1e-13)
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    assert_rel(Ym[:, 2], -yd, MIXED_TOL)


@pytest.mark.parametrize("kernel,tol", [("one_over_r", 6), ("log", 10), ("gaussian", 8)])
def test_fixed_point_m2l_blocks(kernel, tol):
    """The mixed paths' 32-bit fixed-point M2L blocks against the FP64 blocks:
    both mixed results stay within the mixed tolerance of the FP64 path."""
    pts, _, _ = workloads.make("mixture4m", N=65536)
    a = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    a.assemble()
    b = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    b.set_m2l_fixed_point(False)
    b.assemble()
    assert a.m2l_fixed_point() and not b.m2l_fixed_point()
    assert a.m2l_stored() and b.m2l_stored()
    Q = np.random.default_rng(8).standard_normal((65536, 16))
    Ya, Yb = a.computeMatVecProduct(Q, precision="mixed"), b.computeMatVecProduct(Q, precision="mixed")
    ya1, yb1 = a.computeMatVecProduct(Q[:, 3], precision="mixed"), b.computeMatVecProduct(Q[:, 3], precision="mixed")
    for c in (0, 3, 15):
        y64 = a.computeMatVecProduct(Q[:, c])
        assert_rel(Ya[:, c], y64, MIXED_TOL)
        assert_rel(Yb[:, c], y64, MIXED_TOL)
    assert_rel(ya1, a.computeMatVecProduct(Q[:, 3]), MIXED_TOL)
    assert_rel(yb1, b.computeMatVecProduct(Q[:, 3]), MIXED_TOL)
    # the FP64 paths never use the fixed-point blocks
    np.testing.assert_array_equal(a.computeMatVecProduct(Q[:, 0]), b.computeMatVecProduct(Q[:, 0]))


@pytest.mark.parametrize("precision,nrhs", [("fp64", 3), ("mixed", 16), ("mixed", 21), ("fp64_batched", 17)])
def test_host_pipeline_matches_device_pointers(precision, nrhs):
    """Host-pointer calls run in pipelined column passes on separate copy
    streams; their results equal the device-pointer call's bit for bit, with
    a leading dimension larger than N."""
    torch = pytest.importorskip("torch")
    pts, _, _ = workloads.make("mixture4m", N=32768)
    a = A.AFMM(32768, 64, 6, pts, kernel="one_over_r")
    a.assemble()
    ld = 32768 + 5
    Q = np.zeros((nrhs, ld))
    Q[:, :32768] = np.random.default_rng(nrhs).standard_normal((nrhs, 32768))
    Y = np.full((nrhs, ld), 7.0)
    a.matvec_host_ptr(Q.ctypes.data, Y.ctypes.data, nrhs, ld, precision)
    dq = torch.tensor(Q, device="cuda")
    dy = torch.zeros_like(dq)
    a.matvec_device(dq.data_ptr(), dy.data_ptr(), nrhs, ld, precision)
    np.testing.assert_array_equal(Y[:, :32768], dy.cpu().numpy()[:, :32768])
    assert np.all(Y[:, 32768:] == 7.0)


@pytest.mark.gpu
def test_aca_plan_does_not_change_results():
    """The ACA launch plan (CTAs per box and per SM) changes only the setup
    time: ranks, skeletons, pivot columns and the FP64 matvec are identical."""
    pts, q, _ = workloads.make("mixture4m", N=65536)
    base = A.AFMM(65536, 64, 6, pts, kernel="one_over_r")
    base.assemble()
    y0 = base.computeMatVecProduct(q)
    for cluster, per_sm in [(1, 1), (2, 2), (4, 2), (16, 1)]:
        a = A.AFMM(65536, 64, 6, pts, kernel="one_over_r")
        a.set_aca_plan(cluster, per_sm)
        a.assemble()
        assert a.setup_times()[f"assemble_aca_cluster_level{a.nLevels}_s"] == cluster
        for lev in range(2, a.nLevels + 1):
            np.testing.assert_array_equal(a.ranks(lev), base.ranks(lev))
            np.testing.assert_array_equal(a.skeletons(lev), base.skeletons(lev))
            np.testing.assert_array_equal(a.charge_points(lev), base.charge_points(lev))
        np.testing.assert_array_equal(a.computeMatVecProduct(q), y0)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,tol", [("one_over_r", 6), ("log", 10), ("gaussian", 8), ("one_over_r_scaled", 8)])
def test_tcgen05_near_field(kernel, tol):
    """The 16-column mixed near field on tcgen05 tiles (sibling leaf pairs,
    tensor-memory accumulators) against the FP64 path and against the
    mma.sync form, every kernel; leaves of 64 points."""
    pts, _, _ = workloads.make("mixture4m", N=65536)
    a = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    a.assemble()
    Q = np.random.default_rng(6).standard_normal((65536, 16))
    a.set_tuning(p2p_tc=0)
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    a.set_tuning(p2p_tc=1)
    Yt = a.computeMatVecProduct(Q, precision="mixed")
    Yt2 = a.computeMatVecProduct(Q, precision="mixed")
    np.testing.assert_array_equal(Yt, Yt2)  # deterministic
    for c in (0, 5, 15):
        y64 = a.computeMatVecProduct(Q[:, c])
        assert_rel(Yt[:, c], y64, MIXED_TOL)
        assert_rel(Yt[:, c], Ym[:, c], MIXED_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,tol,wl", [("one_over_r", 6, "mixture4m"), ("log", 10, "uniform1m"),
                                           ("gaussian", 8, "mixture4m"), ("one_over_r_scaled", 8, "mixture4m")])
def test_tcgen05_m2l(kernel, tol, wl):
    """The 16-column mixed stored M2L on tcgen05 tiles (row tiles of a
    parent's children, sources over the union of their lists, fixed-point
    blocks decoded to FP32) against the FP64 path and against the FP64-tile
    form; at TOL 10 the ranks exceed 32 (several stages per source box) and
    a parent's children exceed 128 rows (several tiles per parent).  The
    FP64-batched passes do not use it."""
    pts, _, _ = workloads.make(wl, N=65536)
    a = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    a.assemble()
    Q = np.random.default_rng(7).standard_normal((65536, 16))
    a.set_tuning(m2l_tc=0, otf_batched=0)
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    a.set_tuning(m2l_tc=1)
    assert a.tuning()["m2l_tc"] == 1
    Yt = a.computeMatVecProduct(Q, precision="mixed")
    np.testing.assert_array_equal(Yt, a.computeMatVecProduct(Q, precision="mixed"))  # deterministic
    np.testing.assert_array_equal(a.computeMatVecProduct(Q, precision="fp64_batched"), Yb)
    for c in (0, 5, 15):
        y64 = a.computeMatVecProduct(Q[:, c])
        assert_rel(Yt[:, c], y64, MIXED_TOL)
        assert_rel(Yt[:, c], Ym[:, c], MIXED_TOL)
    # with the near field on tcgen05 tiles as well
    a.set_tuning(p2p_tc=1)
    Ytt = a.computeMatVecProduct(Q, precision="mixed")
    for c in (0, 15):
        assert_rel(Ytt[:, c], a.computeMatVecProduct(Q[:, c]), MIXED_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,tol,wl", [("one_over_r", 6, "mixture4m"), ("log", 10, "uniform1m"),
                                           ("log", 12, "mixture4m"), ("gaussian", 8, "mixture4m")])
def test_tcgen05_integer_m2l(kernel, tol, wl):
    """The 16-column mixed stored M2L as exact integer products on tcgen05
    (byte planes of the fixed-point blocks and of the charges, m2l_tc = 2)
    agrees with the FP64-tile form on the same fixed-point blocks to the
    charges' 32-bit rounding, and with the FP64 path within the mixed
    tolerance; deterministic.  TOL 10 / 12 give ranks above 32 (several
    stages per source box) and above 128 (several row tiles per box)."""
    pts, _, _ = workloads.make(wl, N=65536)
    a = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    a.set_m2l_fixed_point(2)
    a.assemble()
    Q = np.random.default_rng(8).standard_normal((65536, 16))
    a.set_tuning(m2l_tc=0, otf_batched=0)
    Ym = a.computeMatVecProduct(Q, precision="mixed")
    Yb = a.computeMatVecProduct(Q, precision="fp64_batched")
    a.set_tuning(m2l_tc=2)
    Yi = a.computeMatVecProduct(Q, precision="mixed")
    np.testing.assert_array_equal(Yi, a.computeMatVecProduct(Q, precision="mixed"))
    np.testing.assert_array_equal(a.computeMatVecProduct(Q, precision="fp64_batched"), Yb)
    for c in (0, 7, 15):
        assert_rel(Yi[:, c], Ym[:, c], 1e-8)
        assert_rel(Yi[:, c], a.computeMatVecProduct(Q[:, c]), MIXED_TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,tol,wl", [("one_over_r", 6, "mixture4m"), ("log", 10, "uniform1m")])
def test_sharded_matvec_sums_to_whole(kernel, tol, wl):
    """afmm_set_shard: each shard computes its subtrees' potentials (zeros
    elsewhere); the shards' outputs sum to the whole product bit for bit in
    every precision, for even and uneven splits; count 1 restores it."""
    pts, _, _ = workloads.make(wl, N=65536)
    a = A.AFMM(65536, 64, tol, pts, kernel=kernel)
    a.assemble()
    Q = np.random.default_rng(9).standard_normal((65536, 16))
    whole = {"fp64": a.computeMatVecProduct(Q[:, 3]), "mixed": a.computeMatVecProduct(Q[:, 3], precision="mixed"),
             "batched": a.computeMatVecProduct(Q, precision="mixed"),
             "fp64_batched": a.computeMatVecProduct(Q, precision="fp64_batched")}
    for count in (2, 3, 5):
        sums = {k: np.zeros_like(v) for k, v in whole.items()}
        owned = np.zeros(65536, bool)
        for i in range(count):
            a.set_shard(i, count)
            assert a.shard()[:2] == (i, count)
            ys = {"fp64": a.computeMatVecProduct(Q[:, 3]),
                  "mixed": a.computeMatVecProduct(Q[:, 3], precision="mixed"),
                  "batched": a.computeMatVecProduct(Q, precision="mixed"),
                  "fp64_batched": a.computeMatVecProduct(Q, precision="fp64_batched")}
            mine = ys["fp64"] != 0
            assert not (owned & mine).any()  # disjoint shards
            owned |= mine
            for k in ys:
                sums[k] += ys[k]
        assert owned.all()
        for k in whole:
            np.testing.assert_array_equal(sums[k], whole[k])
    a.set_shard(0, 1)
    np.testing.assert_array_equal(a.computeMatVecProduct(Q[:, 3]), whole["fp64"])
    with pytest.raises(A.AFMMError):
        a.set_shard(2, 2)
