"""The CPU oracle restatement is pinned against the reference (golden
fixtures generated by running the reference itself, and the compiled
reference when it is present)."""
import numpy as np
import pytest

from oracle_lib import Oracle, RefLib, dense_rows, kd_total_order, lists_closed_form, oracle_lib


def test_oracle_matches_golden(golden):
    o = Oracle(golden["pts"], golden["M"], golden["tol"], golden["kernel"])
    assert o.L == golden["L"]
    np.testing.assert_array_equal(o.permutation(), golden["perm"])
    c, b = o.leaves()
    np.testing.assert_array_equal(c, golden["counts"])
    np.testing.assert_array_equal(b, golden["boxnum"])
    for lev in range(1, o.L + 1):
        nb, inn, out = o.lists(lev)
        np.testing.assert_array_equal(nb, golden[f"nbr{lev}"])
        np.testing.assert_array_equal(inn, golden[f"inner{lev}"])
        np.testing.assert_array_equal(out, golden[f"outer{lev}"])
    o.assemble()
    for lev in range(2, o.L + 1):
        np.testing.assert_array_equal(o.ranks(lev), golden[f"rank{lev}"])
        np.testing.assert_array_equal(o.skeletons(lev), golden[f"skel{lev}"])
    y = o.matvec(golden["q"])
    assert_rel(y, golden["y"], 1e-13)


def assert_rel(y, ref, tol):
    """Relative 2-norm within tol; NaN entries (the reference's output for
    exact duplicate points, whose L2P solve is singular) must match in place."""
    nan = np.isnan(ref)
    np.testing.assert_array_equal(np.isnan(y), nan)
    if (~nan).any():
        rel = np.linalg.norm(y[~nan] - ref[~nan]) / np.linalg.norm(ref[~nan])
        assert rel <= tol, rel


def test_total_order_kd_matches_golden(golden):
    """The GPU's total-order formulation of the KD sort equals the reference's merge sort."""
    np.testing.assert_array_equal(kd_total_order(golden["pts"], golden["L"]), golden["perm"])


def test_closed_form_lists_match_golden(golden):
    for lev in range(1, golden["L"] + 1):
        nb, inn, out = lists_closed_form(lev)
        np.testing.assert_array_equal(nb, golden[f"nbr{lev}"])
        np.testing.assert_array_equal(inn, golden[f"inner{lev}"])
        np.testing.assert_array_equal(out, golden[f"outer{lev}"])


def test_closed_form_lists_deep_levels():
    """Closed form vs the restated recurrence up to level 7 (the golden set reaches 4)."""
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 1, (4 ** 7 * 2, 2))
    o = Oracle(pts, 2, 4, "log")
    assert o.L == 7
    for lev in range(1, 8):
        for a, b in zip(o.lists(lev), lists_closed_form(lev)):
            np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not RefLib.available(), reason="reference not compiled here")
@pytest.mark.parametrize("kernel,tol,M", [("log", 10, 64), ("one_over_r", 6, 64), ("gaussian", 8, 32),
                                           ("one_over_r_scaled", 12, 32)])
def test_oracle_matches_reference_live(kernel, tol, M):
    rng = np.random.default_rng(11)
    pts = rng.uniform(0, 1, (16384, 2))
    q = rng.standard_normal(16384)
    o, r = Oracle(pts, M, tol, kernel), RefLib(pts, M, tol, kernel)
    np.testing.assert_array_equal(o.permutation(), r.permutation())
    o.assemble()
    r.assemble()
    for lev in range(2, o.L + 1):
        np.testing.assert_array_equal(o.ranks(lev), r.ranks(lev))
        np.testing.assert_array_equal(o.skeletons(lev), r.skeletons(lev))
    yo, yr = o.matvec(q), r.matvec(q)
    assert np.linalg.norm(yo - yr) / np.linalg.norm(yr) <= 1e-13


def test_oracle_accuracy_vs_dense():
    rng = np.random.default_rng(5)
    pts = rng.uniform(-1, 1, (4096, 2))
    q = rng.uniform(-1, 1, 4096)
    o = Oracle(pts, 32, 8, "log")
    o.assemble()
    y = o.matvec(q)
    rows = np.arange(4096)
    yd = dense_rows(pts, q, "log", o.L, rows)
    assert np.linalg.norm(y - yd) / np.linalg.norm(yd) < 1e-5


def test_nlevels_formula():
    from afmm2d_b200 import nlevels
    lib = oracle_lib()
    for N in [4096, 6000, 65536, 1 << 20, 1 << 22, 1 << 24, 12345, 100]:
        for M in [1, 16, 20, 32, 64, 100, 200]:
            assert nlevels(N, M) == lib.afo_nlevels(N, M), (N, M)
    assert nlevels(10, 20) == -1


def test_oracle_rejects_shallow_tree():
    with pytest.raises(ValueError):
        Oracle(np.random.default_rng(0).uniform(0, 1, (100, 2)), 64, 8, "log")
