"""User kernels registered from outside the library (AFMM_REGISTER_KERNEL),
the counterpart of the reference's user-defined userkernel::getMatrixEntry
(include/kernel.hpp:58, examples/testAFMM2D.cpp:9-20).  The test kernel, an
inverse multiquadric 1/sqrt(r^2 + c), lives in tests/plugin/imq_kernel.cu and
is compiled into its own library; nothing of it is in libafmm2d.so."""
import ctypes
import os

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads
from oracle_lib import Oracle, kernel_pairs
from test_oracle import assert_rel

HERE = os.path.dirname(os.path.abspath(__file__))
PLUGIN = os.path.join(HERE, "plugin", "libafmm_imq.so")
IMQ = 16  # AFMM_KERNEL_USER_FIRST
C = 1e-4  # kernel parameter c


@pytest.fixture(scope="module")
def plugin():
    if not os.path.exists(PLUGIN):
        pytest.fail("tests/plugin/libafmm_imq.so is missing: run __graft_entry__.build()")
    return A.load_kernel_plugin(PLUGIN)


def test_plugin_registers_its_kernel(plugin):
    assert A.kernel_name(IMQ) == "InverseMultiquadric"
    assert A.kernel_name(1) == "log"
    L = A.lib()
    name = ctypes.c_char_p()
    assert L.afmm_kernel_name(IMQ + 1, ctypes.byref(name)) == 1
    # ids outside the user range, foreign tables and a second table for a taken id are refused
    blob = (ctypes.c_char * 4096)()
    assert L.afmm_register_kernel(3, blob, 64, 1) == 1
    assert L.afmm_register_kernel(IMQ + 2, blob, 64, 1) == 1
    assert L.afmm_register_kernel(IMQ + 2, None, 64, 1) == 1
    # an unregistered user id is rejected before any device work
    h = ctypes.c_void_p()
    pts = np.random.default_rng(0).uniform(0, 1, (4096, 2))
    assert L.afmm_create(4096, 32, 8, ctypes.c_void_p(pts.ctypes.data), 1, IMQ + 1, None, 0, ctypes.byref(h)) == 1


@pytest.mark.gpu
def test_user_kernel_entries(plugin):
    rng = np.random.default_rng(21)
    xy1 = rng.uniform(0, 1, (50000, 2))
    xy2 = xy1 + rng.standard_normal((50000, 2)) * np.exp(rng.uniform(-12, 0, (50000, 1)))
    xy2[:50] = xy1[:50]
    g = A.kernel_eval(IMQ, 2.0 ** -7, xy1, xy2, mode="exact", param=C)
    np.testing.assert_array_equal(g, kernel_pairs("imq", 2.0 ** -7, xy1, xy2, param=C))
    f = A.kernel_eval(IMQ, 2.0 ** -7, xy1, xy2, mode="fp64", param=C)
    assert np.all(np.abs(f - g) <= 4e-16 * np.abs(g))


@pytest.mark.gpu
def test_user_kernel_parity_vs_oracle(plugin):
    """Every stage runs the out-of-tree functor: ranks, skeletons and pivot
    columns bit-exact against the oracle, potentials within 10^-TOL, and the
    mixed, batched and many-problem paths within their tolerances."""
    pts, _, _ = workloads.make("mixture4m", N=32768)
    q = np.random.default_rng(3).standard_normal(32768)
    a = A.AFMM(32768, 64, 8, pts, kernel=IMQ, kparam=C)
    a.assemble()
    o = Oracle(pts, 64, 8, "imq", kparam=C)
    o.assemble()
    for lev in range(2, a.nLevels + 1):
        np.testing.assert_array_equal(a.ranks(lev), o.ranks(lev))
        np.testing.assert_array_equal(a.skeletons(lev), o.skeletons(lev))
        np.testing.assert_array_equal(a.charge_points(lev), o.charge_points(lev))
    yo = o.matvec(q)
    assert_rel(a.computeMatVecProduct(q), yo, 1e-8)
    assert_rel(a.computeMatVecProduct(q, precision="mixed"), yo, 1e-6)
    Q = np.stack([q] + [np.random.default_rng(k).standard_normal(32768) for k in range(15)], 1)
    assert_rel(a.computeMatVecProduct(Q, precision="mixed")[:, 0], yo, 1e-6)
    assert_rel(a.computeMatVecProduct(Q, precision="fp64_batched")[:, 0], yo, 1e-8)
    b = A.AFMM(32768, 64, 8, pts, kernel=IMQ, kparam=C)
    b.set_m2l_storage("on_the_fly")
    b.assemble()
    assert_rel(b.computeMatVecProduct(q), yo, 1e-8)
    st = A.AFMMSet([a])
    assert np.array_equal(st.matvec([q])[0], a.computeMatVecProduct(q))
    st.close()
