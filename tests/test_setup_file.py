"""Setup files (afmm_save / afmm_load): a versioned binary image of the
assembled setup.  A loaded handle skips the KD sort and the ACA and must give
the same bits as the handle that was saved; damaged files are rejected on the
host before any device work."""
import ctypes

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads


def _load_status(path):
    h = ctypes.c_void_p()
    st = A.lib().afmm_load(str(path).encode(), ctypes.byref(h))
    return st, h, A.lib().afmm_last_error(None).decode()


def test_load_rejects_missing_and_foreign_files(tmp_path):
    st, h, msg = _load_status(tmp_path / "missing.bin")
    assert st == 1 and not h.value and "cannot open" in msg
    p = tmp_path / "foreign.bin"
    p.write_bytes(b"not a setup file at all" * 10)
    st, h, msg = _load_status(p)
    assert st == 1 and not h.value and "not an AFMM2D setup file" in msg
    assert A.lib().afmm_load(None, ctypes.byref(h)) == 1
    assert A.lib().afmm_save(None, b"x") == 1


@pytest.mark.gpu
@pytest.mark.parametrize("name,N,kernel,tol", [("mixture4m", 65536, "one_over_r", 6), ("uniform1m", 32768, "log", 10)])
def test_saved_setup_reloads_bit_for_bit(tmp_path, name, N, kernel, tol):
    pts, _, _ = workloads.make(name, N=N)
    a = A.AFMM(N, 64, tol, pts, kernel=kernel)
    a.assemble()
    path = tmp_path / "setup.afmm"
    a.save(path)
    b = A.AFMM.load(path)
    assert (b.N, b.MinParticlesInLeaf, b.TOL_POW, b.nLevels, b.kernel_id) == (N, 64, tol, a.nLevels, a.kernel_id)
    np.testing.assert_array_equal(b.permutation(), a.permutation())
    assert b.counts() == a.counts()
    for lev in range(2, a.nLevels + 1):
        np.testing.assert_array_equal(b.ranks(lev), a.ranks(lev))
        np.testing.assert_array_equal(b.skeletons(lev), a.skeletons(lev))
        np.testing.assert_array_equal(b.charge_points(lev), a.charge_points(lev))
    Q = np.random.default_rng(1).standard_normal((N, 16))
    for prec, cols in (("fp64", 0), ("mixed", 0), ("mixed", slice(None)), ("fp64_batched", slice(None))):
        np.testing.assert_array_equal(b.computeMatVecProduct(Q[:, cols], prec), a.computeMatVecProduct(Q[:, cols], prec))
    # saving the loaded handle reproduces the file byte for byte
    path2 = tmp_path / "again.afmm"
    b.save(path2)
    assert path2.read_bytes() == path.read_bytes()


@pytest.mark.gpu
def test_damaged_setup_files_are_rejected(tmp_path):
    pts, _, _ = workloads.make("uniform1m", N=16384)
    a = A.AFMM(16384, 64, 8, pts, kernel="log")
    a.assemble()
    path = tmp_path / "setup.afmm"
    a.save(path)
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.afmm"
    flipped = bytearray(raw)
    flipped[len(raw) - 100] ^= 0x40  # inside the last level's L2P operators
    bad.write_bytes(bytes(flipped))
    st, h, msg = _load_status(bad)
    assert st == 1 and not h.value and "digest" in msg
    bad.write_bytes(bytes(raw[: len(raw) // 2]))
    st, h, msg = _load_status(bad)
    assert st == 1 and not h.value and "truncated" in msg
    version = bytearray(raw)
    version[8] = 99
    bad.write_bytes(bytes(version))
    st, h, msg = _load_status(bad)
    assert st == 1 and "version" in msg
    with pytest.raises(A.AFMMError):
        A.AFMM(16384, 64, 8, pts, kernel="log").save(tmp_path / "unassembled.afmm")
