"""The allocation-free KD permutation (afmm_kd_permutation_noalloc).

Some callers cannot allocate GPU memory: their device memory is already
reserved by another framework's caching allocator, they must keep a fixed and
declared footprint, or they cannot pay a cudaMalloc/cudaFree pair per call
(cudaFree synchronises the whole device).  For them the library computes the
KD permutation with a static 5 MiB scratch array (up to 65,536 points).  This
file is collected last so that a run stopping at the first failure has run
every other test first; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536


def noalloc(N, M, dxy, dperm, dsorted):
    return A.lib().afmm_kd_permutation_noalloc(N, M, ctypes.c_void_p(dxy.data_ptr()),
                                              ctypes.c_void_p(dperm.data_ptr()),
                                              None if dsorted is None else ctypes.c_void_p(dsorted.data_ptr()), None)


@pytest.mark.parametrize("name,N,M", [("mixture4m", MAX_POINTS, 64), ("uniform1m", 50000, 32)])
def test_no_alloc_permutation_matches_afmm_create(name, N, M):
    torch = pytest.importorskip("torch")
    pts = workloads.make(name, N=N)[0]
    ref = A.AFMM(N, M, 6, pts, kernel="one_over_r").permutation()  # the existing entry point
    dxy = torch.tensor(pts, device="cuda").contiguous()
    perm = torch.empty(N, dtype=torch.int64, device="cuda")
    srt = torch.empty((N, 2), dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row share the static scratch
        perm.fill_(-1)
        srt.zero_()
        torch.cuda.synchronize()
        allocs = A.device_alloc_count()
        assert noalloc(N, M, dxy, perm, srt) == 0, A.lib().afmm_last_error(None)
        # the library counts every device allocation it makes: the call made none
        assert A.device_alloc_count() == allocs
        # integer output: exact agreement is the tolerance
        np.testing.assert_array_equal(perm.cpu().numpy(), ref)
        np.testing.assert_array_equal(srt.cpu().numpy(), pts[ref])


def test_alloc_counter_sees_the_allocating_entry_point():
    pts = workloads.make("uniform1m", N=8192)[0]
    allocs = A.device_alloc_count()
    A.AFMM(8192, 32, 6, pts, kernel="log").close()
    assert A.device_alloc_count() > allocs


def test_no_alloc_rejects_sizes_beyond_the_limit():
    torch = pytest.importorskip("torch")
    N = MAX_POINTS + 1
    dxy = torch.zeros((N, 2), dtype=torch.float64, device="cuda")
    perm = torch.empty(N, dtype=torch.int64, device="cuda")
    assert noalloc(N, 64, dxy, perm, None) == 1
    assert b"65536" in A.lib().afmm_last_error(None)
