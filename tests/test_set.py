"""Many independent problems in one call (afmm_set_*): every stage fused over
all problems and replayed from one CUDA graph.  Each problem's potentials must
have the same bits as its own FP64 matvec, which the parity tests pin to the
reference."""
import ctypes

import numpy as np
import pytest

import afmm2d_b200 as A
from afmm2d_b200 import workloads


def test_set_entry_points_reject_null_arguments():
    L = A.lib()
    out = ctypes.c_void_p()
    assert L.afmm_set_create(None, 0, ctypes.byref(out)) != 0
    assert not out.value
    assert L.afmm_set_create(None, 1, None) == 1  # AFMM_BAD_ARG: no output pointer
    assert L.afmm_set_matvec(None, None, None, 0) == 1
    assert L.afmm_set_get_offsets(None, None) == 1
    assert L.afmm_set_get_launches(None, None, None) == 1
    assert L.afmm_set_destroy(None) == 0


def test_many_problem_workload_shape():
    probs, p = workloads.many_problems(count=16)
    sizes = [len(q) for _, q in probs]
    assert sizes == list(workloads.many_sizes(16))
    assert all(2048 <= n <= 65536 for n in sizes)
    assert p["kernel"] == "log" and p["M"] == 32 and p["tol"] == 8
    a, _ = workloads.many_problems(count=3)
    b, _ = workloads.many_problems(count=3)
    assert all(np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]) for x, y in zip(a, b))


def _problems(count, nmax):
    probs, p = workloads.many_problems(count=count, nmax=nmax)
    hs = []
    for pts, _ in probs:
        h = A.AFMM(len(pts), p["M"], p["tol"], pts, kernel=p["kernel"])
        h.assemble()
        hs.append(h)
    return probs, hs


@pytest.mark.gpu
def test_set_matches_each_problem_bit_for_bit():
    probs, hs = _problems(10, 16384)
    own = [h.computeMatVecProduct(q, "fp64") for h, (_, q) in zip(hs, probs)]
    st = A.AFMMSet(hs)
    per, n0 = st.launches()
    assert n0 == 0 and per >= 6
    ys = st.matvec([q for _, q in probs])
    for y, ref in zip(ys, own):
        assert np.array_equal(y, ref)
    # the recorded graph is replayed: same bits again, one graph launch per call
    ys2 = st.matvec([q for _, q in probs])
    assert all(np.array_equal(a, b) for a, b in zip(ys, ys2))
    assert st.launches()[1] == 2
    # new charges through the same graph
    rng = np.random.default_rng(5)
    q3 = [rng.standard_normal(len(q)) for _, q in probs]
    ys3 = st.matvec(q3)
    for h, q, y in zip(hs, q3, ys3):
        assert np.array_equal(y, h.computeMatVecProduct(q, "fp64"))
    st.close()


@pytest.mark.gpu
def test_set_device_pointers_and_sizes_of_every_level_count():
    import torch
    # sizes giving 3, 4 and 5 levels (M = 32) in one set
    probs, hs = _problems(6, 65536)
    levels = {h.nLevels for h in hs}
    st = A.AFMMSet(hs)
    q = torch.from_numpy(np.concatenate([q for _, q in probs])).cuda()
    y = torch.empty_like(q)
    st.matvec_device(q.data_ptr(), y.data_ptr())
    got = y.cpu().numpy()
    for k, (h, (_, qk)) in enumerate(zip(hs, probs)):
        assert np.array_equal(got[st.offsets[k]:st.offsets[k + 1]], h.computeMatVecProduct(qk, "fp64"))
    assert len(levels) >= 2
    st.close()


@pytest.mark.gpu
def test_set_rejects_mixed_kernels_and_unassembled_handles():
    rng = np.random.default_rng(1)
    pts = rng.uniform(0, 1, (4096, 2))
    a = A.AFMM(4096, 32, 8, pts, kernel="log")
    a.assemble()
    b = A.AFMM(4096, 32, 8, pts, kernel="one_over_r")
    b.assemble()
    with pytest.raises(A.AFMMError) as e:
        A.AFMMSet([a, b])
    assert e.value.status == 1
    c = A.AFMM(4096, 32, 8, pts, kernel="log")
    with pytest.raises(A.AFMMError) as e:
        A.AFMMSet([a, c])
    assert e.value.status == 6


@pytest.mark.gpu
def test_set_sweep_wait_gives_up_with_timeout_status():
    """The persistent sweeps' device waits are bounded: with the test margin
    no wait can be satisfied, the matvec returns AFMM_TIMEOUT after the time
    limit instead of hanging, and the set works again once it is removed."""
    import time
    probs, hs = _problems(4, 8192)
    st = A.AFMMSet(hs)
    qs = [q for _, q in probs]
    good = st.matvec(qs)
    st.set_sweep_wait_margin(1)
    t0 = time.perf_counter()
    with pytest.raises(A.AFMMError) as e:
        st.matvec(qs)
    assert e.value.status == 4  # AFMM_TIMEOUT
    assert time.perf_counter() - t0 < 60
    st.set_sweep_wait_margin(0)
    again = st.matvec(qs)
    assert all(np.array_equal(a, b) for a, b in zip(good, again))
    with pytest.raises(A.AFMMError):
        st.set_sweep_wait_margin(-1)
    st.close()
