"""C-ABI checks that need no GPU: the library loads, exports every entry
point declared in include/afmm2d.h, and validates arguments before touching a
device."""
import ctypes
import os
import re

import numpy as np
import pytest

import afmm2d_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:afmm_status|const char\*)\s+(afmm_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = A.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_status_strings():
    lib = A.lib()
    assert lib.afmm_version().decode().startswith("afmm2d-b200")
    assert lib.afmm_status_string(1).decode() == "bad argument"


def _create(N, M, pts, kernel=1, kp=None):
    h = ctypes.c_void_p()
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    st = A.lib().afmm_create(N, M, 8, ctypes.c_void_p(pts.ctypes.data), 1, kernel,
                             None if kp is None else ctypes.c_void_p(kp.ctypes.data), 0 if kp is None else 1,
                             ctypes.byref(h))
    return st, h


def test_rejects_fewer_than_two_levels():
    st, h = _create(100, 64, np.zeros((100, 2)))
    assert st == 1 and not h.value
    assert b"nLevels" in A.lib().afmm_last_error(None)


def test_rejects_bad_arguments():
    lib = A.lib()
    h = ctypes.c_void_p()
    assert lib.afmm_create(4096, 32, 8, None, 1, 1, None, 0, ctypes.byref(h)) == 1
    assert _create(4096, 32, np.zeros((4096, 2)), kernel=9)[0] == 1
    pts = np.random.default_rng(0).uniform(0, 1, (4096, 2))
    pts[17, 1] = np.nan
    st, _ = _create(4096, 32, pts)
    assert st == 1 and b"non-finite" in lib.afmm_last_error(None)
    assert _create(4096, 0, pts)[0] == 1
    assert _create(4096, 32, np.zeros((4096, 2)), kernel=3, kp=np.array([-1.0]))[0] == 1
    assert lib.afmm_assemble(None) == 1
    assert lib.afmm_matvec(None, None, None, 1, 1, 0, 0) == 1


def test_null_handle_queries_are_rejected():
    lib = A.lib()
    n = ctypes.c_int()
    assert lib.afmm_get_nlevels(None, ctypes.byref(n)) == 1
    assert lib.afmm_set_m2l_storage(None, 0) == 1
    assert lib.afmm_get_m2l_stored(None, ctypes.byref(n)) == 1
    assert lib.afmm_get_setup_phases(None, 0, None, None, ctypes.byref(n)) == 1
    assert lib.afmm_set_get_stage_times(None, 0, None, None, ctypes.byref(n)) == 1
    assert lib.afmm_set_get_stream(None, None) == 1
    assert lib.afmm_destroy(None) == 0


def test_no_device_is_reported_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pts = np.random.default_rng(0).uniform(0, 1, (4096, 2))
    st, h = _create(4096, 32, pts)
    assert st == 7 and not h.value


def test_python_mirror_raises_on_bad_config():
    with pytest.raises(A.AFMMError):
        A.AFMM(100, 64, 8, np.zeros((100, 2)))


def test_measurement_helpers_reject_null_pointers():
    lib = A.lib()
    assert lib.afmm_measure_fma_peaks(None, None) == 1
    assert lib.afmm_measure_fp64_pipes(None, None, None) == 1


@pytest.mark.gpu
def test_measurement_helpers_report_positive_peaks():
    """The roofline denominators the bench measures live: FP64 / FP32 FMA,
    FP64 tensor (DMMA) and both FP64 forms issued together."""
    fp64, fp32 = A.measure_fma_peaks()
    dmma, dfma, both = A.measure_fp64_pipes()
    for v in (fp64, fp32, dmma, dfma, both):
        assert np.isfinite(v) and v > 1.0
    assert fp32 > fp64
