"""ctypes wrappers of the CPU oracles (test infrastructure only).

``Oracle`` drives oracle/libafmm_oracle.so, this project's C++ restatement of
the reference algorithm; ``RefLib`` drives oracle/_ref/libafmm2d_ref.so, the
reference's own sources compiled here against an Eigen-API shim.  Both share
one C API shape (prefixes ``afo_`` and ``ref_``).
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libafmm_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libafmm2d_ref.so")
KERNEL_IDS = {"one_over_r_scaled": 0, "log": 1, "one_over_r": 2, "gaussian": 3, "imq": 16}

vp, I, D, L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long


def _load(path, pre):
    lib = ctypes.CDLL(path)
    f = lambda n: getattr(lib, pre + n)  # noqa: E731
    f("create").restype = vp
    f("create").argtypes = [I, I, I, vp, I, D]
    for n, a in [("assemble", [vp]), ("matvec", [vp, vp, vp]), ("get_permutation", [vp, vp]),
                 ("get_sorted_locations", [vp, vp]), ("get_leaves", [vp, vp, vp]),
                 ("get_lists", [vp, I, vp, vp, vp]), ("get_ranks", [vp, I, vp])]:
        f(n).argtypes = a
        f(n).restype = None
    for n in ("get_skeletons", "get_charge_points"):
        f(n).argtypes = [vp, I, vp]
        f(n).restype = L
    f("get_l2p").argtypes = [vp, I, I, vp, vp, vp]
    f("get_l2p").restype = L
    f("get_stage").argtypes = [vp, I, I, vp]
    f("get_stage").restype = L
    return lib, f


class _Base:
    PATH = None
    PRE = None
    _cache = {}

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self, pts, M, tol, kernel, kparam=0.01):
        key = (self.PATH, self.PRE)
        if key not in _Base._cache:
            _Base._cache[key] = _load(self.PATH, self.PRE)
        self.lib, self.f = _Base._cache[key]
        self.pts = np.ascontiguousarray(pts, dtype=np.float64)
        self.N = len(self.pts)
        kid = KERNEL_IDS[kernel] if isinstance(kernel, str) else kernel
        self.h = self.f("create")(self.N, M, tol, self.pts.ctypes.data, kid, kparam)
        if not self.h:
            raise ValueError("oracle rejected the configuration (nLevels < 2)")
        self.L = self._nlevels()

    def _nlevels(self):
        raise NotImplementedError

    def assemble(self):
        self.f("assemble")(self.h)

    def matvec(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        y = np.zeros(self.N)
        self.f("matvec")(self.h, q.ctypes.data, y.ctypes.data)
        return y

    def permutation(self):
        p = np.zeros(self.N, np.int64)
        self.f("get_permutation")(self.h, p.ctypes.data)
        return p

    def sorted_locations(self):
        xy = np.zeros(2 * self.N)
        self.f("get_sorted_locations")(self.h, xy.ctypes.data)
        return xy

    def leaves(self):
        n = 4 ** self.L
        c, b = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.f("get_leaves")(self.h, c.ctypes.data, b.ctypes.data)
        return c, b

    def lists(self, level):
        a = [np.zeros(4 ** level * s, np.int32) for s in (8, 16, 24)]
        self.f("get_lists")(self.h, level, *[x.ctypes.data for x in a])
        return a

    def ranks(self, level):
        r = np.zeros(4 ** level, np.int32)
        self.f("get_ranks")(self.h, level, r.ctypes.data)
        return r

    def _ids(self, name, level):
        n = self.f(name)(self.h, level, None)
        ids = np.zeros(max(n, 1), np.int32)
        self.f(name)(self.h, level, ids.ctypes.data)
        return ids[:n]

    def skeletons(self, level):
        return self._ids("get_skeletons", level)

    def charge_points(self, level):
        return self._ids("get_charge_points", level)

    def l2p(self, level, k):
        r, c = ctypes.c_int32(), ctypes.c_int32()
        self.f("get_l2p")(self.h, level, k, ctypes.byref(r), ctypes.byref(c), None)
        out = np.zeros((r.value, c.value))
        if out.size:
            self.f("get_l2p")(self.h, level, k, ctypes.byref(r), ctypes.byref(c), out.ctypes.data)
        return out

    def stage(self, level, which):
        n = self.f("get_stage")(self.h, level, which, None)
        v = np.zeros(max(n, 1))
        self.f("get_stage")(self.h, level, which, v.ctypes.data)
        return v[:n]


class Oracle(_Base):
    PATH = ORACLE_SO
    PRE = "afo_"

    def _nlevels(self):
        self.lib.afo_get_nlevels.argtypes = [vp]
        return self.lib.afo_get_nlevels(self.h)

    def __del__(self):
        try:
            self.lib.afo_destroy.argtypes = [vp]
            self.lib.afo_destroy(self.h)
        except Exception:
            pass


class RefLib(_Base):
    """The reference itself.  Its objects are never freed (the reference's
    destructor double-frees, src/KDTree.cpp:202-203 vs src/AFMM2D.cpp:77-78)."""
    PATH = REF_SO
    PRE = "ref_"

    def _nlevels(self):
        self.lib.ref_nlevels.argtypes = [vp]
        return self.lib.ref_nlevels(self.h)


def oracle_lib():
    lib = ctypes.CDLL(ORACLE_SO)
    lib.afo_nlevels.argtypes = [I, I]
    lib.afo_lists_closed_form.argtypes = [I, vp, vp, vp]
    lib.afo_lists_closed_form.restype = None
    lib.afo_kd_total_order.argtypes = [I, I, vp, vp]
    lib.afo_kd_total_order.restype = None
    lib.afo_dense_rows.argtypes = [I, vp, I, D, D, vp, I, vp, vp]
    lib.afo_dense_rows.restype = None
    return lib


def dense_rows(pts, q, kernel, L, rows, kparam=0.01):
    """Direct FP64 (compensated) y[rows] = sum_j K(x_rows, x_j) q_j, original order."""
    lib = oracle_lib()
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    y = np.zeros(len(rows))
    kid = KERNEL_IDS[kernel] if isinstance(kernel, str) else kernel
    lib.afo_dense_rows(len(pts), pts.ctypes.data, kid, 0.5 ** L, kparam, q.ctypes.data, len(rows),
                       rows.ctypes.data, y.ctypes.data)
    return y


def kernel_pairs(kernel, a, xy1, xy2, param=0.01):
    """K(xy1[t], xy2[t]) with the oracle's kernels (host libm)."""
    lib = oracle_lib()
    lib.afo_kernel_pairs.argtypes = [I, D, D, L, vp, vp, vp]
    lib.afo_kernel_pairs.restype = None
    xy1 = np.ascontiguousarray(xy1, dtype=np.float64)
    xy2 = np.ascontiguousarray(xy2, dtype=np.float64)
    out = np.zeros(len(xy1))
    kid = KERNEL_IDS[kernel] if isinstance(kernel, str) else kernel
    lib.afo_kernel_pairs(kid, a, param, len(xy1), xy1.ctypes.data, xy2.ctypes.data, out.ctypes.data)
    return out


def kd_total_order(pts, L):
    lib = oracle_lib()
    pts = np.ascontiguousarray(pts, dtype=np.float64)
    p = np.zeros(len(pts), np.int64)
    lib.afo_kd_total_order(len(pts), L, pts.ctypes.data, p.ctypes.data)
    return p


def lists_closed_form(level):
    lib = oracle_lib()
    a = [np.zeros(4 ** level * s, np.int32) for s in (8, 16, 24)]
    lib.afo_lists_closed_form(level, *[x.ctypes.data for x in a])
    return a
