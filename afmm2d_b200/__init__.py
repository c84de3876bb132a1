"""AFMM2D on B200: Python mirror of the reference ``AFMM`` interface.

The reference (vaishna77/AFMM2D, include/AFMM2D.hpp:14-33) exposes

    AFMM(int N, int MinParticlesInLeaf, int TOL_POW, Eigen::MatrixXd& loc)
    void assemble()
    Eigen::VectorXd computeMatVecProduct(Eigen::VectorXd)
    void evaluateError()
    double* sorted_Locations, *sorted_Properties;  unsigned nLevels

with the kernel supplied as ``userkernel::getMatrixEntry``.  This module
offers the same class over the C ABI of ``libafmm2d.so`` (include/afmm2d.h);
every computation runs in the CUDA library, and importing fails loudly when
the library is missing.  The kernel is chosen by name or id (``KERNELS``).
"""
import ctypes
import os

import numpy as np

__all__ = ["AFMM", "AFMMError", "AFMMSet", "KERNELS", "PRECISIONS", "device_alloc_count", "kernel_eval", "kernel_name",
           "lib", "load_kernel_plugin", "nlevels"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libafmm2d.so")

KERNELS = {"one_over_r_scaled": 0, "log": 1, "one_over_r": 2, "gaussian": 3}
PRECISIONS = {"fp64": 0, "mixed": 1, "fp64_batched": 2}
STATUS = {0: "ok", 1: "bad argument", 2: "out of device memory", 3: "CUDA error", 4: "device wait timed out",
          5: "non-finite values", 6: "not assembled", 7: "no sm_100 device"}

_vp, _i, _i64, _u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64
_SIGS = {
    "afmm_create": [_i, _i, _i, _vp, _i, _i, _vp, _i, _vp],
    "afmm_assemble": [_vp],
    "afmm_save": [_vp, ctypes.c_char_p],
    "afmm_load": [ctypes.c_char_p, _vp],
    "afmm_matvec": [_vp, _vp, _vp, _i, _i64, _i, _i],
    "afmm_eval_error": [_vp, _i, _u64, _vp],
    "afmm_get_permutation": [_vp, _vp],
    "afmm_get_sorted_locations": [_vp, _vp],
    "afmm_get_nlevels": [_vp, _vp],
    "afmm_get_params": [_vp, _vp, _vp],
    "afmm_get_leaves": [_vp, _vp, _vp],
    "afmm_get_lists": [_vp, _i, _vp, _vp, _vp],
    "afmm_get_ranks": [_vp, _i, _vp],
    "afmm_get_skeletons": [_vp, _i, _vp, _vp],
    "afmm_get_charge_points": [_vp, _i, _vp, _vp],
    "afmm_get_l2p": [_vp, _i, _i, _vp, _vp, _vp],
    "afmm_set_profiling": [_vp, _i],
    "afmm_set_m2l_storage": [_vp, _i],
    "afmm_get_m2l_stored": [_vp, _vp],
    "afmm_set_m2l_fixed_point": [_vp, _i],
    "afmm_set_aca_plan": [_vp, _i, _i],
    "afmm_get_m2l_fixed_point": [_vp, _vp],
    "afmm_get_stage_times": [_vp, _i, _vp, _vp, _vp],
    "afmm_get_setup_times": [_vp, _vp],
    "afmm_get_counts": [_vp, _vp],
    "afmm_get_setup_phases": [_vp, _i, _vp, _vp, _vp],
    "afmm_get_launch_count": [_vp, _vp],
    "afmm_get_stream": [_vp, _vp],
    "afmm_kernel_eval": [_i, ctypes.c_double, ctypes.c_double, _i64, _vp, _vp, _vp, _i],
    "afmm_measure_fma_peaks": [_vp, _vp],
    "afmm_measure_fp64_pipes": [_vp, _vp, _vp],
    "afmm_set_shard": [_vp, _i, _i],
    "afmm_get_shard": [_vp, _vp, _vp, _vp],
    "afmm_shard_range": [_i, _i, _i, _vp, _vp, _vp],
    "afmm_kd_permutation_noalloc": [_i, _i, _vp, _vp, _vp, _vp],
    "afmm_get_device_alloc_count": [_vp],
    "afmm_autotune": [_vp, _i, ctypes.c_char_p, _vp],
    "afmm_get_tuning": [_vp, _vp, _i],
    "afmm_set_tuning": [_vp, _vp, _i],
    "afmm_register_kernel": [_i, _vp, ctypes.c_size_t, _i],
    "afmm_kernel_name": [_i, _vp],
    "afmm_destroy": [_vp],
    "afmm_set_create": [_vp, _i, _vp],
    "afmm_set_matvec": [_vp, _vp, _vp, _i],
    "afmm_set_get_offsets": [_vp, _vp],
    "afmm_set_get_launches": [_vp, _vp, _vp],
    "afmm_set_get_stream": [_vp, _vp],
    "afmm_set_sweep_wait_margin": [_vp, _i],
    "afmm_set_get_stage_times": [_vp, _i, _vp, _vp, _vp],
    "afmm_set_destroy": [_vp],
}
_lib = None


class AFMMError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Loads ``libafmm2d.so`` (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m afmm2d_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _i
        L.afmm_last_error.argtypes = [_vp]
        L.afmm_last_error.restype = ctypes.c_char_p
        L.afmm_set_last_error.argtypes = [_vp]
        L.afmm_set_last_error.restype = ctypes.c_char_p
        L.afmm_status_string.argtypes = [_i]
        L.afmm_status_string.restype = ctypes.c_char_p
        L.afmm_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(st, h=None):
    if st != 0:
        raise AFMMError(st, lib().afmm_last_error(h).decode())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def kernel_eval(kernel, a, xy1, xy2, mode="exact", param=0.01):
    """K(xy1[t], xy2[t]) for point pairs on the GPU.  mode: "exact" (setup
    arithmetic), "fp64" (matvec form) or "fp32"."""
    kid = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
    xy1 = np.ascontiguousarray(xy1, dtype=np.float64).reshape(-1, 2)
    xy2 = np.ascontiguousarray(xy2, dtype=np.float64).reshape(-1, 2)
    out = np.zeros(len(xy1))
    m = {"exact": 0, "fp64": 1, "fp32": 2}[mode]
    _check(lib().afmm_kernel_eval(kid, float(a), float(param), len(xy1), _ptr(xy1), _ptr(xy2), _ptr(out), m))
    return out


def measure_fma_peaks():
    """(FP64, FP32) FMA throughput of the current device in TFLOP/s."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(lib().afmm_measure_fma_peaks(ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def shard_range(nlevels, index, count):
    """(level, k0, k1): the boxes [k0, k1) of `level` that shard `index` of
    `count` owns on a tree of `nlevels` levels (no device needed)."""
    lev, a, b = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
    _check(lib().afmm_shard_range(int(nlevels), int(index), int(count), ctypes.byref(lev), ctypes.byref(a),
                                  ctypes.byref(b)))
    return lev.value, a.value, b.value


def measure_fp64_pipes():
    """(DMMA, DFMA, both together) FP64 throughput of the current device in TFLOP/s."""
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _check(lib().afmm_measure_fp64_pipes(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return a.value, b.value, c.value


_plugins = []


def load_kernel_plugin(path):
    """Loads a user kernel library (built from a translation unit using
    AFMM_REGISTER_KERNEL, see include/afmm2d_kernel.cuh); its kernel ids are
    then accepted by AFMM(kernel=id).  Returns the ctypes library handle."""
    lib()
    h = ctypes.CDLL(os.path.abspath(path))
    _plugins.append(h)
    return h


def kernel_name(kernel_id):
    """Name of a built-in or registered kernel id."""
    p = ctypes.c_char_p()
    _check(lib().afmm_kernel_name(int(kernel_id), ctypes.byref(p)))
    return p.value.decode()


def device_alloc_count():
    """Device allocations (cudaMalloc) the library has made in this process."""
    n = ctypes.c_int64()
    _check(lib().afmm_get_device_alloc_count(ctypes.byref(n)))
    return n.value


def nlevels(N, M):
    """nLevels exactly as src/AFMM2D.cpp:7 computes it (integer N/M, truncated)."""
    if N <= 0 or M <= 0 or N // M < 1:
        return -1
    return int(np.log(float(N // M)) / np.log(4.0))


class AFMM:
    """AFMM(N, MinParticlesInLeaf, TOL_POW, loc, kernel="log", kparam=None).

    ``loc`` is an (N, 2) array of point coordinates (the reference's
    ``Eigen::MatrixXd loc(N, 2)``).  Construction builds the KD-tree
    permutation and the interaction lists on the GPU (src/AFMM2D.cpp:3-39).
    """

    def __init__(self, N, MinParticlesInLeaf, TOL_POW, loc, kernel="log", kparam=None, _handle=None):
        L = lib()
        if _handle is not None:  # AFMM.load
            self._adopt(_handle)
            return
        kid = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
        loc = np.ascontiguousarray(np.asarray(loc, dtype=np.float64).reshape(N, 2))
        kp = np.array([kparam if kparam is not None else 0.01], dtype=np.float64)
        h = ctypes.c_void_p()
        st = L.afmm_create(int(N), int(MinParticlesInLeaf), int(TOL_POW), _ptr(loc), 1, kid, _ptr(kp),
                           1 if kparam is not None else 0, ctypes.byref(h))
        _check(st, None)
        self._h = h
        self.N = int(N)
        self.MinParticlesInLeaf = int(MinParticlesInLeaf)
        self.TOL_POW = int(TOL_POW)
        self.kernel_id = kid
        n = ctypes.c_int()
        _check(L.afmm_get_nlevels(h, ctypes.byref(n)), h)
        self.nLevels = n.value
        self.assembled = False

    def _adopt(self, h):
        self._h = h
        v = np.zeros(5, np.int32)
        _check(lib().afmm_get_params(h, _ptr(v), None), h)
        self.N, self.MinParticlesInLeaf, self.TOL_POW, self.nLevels, self.kernel_id = (int(x) for x in v)
        self.assembled = True

    def save(self, path):
        """Writes the assembled setup (permutation, ranks, skeletons, L2P) to
        a versioned binary file that AFMM.load reads back."""
        _check(lib().afmm_save(self._h, os.fsencode(path)), self._h)

    @classmethod
    def load(cls, path):
        """An assembled AFMM from a file written by save(), without the KD
        sort and the ACA; its matvecs have the same bits as the saved one's."""
        h = ctypes.c_void_p()
        _check(lib().afmm_load(os.fsencode(path), ctypes.byref(h)))
        return cls(0, 0, 0, None, _handle=h)

    # ------------------------------------------------------- reference API
    def assemble(self):
        """ACA skeletons, L2P and M2L blocks of every box (src/AFMM2D.cpp:41-44)."""
        _check(lib().afmm_assemble(self._h), self._h)
        self.assembled = True

    M2L_STORAGE = {"auto": 0, "store": 1, "on_the_fly": 2}

    def set_m2l_storage(self, mode):
        """M2L block storage before assemble(): "auto" (store when they fit),
        "store", or "on_the_fly" (entries evaluated in FP64 by every matvec)."""
        _check(lib().afmm_set_m2l_storage(self._h, self.M2L_STORAGE[mode]), self._h)

    def set_shard(self, index, count):
        """After assemble(): compute only shard `index` of `count` (its
        subtrees' potentials; zeros elsewhere), so that the shards' outputs
        sum to the whole product.  count = 1 restores the whole problem."""
        _check(lib().afmm_set_shard(self._h, int(index), int(count)), self._h)

    def shard(self):
        """(index, count, level) of the handle's shard."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().afmm_get_shard(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), self._h)
        return a.value, b.value, c.value

    def set_m2l_fixed_point(self, on):
        """Before assemble(): keep a 32-bit fixed-point copy of the stored M2L
        blocks for the mixed-precision paths (default on, when it fits); 2
        also keeps its byte planes for the integer tcgen05 M2L (m2l_tc = 2)."""
        _check(lib().afmm_set_m2l_fixed_point(self._h, int(on)), self._h)

    def set_aca_plan(self, cluster=0, ctas_per_sm=0):
        """Before assemble(): CTAs per box and per SM of the ACA kernel
        (0 = automatic); results do not depend on it, only the setup time."""
        _check(lib().afmm_set_aca_plan(self._h, int(cluster), int(ctas_per_sm)), self._h)

    def m2l_fixed_point(self):
        v = ctypes.c_int()
        _check(lib().afmm_get_m2l_fixed_point(self._h, ctypes.byref(v)), self._h)
        return bool(v.value)

    def m2l_stored(self):
        v = ctypes.c_int()
        _check(lib().afmm_get_m2l_stored(self._h, ctypes.byref(v)), self._h)
        return bool(v.value)

    def computeMatVecProduct(self, b, precision="fp64"):
        """y = K b in the original point order (src/AFMM2D.cpp:46-65)."""
        b = np.ascontiguousarray(np.asarray(b, dtype=np.float64))
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        q = np.asfortranarray(b.reshape(self.N, nrhs))
        y = np.zeros((self.N, nrhs), dtype=np.float64, order="F")
        _check(lib().afmm_matvec(self._h, _ptr(q), _ptr(y), nrhs, self.N, PRECISIONS[precision], 0), self._h)
        return y[:, 0] if b.ndim == 1 else y

    def evaluateError(self, nsample=1, seed=0):
        """Relative error of the last FP64 matvec against direct evaluation over
        ``nsample`` seeded leaves (src/AFMM2D.cpp:67-74; all leaves if <= 0)."""
        e = ctypes.c_double()
        _check(lib().afmm_eval_error(self._h, int(nsample), int(seed), ctypes.byref(e)), self._h)
        return e.value

    @property
    def sorted_Properties(self):
        """Original index of each sorted point, as doubles (include/AFMM2D.hpp:25)."""
        return self.permutation().astype(np.float64)

    @property
    def sorted_Locations(self):
        """Sorted locations, interleaved x, y (include/AFMM2D.hpp:24)."""
        xy = np.zeros(2 * self.N)
        _check(lib().afmm_get_sorted_locations(self._h, _ptr(xy)), self._h)
        return xy

    # ------------------------------------------------------------- extras
    def matvec_device(self, q_ptr, y_ptr, nrhs, ld, precision="fp64"):
        """y = K q with device pointers (e.g. torch ``data_ptr()``), column-major N x nrhs."""
        _check(lib().afmm_matvec(self._h, ctypes.c_void_p(q_ptr), ctypes.c_void_p(y_ptr), int(nrhs), int(ld),
                                 PRECISIONS[precision], 1), self._h)

    def matvec_host_ptr(self, q_ptr, y_ptr, nrhs, ld, precision="fp64"):
        """y = K q with host pointers (e.g. pinned memory)."""
        _check(lib().afmm_matvec(self._h, ctypes.c_void_p(q_ptr), ctypes.c_void_p(y_ptr), int(nrhs), int(ld),
                                 PRECISIONS[precision], 0), self._h)

    def permutation(self):
        p = np.zeros(self.N, dtype=np.int64)
        _check(lib().afmm_get_permutation(self._h, _ptr(p)), self._h)
        return p

    def leaves(self):
        n = 4 ** self.nLevels
        c = np.zeros(n, np.int32)
        b = np.zeros(n, np.int32)
        _check(lib().afmm_get_leaves(self._h, _ptr(c), _ptr(b)), self._h)
        return c, b

    def lists(self, level):
        n = 4 ** level
        a = [np.zeros(n * s, np.int32) for s in (8, 16, 24)]
        _check(lib().afmm_get_lists(self._h, int(level), *[_ptr(x) for x in a]), self._h)
        return a

    def ranks(self, level):
        r = np.zeros(4 ** level, np.int32)
        _check(lib().afmm_get_ranks(self._h, int(level), _ptr(r)), self._h)
        return r

    def _ids(self, fn, level):
        c = ctypes.c_int64()
        _check(fn(self._h, int(level), None, ctypes.byref(c)), self._h)
        ids = np.zeros(max(c.value, 1), np.int32)
        _check(fn(self._h, int(level), _ptr(ids), ctypes.byref(c)), self._h)
        return ids[: c.value]

    def skeletons(self, level):
        return self._ids(lib().afmm_get_skeletons, level)

    def charge_points(self, level):
        return self._ids(lib().afmm_get_charge_points, level)

    def l2p(self, level, k):
        r, c = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().afmm_get_l2p(self._h, int(level), int(k), ctypes.byref(r), ctypes.byref(c), None), self._h)
        out = np.zeros((r.value, c.value))
        if r.value * c.value:
            _check(lib().afmm_get_l2p(self._h, int(level), int(k), ctypes.byref(r), ctypes.byref(c), _ptr(out)),
                   self._h)
        return out

    TUNING_KEYS = ("pf_fp64", "pf_batched", "otf_mixed", "otf_batched", "host_pass_cols", "m2l_t16", "p2p_tc",
                   "m2l_tc")

    def autotune(self, what=0, cache=None):
        """Times the launch parameters on this problem and keeps the fastest
        (what: bit 0 prefetch windows, bit 1 per-level M2L forms, bit 2 host
        pass width, bit 3 M2L form (FP64 tiles or tcgen05 integer products), bit 4 tcgen05 near field; 0 = all).  With `cache` (a file path) a stored result for
        the same device and problem structure is reused.  Returns
        (tuning dict, from_cache)."""
        hit = ctypes.c_int()
        _check(lib().afmm_autotune(self._h, int(what), None if cache is None else os.fsencode(cache),
                                   ctypes.byref(hit)), self._h)
        return self.tuning(), bool(hit.value)

    def tuning(self):
        v = np.zeros(len(self.TUNING_KEYS), np.int64)
        _check(lib().afmm_get_tuning(self._h, _ptr(v), len(v)), self._h)
        return dict(zip(self.TUNING_KEYS, v.tolist()))

    def set_tuning(self, **kw):
        v = np.array([kw.get(k, x) for k, x in self.tuning().items()], np.int64)
        _check(lib().afmm_set_tuning(self._h, _ptr(v), len(v)), self._h)

    def set_profiling(self, on=True):
        """True / 1: per-stage CUDA events; 2: the same with the batched near
        field run after the far field (each stage its kernels' own time)."""
        _check(lib().afmm_set_profiling(self._h, int(on)), self._h)

    def stage_times(self):
        """Per-stage device milliseconds of the last matvec (profiling on)."""
        n = ctypes.c_int()
        names = (ctypes.c_char_p * 64)()
        ms = (ctypes.c_double * 64)()
        _check(lib().afmm_get_stage_times(self._h, 64, names, ms, ctypes.byref(n)), self._h)
        return {names[i].decode(): ms[i] for i in range(min(n.value, 64))}

    def setup_times(self):
        t = np.zeros(2)
        _check(lib().afmm_get_setup_times(self._h, _ptr(t)), self._h)
        out = {"create_s": t[0], "assemble_s": t[1]}
        n = ctypes.c_int()
        names = (ctypes.c_char_p * 64)()
        secs = (ctypes.c_double * 64)()
        _check(lib().afmm_get_setup_phases(self._h, 64, names, secs, ctypes.byref(n)), self._h)
        out.update({"assemble_" + names[i].decode() + "_s": secs[i] for i in range(min(n.value, 64))})
        return out

    def counts(self):
        c = np.zeros(7, np.int64)
        _check(lib().afmm_get_counts(self._h, _ptr(c)), self._h)
        keys = ["nlevels", "N", "sum_rank", "l2p_entries", "m2l_entries", "near_evals", "far_entries"]
        return dict(zip(keys, c.tolist()))

    def launch_count(self):
        n = ctypes.c_int64()
        _check(lib().afmm_get_launch_count(self._h, ctypes.byref(n)), self._h)
        return n.value

    def stream(self):
        s = ctypes.c_void_p()
        _check(lib().afmm_get_stream(self._h, ctypes.byref(s)), self._h)
        return s.value

    def close(self):
        if getattr(self, "_h", None):
            lib().afmm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AFMMSet:
    """Many assembled ``AFMM`` problems applied in one call: every stage of
    the FP64 matvec is one fused launch over all problems, recorded once in a
    CUDA graph and replayed per call.  Each problem's result has the same bits
    as its own ``computeMatVecProduct(q, "fp64")``.  The problems stay owned
    by the caller and must outlive the set."""

    def __init__(self, problems):
        self.problems = list(problems)
        arr = (ctypes.c_void_p * len(self.problems))(*[p._h.value for p in self.problems])
        h = ctypes.c_void_p()
        _check(lib().afmm_set_create(arr, len(self.problems), ctypes.byref(h)))
        self._h = h
        self.offsets = np.zeros(len(self.problems) + 1, np.int64)
        self._call("afmm_set_get_offsets", _ptr(self.offsets))
        self.total = int(self.offsets[-1])

    def _call(self, name, *args):
        st = getattr(lib(), name)(self._h, *args)
        if st != 0:
            raise AFMMError(st, lib().afmm_set_last_error(self._h).decode())

    def matvec(self, qs):
        """qs: list of per-problem charge vectors (original point order) or
        one concatenated vector; returns the list of potentials."""
        q = np.ascontiguousarray(np.concatenate(qs) if isinstance(qs, (list, tuple)) else qs, dtype=np.float64)
        if q.shape != (self.total,):
            raise ValueError(f"need {self.total} charges in total")
        y = np.zeros(self.total)
        self._call("afmm_set_matvec", _ptr(q), _ptr(y), 0)
        return [y[self.offsets[p]:self.offsets[p + 1]] for p in range(len(self.problems))]

    def matvec_device(self, q_ptr, y_ptr):
        """Concatenated charges / potentials in device memory (raw pointers)."""
        self._call("afmm_set_matvec", ctypes.c_void_p(q_ptr), ctypes.c_void_p(y_ptr), 1)

    def launches(self):
        """(fused launches per matvec recorded in the graph, graph launches so far)"""
        a, b = ctypes.c_int(), ctypes.c_int64()
        self._call("afmm_set_get_launches", ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def stream(self):
        s = ctypes.c_void_p()
        self._call("afmm_set_get_stream", ctypes.byref(s))
        return s.value

    def set_sweep_wait_margin(self, margin):
        """Test hook of the sweeps' bounded waits (afmm_set_sweep_wait_margin)."""
        self._call("afmm_set_sweep_wait_margin", int(margin))

    def stage_times(self):
        """Device milliseconds per stage of the last matvec."""
        n = ctypes.c_int()
        names = (ctypes.c_char_p * 16)()
        ms = (ctypes.c_double * 16)()
        self._call("afmm_set_get_stage_times", 16, names, ms, ctypes.byref(n))
        return {names[i].decode(): ms[i] for i in range(min(n.value, 16))}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().afmm_set_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
