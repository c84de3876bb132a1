"""Builds the in-tree CUDA library ``afmm2d_b200/libafmm2d.so`` for sm_100a.

Usage: ``python -m afmm2d_b200.build`` (or ``build()`` from Python).  The
library is compiled with nvcc directly (no JIT cache), so the ``.so`` travels
with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libafmm2d.so")
SOURCES = ["kd_sort.cu", "aca.cu", "fmm.cu", "mixed.cu", "batched.cu", "set.cu", "capi.cu",
           "kernels_one_over_r_scaled.cu", "kernels_log.cu", "kernels_one_over_r.cu", "kernels_gaussian.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3",
    "-shared",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "afmm2d.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compiles every source to an object under _build/ in parallel, then
    links the shared library."""
    if not force and not needs_build():
        return OUT
    objdir = os.path.join(HERE, "..", "_build")
    os.makedirs(objdir, exist_ok=True)
    cflags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), *cflags, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, cwd=CSRC)))
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return OUT


def build_kernel_plugin(source, out, verbose=False):
    """Compiles a user kernel translation unit (one that includes
    include/afmm2d_kernel.cuh and uses AFMM_REGISTER_KERNEL) into a shared
    library linked against libafmm2d.so; loading it registers the kernel."""
    include = os.path.abspath(os.path.join(HERE, "..", "include"))
    rel = os.path.relpath(HERE, os.path.dirname(os.path.abspath(out)))
    cmd = [nvcc(), *NVCC_FLAGS, "-I", include, os.path.abspath(source), "-o", os.path.abspath(out),
           "-L", HERE, "-lafmm2d", "-Xlinker", "-rpath,$ORIGIN/" + rel]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=os.path.dirname(os.path.abspath(source)))
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
