"""Generates tests/golden/full_size/uniform1m_log_tol10.npz by running the REFERENCE at
full size: N = 1,048,576 points uniform in [0,1]^2, log kernel, M = 64,
TOL_POW = 10, one charge vector N(0,1) (afmm2d_b200.workloads "uniform1m").

The reference's own sources are compiled here (``make -C oracle ref``, which
needs the reference checkout) against the Eigen-API shim.  The full outputs
are large, so the fixture keeps what a bit-exact or 1e-10 comparison needs
in compact form:
  * leaf counts and the DFS -> quadtree box map (full),
  * ranks of every box of levels 2..7 (full),
  * SHA-256 of the permutation, of every level's lists, skeletons and pivot
    columns (little-endian int64 / int32 bytes),
  * the potentials at 32,768 seeded sample rows and the 2-norm of the full
    potential vector.
Run from the repository root (about 15 minutes on 8 cores):

    python tests/golden/make_uniform1m_fixture.py
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle_lib import RefLib  # noqa: E402

from afmm2d_b200 import workloads  # noqa: E402

OUT = os.path.join(HERE, "full_size", "uniform1m_log_tol10.npz")
SAMPLE_ROWS = 32768
SAMPLE_SEED = 0xC2


def sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def main():
    if not RefLib.available():
        sys.exit("build the reference first: make -C oracle ref REF=<reference checkout>")
    pts, q, p = workloads.make("uniform1m")
    t0 = time.time()
    r = RefLib(pts, p["M"], p["tol"], p["kernel"])
    t1 = time.time()
    r.assemble()
    t2 = time.time()
    y = r.matvec(q)
    t3 = time.time()
    counts, boxnum = r.leaves()
    rows = np.sort(np.random.Generator(np.random.PCG64(SAMPLE_SEED)).choice(len(pts), SAMPLE_ROWS, replace=False))
    d = dict(N=len(pts), M=p["M"], tol=p["tol"], kernel=p["kernel"], L=r.L, counts=counts, boxnum=boxnum,
             perm_sha=sha(r.permutation(), "<i8"), rows=rows.astype(np.int64), y_rows=y[rows],
             y_norm=np.linalg.norm(y), ref_seconds=np.array([t1 - t0, t2 - t1, t3 - t2]))
    for lev in range(1, r.L + 1):
        d[f"lists_sha{lev}"] = sha(np.concatenate(r.lists(lev)), "<i4")
    for lev in range(2, r.L + 1):
        d[f"rank{lev}"] = r.ranks(lev)
        d[f"skel_sha{lev}"] = sha(r.skeletons(lev), "<i4")
        d[f"cpiv_sha{lev}"] = sha(r.charge_points(lev), "<i4")
    np.savez_compressed(OUT, **d)
    print(f"L={r.L} create {t1 - t0:.1f} s, assemble {t2 - t1:.1f} s, matvec {t3 - t2:.1f} s; wrote {OUT}")


if __name__ == "__main__":
    main()
