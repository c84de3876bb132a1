"""Generates the golden fixtures in this directory by running the REFERENCE.

The reference's own sources are compiled here (``make -C oracle ref``, which
needs the reference checkout) against the Eigen-API shim; this script drives
that library on small seeded inputs and stores inputs and outputs as .npz:
permutation, leaf counts, box-number map, interaction lists, per-level ranks
and skeletons, and the matvec output.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_lib import RefLib  # noqa: E402


def grid_with_ties(n_side, rng):
    g = np.stack(np.meshgrid(np.arange(n_side), np.arange(n_side)), -1).reshape(-1, 2) / n_side
    return g[rng.permutation(len(g))].astype(np.float64)


def cases():
    rng = np.random.Generator(np.random.PCG64(0xAF3D))
    out = {}
    out["uniform4k_log"] = (rng.uniform(-1, 1, (4096, 2)), rng.uniform(-1, 1, 4096), 32, 8, "log")
    out["grid4k_oneoverr"] = (grid_with_ties(64, rng), rng.standard_normal(4096), 32, 6, "one_over_r")
    c = rng.uniform(0, 1, (16, 2))
    mix = c[rng.integers(0, 16, 8192)] + 0.02 * rng.standard_normal((8192, 2))
    out["mixture8k_oneoverr"] = (mix, rng.standard_normal(8192), 64, 6, "one_over_r")
    out["ragged6000_scaled"] = (rng.uniform(0, 1, (6000, 2)), rng.standard_normal(6000), 20, 10, "one_over_r_scaled")
    out["uniform4k_gauss"] = (rng.uniform(0, 1, (4096, 2)), rng.standard_normal(4096), 16, 8, "gaussian")
    th = rng.uniform(0, 20 * np.pi, 4096)
    sp = np.stack([0.05 * th * np.cos(th), 0.05 * th * np.sin(th)], 1) + 1e-4 * rng.standard_normal((4096, 2))
    sp = np.concatenate([sp, rng.uniform(sp.min(0), sp.max(0), (4096, 2))])
    out["spiral8k_log"] = (sp, rng.standard_normal(8192), 32, 10, "log")
    # duplicates and signed zeros: exact coordinate ties
    base = rng.uniform(-1, 1, (1024, 2))
    base[:64, 0] = 0.0
    base[64:128, 0] = -0.0
    base[128:160, 1] = -0.0
    dup = np.concatenate([base, base[rng.permutation(1024)]])
    out["dups2k_log"] = (dup, rng.standard_normal(2048), 16, 8, "log")
    out["dups2k_oneoverr"] = (dup, rng.standard_normal(2048), 16, 8, "one_over_r")
    return out


def main():
    if not RefLib.available():
        sys.exit("build the reference first: make -C oracle ref")
    for name, (pts, q, M, tol, kern) in cases().items():
        r = RefLib(pts, M, tol, kern)
        r.assemble()
        y = r.matvec(q)
        counts, boxnum = r.leaves()
        d = dict(pts=pts, q=q, M=M, tol=tol, kernel=kern, L=r.L, perm=r.permutation(), counts=counts,
                 boxnum=boxnum, y=y)
        for lev in range(1, r.L + 1):
            nb, inn, out = r.lists(lev)
            d[f"nbr{lev}"], d[f"inner{lev}"], d[f"outer{lev}"] = nb, inn, out
        for lev in range(2, r.L + 1):
            d[f"rank{lev}"] = r.ranks(lev)
            d[f"skel{lev}"] = r.skeletons(lev)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print(name, "N", len(pts), "L", r.L, "mean leaf rank", d[f"rank{r.L}"].mean())


if __name__ == "__main__":
    main()
