"""Seeded synthetic inputs for the AFMM2D workloads.

Each workload is (points, charges, parameters).  Points are float64 (N, 2);
charges float64 (N,) or (N, nrhs).  The generators use numpy's PCG64 with a
fixed seed per workload so every run sees the same inputs.

Workloads (kernel, MinParticlesInLeaf M, TOL_POW):
  uniform4k   N=4,096 uniform in [-1,1]^2, log, M=32, TOL 8, charges U[-1,1]
  uniform1m   N=1,048,576 uniform in [0,1]^2, log, M=64, TOL 10, charges N(0,1)
  mixture4m   N=4,194,304 from a 16-component Gaussian mixture (centres
              uniform in [0,1]^2, sigma 0.02), 1/r, M=64, TOL 6, charges N(0,1)
  gauss1m     N=1,048,576 uniform in [0,1]^2, exp(-r^2/0.01), M=64, TOL 8,
              64 charge vectors N(0,1)
  many        256 problems, N log-uniform in [2048, 65536], log, M=32, TOL 8
  spiral16m   N=16,777,216: half on the spiral r = 0.05*theta, theta in
              [0, 20*pi], jitter N(0, 1e-4^2) per coordinate, half uniform in
              the spiral's bounding box; log, M=64, TOL 12
"""
import numpy as np

WORKLOADS = {
    "uniform4k": dict(N=4096, M=32, tol=8, kernel="log", seed=0xAF3D2D01),
    "uniform1m": dict(N=1 << 20, M=64, tol=10, kernel="log", seed=0xAF3D2D02),
    "mixture4m": dict(N=1 << 22, M=64, tol=6, kernel="one_over_r", seed=0xAF3D2D03),
    "gauss1m": dict(N=1 << 20, M=64, tol=8, kernel="gaussian", seed=0xAF3D2D04, nrhs=64),
    "many": dict(count=256, nmin=2048, nmax=65536, M=32, tol=8, kernel="log", seed=0xAF3D2D05),
    "spiral16m": dict(N=1 << 24, M=64, tol=12, kernel="log", seed=0xAF3D2D06),
}


def uniform(N, lo, hi, rng):
    return rng.uniform(lo, hi, size=(N, 2))


def mixture(N, rng, components=16, sigma=0.02):
    centres = rng.uniform(0.0, 1.0, size=(components, 2))
    comp = rng.integers(0, components, size=N)
    return centres[comp] + sigma * rng.standard_normal((N, 2))


def spiral(N, rng):
    h = N // 2
    theta = rng.uniform(0.0, 20 * np.pi, size=h)
    r = 0.05 * theta
    s = np.stack([r * np.cos(theta), r * np.sin(theta)], axis=1) + 1e-4 * rng.standard_normal((h, 2))
    lo, hi = s.min(axis=0), s.max(axis=0)
    u = rng.uniform(lo, hi, size=(N - h, 2))
    return np.concatenate([s, u], axis=0)


def make(name, N=None, seed=None, nrhs=None):
    """Returns (points, charges, params) for a workload; N overrides the size
    (same distribution) for bounded samples and parity tests."""
    p = dict(WORKLOADS[name])
    if N is not None:
        p["N"] = int(N)
    if seed is not None:
        p["seed"] = seed
    if nrhs is not None:
        p["nrhs"] = nrhs
    rng = np.random.Generator(np.random.PCG64(p["seed"]))
    n = p["N"]
    if name == "uniform4k":
        pts = uniform(n, -1.0, 1.0, rng)
        q = rng.uniform(-1.0, 1.0, size=n)
    elif name in ("uniform1m", "gauss1m"):
        pts = uniform(n, 0.0, 1.0, rng)
        q = rng.standard_normal(n if p.get("nrhs", 1) == 1 else (n, p["nrhs"]))
    elif name == "mixture4m":
        pts = mixture(n, rng)
        q = rng.standard_normal(n if p.get("nrhs", 1) == 1 else (n, p["nrhs"]))
    elif name == "spiral16m":
        pts = spiral(n, rng)
        q = rng.standard_normal(n)
    else:
        raise KeyError(name)
    return np.ascontiguousarray(pts), np.ascontiguousarray(q), p


def many_sizes(count=256, nmin=2048, nmax=65536, seed=0xAF3D2D05):
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.round(np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=count))).astype(np.int64)


def many_problems(count=256, nmin=2048, nmax=65536, seed=0xAF3D2D05):
    """The many-problem workload: `count` independent problems, N log-uniform
    in [nmin, nmax] (many_sizes), points uniform in [0,1]^2, charges N(0,1);
    problem k draws from its own stream (seed + 1 + k).  Returns a list of
    (points, charges) and the shared parameters (log, M = 32, TOL 8)."""
    p = dict(WORKLOADS["many"])
    sizes = many_sizes(count, nmin, nmax, seed)
    probs = []
    for k, n in enumerate(sizes):
        rng = np.random.Generator(np.random.PCG64(seed + 1 + k))
        pts = uniform(int(n), 0.0, 1.0, rng)
        probs.append((np.ascontiguousarray(pts), rng.standard_normal(int(n))))
    return probs, p
