"""Seeded synthetic point clouds and load vectors for the benchmark workloads.

The reference's point sets (data/ln1M.pts, p1M.pts, ...) are not shipped, so
the workloads use numpy PCG64 generators with the documented recipes.  The
``.pts`` format is the reference's (src/oct/OctFunctions.C:313-370): a uint32
count followed by 3*count float64 coordinates.
"""
from __future__ import annotations

import numpy as np


def clamp_unit(pts: np.ndarray, max_depth: int) -> np.ndarray:
    """Clamp into [0, 1) as solve_neumann does (examples/src/backend/omgNeumann.C:860-864):
    negatives become 0, values >= 1 become 1 - 2^-(maxDepth+1)."""
    p = np.array(pts, dtype=np.float64, copy=True)
    p[p < 0] = 0.0
    p[p >= 1] = 1.0 - np.ldexp(0.5, -max_depth)
    return p


def gaussian_cloud(n: int, seed: int, mean=0.5, sigma=0.1) -> np.ndarray:
    """n points, each coordinate N(mean, sigma) in float64 (PCG64 seed)."""
    rng = np.random.default_rng(seed)
    return rng.normal(mean, sigma, (n, 3))


def lognormal_cloud(n: int, seed: int) -> np.ndarray:
    """n points, each coordinate exp(N(0,1)) divided by the per-axis max."""
    rng = np.random.default_rng(seed)
    p = np.exp(rng.normal(0.0, 1.0, (n, 3)))
    return p / p.max(axis=0, keepdims=True)


def uniform_cloud(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, (n, 3))


def uniform_rhs(n: int, seed: int) -> np.ndarray:
    """Load vector with i.i.d. U[-1, 1] entries (as ComputeRandomRHS fills a Vec,
    examples/src/backend/omgRhs.C:1262-1287, with a seeded generator)."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


# Named workloads: (points, maxDepth).  Sizes follow the benchmark recipes.
def workload_points(name: str, scale: float = 1.0):
    if name == "gauss131k_d10":
        n = max(8, int(131072 * scale))
        return clamp_unit(gaussian_cloud(n, 0), 10), 10
    if name == "lognormal1m_d14":
        n = max(8, int(1048576 * scale))
        return clamp_unit(lognormal_cloud(n, 2), 14), 14
    if name == "lognormal4m_d16":
        n = max(8, int(4194304 * scale))
        return clamp_unit(lognormal_cloud(n, 4), 16), 16
    if name == "uniform512k_d12":
        n = max(8, int(524288 * scale))
        return clamp_unit(uniform_cloud(n, 5), 12), 12
    raise KeyError(name)


def batch_clouds(count: int = 32, first_seed: int = 100, depth: int = 12, n_lo: float = 1e4, n_hi: float = 5e5):
    """Independent Gaussian clouds: per seed, n log-uniform in [n_lo, n_hi],
    sigma U[0.05, 0.2], centre U[0.3, 0.7]^3, coordinates N(centre, sigma),
    clamped to [0, 1)."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(first_seed + i)
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        sigma = rng.uniform(0.05, 0.2)
        c = rng.uniform(0.3, 0.7, 3)
        out.append(clamp_unit(rng.normal(c, sigma, (n, 3)), depth))
    return out, depth


def sphere_coefficients(centers: np.ndarray, inside=1.0e4, outside=1.0, radius=0.25) -> np.ndarray:
    """Per-element [alpha, beta]: alpha = `inside` when the element centre lies
    within `radius` of (0.5,0.5,0.5), else `outside`; beta = 1."""
    r = np.linalg.norm(centers - 0.5, axis=1)
    coef = np.empty((len(centers), 2))
    coef[:, 0] = np.where(r < radius, inside, outside)
    coef[:, 1] = 1.0
    return coef.reshape(-1)


def read_pts(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(4), np.uint32)[0])
        return np.frombuffer(f.read(24 * n), np.float64).reshape(n, 3).copy()


def write_pts(path: str, pts: np.ndarray) -> None:
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    with open(path, "wb") as f:
        f.write(np.uint32(len(pts)).tobytes())
        f.write(pts.tobytes())
