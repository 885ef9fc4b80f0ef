"""Loaders of the reference-generated golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

from oracle.oracle import OCT_DTYPE

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MESH_CASES = ["corner_points_d5", "uniform600_d7", "gauss1k_d8", "lognormal1k_d10"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def u32_to_octs(a):
    o = np.zeros(len(a), OCT_DTYPE)
    o["x"], o["y"], o["z"], o["lf"] = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    return o


def octs_to_u32(o):
    return np.stack([o["x"], o["y"], o["z"], o["lf"] & 31], 1).astype(np.uint32)


def p2o_cases():
    g = load("p2o_tiny")
    keys = sorted(k[:-4] for k in g if k.endswith("_pts"))
    return g, keys


def depth_of(key):
    return int(key.split("_d")[-1])


def table_digest(a):
    m = a.shape[-1]
    w = (7.0 * np.arange(m)[:, None] + 3.0 * np.arange(m)[None, :] + 1.0) / (10.0 * m)
    return np.stack([a.sum(axis=(2, 3)), (a * a).sum(axis=(2, 3)), np.abs(a).sum(axis=(2, 3)),
                     (a * w).sum(axis=(2, 3))], -1)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))
