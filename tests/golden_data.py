"""Loaders of the reference-generated golden fixtures (tests/golden/*.npz)."""
import hashlib
import math
import os
import subprocess
import tempfile

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


# ---- the small configuration at full size (tests/golden/cfg1_gauss131k_d10.npz) ----
CFG1 = "gauss131k_d10"
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "dendro_ref")
REF_CWD = os.path.join(ROOT, "oracle", "_ref", "stencils")


def digest(a):
    """sha256 of an array's uint32 bytes (C order), as make_golden.py writes them."""
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def projections(y, k=4, seed=77):
    """y projected on k seeded unit vectors, as make_golden.py writes them."""
    g = np.random.default_rng(seed).normal(size=(k, len(y)))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    return np.array([math.fsum(gi * y) for gi in g])


def maps_table(level, cnum, hmask, nlist):
    """The reference DA dump's per-element columns 3.. (level, child number,
    hanging mask, 8 node ids) as one uint32 table."""
    return np.column_stack([level, cnum, hmask, nlist]).astype(np.uint32)


def check_y_digest(y, g):
    """y against the reference's stored norm and projections: the projections
    of an error e of y are about |e| / sqrt(N), so agreement to 1e-12 |y|
    rules out errors above roughly 1e-9 |y| (the 1e-12 comparison itself is
    made against the reference binary or the oracle)."""
    ny = float(g["y_norm"])
    assert abs(np.linalg.norm(y) - ny) <= 1e-12 * ny
    assert np.max(np.abs(projections(y) - g["y_proj"])) <= 1e-12 * ny


def reference_matvec(bal_u32, depth, x, coef=None):
    """y from the reference's own Jacobian2MatMult (the compiled reference,
    oracle/_ref/dendro_ref), or None when that binary is absent."""
    if not os.path.exists(REF_BIN):
        return None
    with tempfile.TemporaryDirectory() as tmp:
        np.ascontiguousarray(bal_u32, np.uint32).tofile(os.path.join(tmp, "bal.u32"))
        np.ascontiguousarray(x, np.float64).tofile(os.path.join(tmp, "x.f64"))
        cpath = "none"
        if coef is not None:
            cpath = os.path.join(tmp, "coef.f64")
            np.ascontiguousarray(coef, np.float64).tofile(cpath)
        r = subprocess.run([REF_BIN, "matvec", os.path.join(tmp, "bal.u32"), str(depth), os.path.join(tmp, "x.f64"),
                            cpath, os.path.join(tmp, "y.f64")], cwd=REF_CWD, capture_output=True, text=True,
                           timeout=1200)
        assert r.returncode == 0, r.stderr[-2000:]
        return np.fromfile(os.path.join(tmp, "y.f64"))


def elastic_inputs(g, sizes):
    """The seeded 3-dof inputs of the elastic transfer fixture (fine, coarse)
    per level, as make_golden.py drew them; sizes = node counts per level."""
    out = []
    for l in range(int(g["nlevels"]) - 1):
        xf = np.random.default_rng(60 + l).uniform(-1, 1, 3 * int(sizes[l]))
        xc = np.random.default_rng(70 + l).uniform(-1, 1, 3 * int(sizes[l + 1]))
        out.append((xf, xc))
    return out
