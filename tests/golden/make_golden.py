"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs oracle/_ref/dendro_ref -- the reference's own octree, mesh, operator and
transfer sources compiled single-rank by oracle/ref_build/build_ref.py -- on
seeded inputs and stores its outputs as compressed .npz files, plus digests
of the reference's stencil tables (Stencils/*.inp).  Needs the reference
tree and the reference build; the fixtures it writes are committed and the
tests read only them.

    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py --io-only  # the file-format fixtures io_*.npz
    python tests/golden/make_golden.py --jac3-only  # Jacobian3 fixture + stencil digests
    python tests/golden/make_golden.py --dirichlet-only  # Dirichlet operator fixtures

The file-format fixtures also run oracle/_ref/dendro_ref_dumpmesh, the
reference's examples/src/drivers/dumpMesh.C built single-rank.

Inputs whose linear octree the reference cannot produce (its points2Octree
does not terminate above 8 points at its HEAD) start from the oracle's
linear octree; the reference then balances, coarsens, meshes, applies the
operators and the transfers.
"""
from __future__ import annotations

import hashlib
import math
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dendro_b200 import inputs as I  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "dendro_ref")
REF_CWD = os.path.join(ROOT, "oracle", "_ref", "stencils")
STENCILS = os.path.join(os.environ.get("DENDRO_REFERENCE", "/root/reference"), "Stencils")

MU, LAM = 1.0 / (2.0 * 1.3), 0.3 / (1.3 * 0.4)  # E = 1, nu = 0.3


def run(*args, timeout=3600):
    r = subprocess.run([REF_BIN, *map(str, args)], cwd=REF_CWD, capture_output=True, text=True, timeout=timeout)
    if r.returncode:
        raise RuntimeError(f"reference run {args[0]} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stderr


def octs_to_u32(o):
    return np.stack([o["x"], o["y"], o["z"], o["lf"] & 31], 1).astype(np.uint32)


def read_octs(path):
    return np.fromfile(path, np.uint32).reshape(-1, 4)


P2O_CASES = [(n, seed, depth) for n in (4, 8) for seed in range(4) for depth in (6, 10)]

MESH_CASES = {
    "corner_points_d5": lambda: (np.array([[0, 0, 0], [1 - 2.0 ** -6] * 3, [0.5, 0.5, 0.5], [0.49, 0.51, 0.5]]), 5),
    "uniform600_d7": lambda: (I.clamp_unit(I.uniform_cloud(600, 11), 7), 7),
    "gauss1k_d8": lambda: (I.clamp_unit(I.gaussian_cloud(1000, 12), 8), 8),
    "lognormal1k_d10": lambda: (I.clamp_unit(I.lognormal_cloud(1000, 13), 10), 10),
}
TRANSFER_CASE = ("gauss1k_d8", 3)


def p2o_fixture(tmp):
    rec = {}
    for n, seed, depth in P2O_CASES:
        pts = np.random.default_rng(1000 + 17 * n + seed).uniform(0, 1, (n, 3))
        pts.tofile(os.path.join(tmp, "pts.f64"))
        try:
            run("octree", os.path.join(tmp, "pts.f64"), depth, 1, tmp, timeout=20)
        except subprocess.TimeoutExpired:
            print(f"points2Octree did not terminate: n={n} seed={seed} depth={depth}")
            continue
        key = f"n{n}_s{seed}_d{depth}"
        rec[key + "_pts"] = pts
        rec[key + "_p2o"] = read_octs(os.path.join(tmp, "p2o.u32"))
        rec[key + "_bal"] = read_octs(os.path.join(tmp, "bal.u32"))
    np.savez_compressed(os.path.join(OUT, "p2o_tiny.npz"), **rec)


def mesh_fixture(tmp, name):
    pts, depth = MESH_CASES[name]()
    lin = O.points2octree(pts, depth, 1)
    octs_to_u32(lin).tofile(os.path.join(tmp, "lin.u32"))
    run("balance", os.path.join(tmp, "lin.u32"), depth, tmp)
    bal = read_octs(os.path.join(tmp, "bal.u32"))
    coarse = read_octs(os.path.join(tmp, "coarse.u32"))
    bal.tofile(os.path.join(tmp, "bal_in.u32"))
    run("mesh", os.path.join(tmp, "bal_in.u32"), depth, tmp)
    elem = np.fromfile(os.path.join(tmp, "elem.u32"), np.uint32).reshape(-1, 14)
    node_xyz = np.fromfile(os.path.join(tmp, "node_xyz.u32"), np.uint32).reshape(-1, 3)
    N = len(node_xyz)
    x = np.random.default_rng(7).uniform(-1, 1, N)
    x.tofile(os.path.join(tmp, "x.f64"))
    run("matvec", os.path.join(tmp, "bal_in.u32"), depth, os.path.join(tmp, "x.f64"), "none",
        os.path.join(tmp, "y.f64"))
    y = np.fromfile(os.path.join(tmp, "y.f64"))
    # variable coefficients: a = 1e4 inside the sphere r < 0.25, b = 1
    s = 2.0 ** -(elem[:, 3].astype(np.float64) - 1)
    cen = elem[:, :3] / 2.0 ** depth + 0.5 * s[:, None]
    coef = I.sphere_coefficients(cen)
    coef.tofile(os.path.join(tmp, "coef.f64"))
    run("matvec", os.path.join(tmp, "bal_in.u32"), depth, os.path.join(tmp, "x.f64"), os.path.join(tmp, "coef.f64"),
        os.path.join(tmp, "yc.f64"))
    yc = np.fromfile(os.path.join(tmp, "yc.f64"))
    x3 = np.random.default_rng(8).uniform(-1, 1, 3 * N)
    x3.tofile(os.path.join(tmp, "x3.f64"))
    run("elastic", os.path.join(tmp, "bal_in.u32"), depth, os.path.join(tmp, "x3.f64"), os.path.join(tmp, "y3.f64"))
    y3 = np.fromfile(os.path.join(tmp, "y3.f64"))
    np.savez_compressed(os.path.join(OUT, f"mesh_{name}.npz"), depth=depth, lin=octs_to_u32(lin), bal=bal,
                        coarse=coarse, elem=elem, node_xyz=node_xyz, x=x, y=y, coef=coef, yc=yc, x3=x3, y3=y3,
                        mu=MU, lam=LAM)


def transfer_fixture(tmp):
    name, nlevels = TRANSFER_CASE
    pts, depth = MESH_CASES[name]()
    bal = O.balance(O.points2octree(pts, depth, 1), depth)
    octs_to_u32(bal).tofile(os.path.join(tmp, "bal_t.u32"))
    dm = O.DAMG(bal, depth, nlevels)
    rec = {"depth": depth, "nlevels": dm.nlevels}
    for l in range(dm.nlevels - 1):
        xf = np.random.default_rng(30 + l).uniform(-1, 1, int(dm.N[l]))
        xc = np.random.default_rng(40 + l).uniform(-1, 1, int(dm.N[l + 1]))
        xf.tofile(os.path.join(tmp, f"level{l}_in.f64"))
        xc.tofile(os.path.join(tmp, f"coarse{l}_in.f64"))
        rec[f"xf{l}"], rec[f"xc{l}"] = xf, xc
    run("transfer", os.path.join(tmp, "bal_t.u32"), depth, nlevels, tmp)
    for l in range(dm.nlevels):
        rec[f"elem{l}"] = np.fromfile(os.path.join(tmp, f"level{l}_elem.u32"), np.uint32).reshape(-1, 14)
        rec[f"node_xyz{l}"] = np.fromfile(os.path.join(tmp, f"level{l}_node_xyz.u32"), np.uint32).reshape(-1, 3)
    for l in range(dm.nlevels - 1):
        rec[f"restrict{l}"] = np.fromfile(os.path.join(tmp, f"restrict{l}.f64"))
        rec[f"prolong{l}"] = np.fromfile(os.path.join(tmp, f"prolong{l}.f64"))
    rec["bal"] = octs_to_u32(bal)
    np.savez_compressed(os.path.join(OUT, f"transfer_{name}.npz"), **rec)


def elastic_transfer_fixture(tmp):
    """The reference's intergrid transfers of 3-dof vectors in the elasticity
    solver's set-up order (dof 3, suppressed DOFs, elasticity contexts) and
    each level's boundary flags, on the transfer case's hierarchy."""
    name, nlevels = TRANSFER_CASE
    pts, depth = MESH_CASES[name]()
    bal = O.balance(O.points2octree(pts, depth, 1), depth)
    octs_to_u32(bal).tofile(os.path.join(tmp, "bal_e.u32"))
    dm = O.DAMG(bal, depth, nlevels)
    rec = {"depth": depth, "nlevels": dm.nlevels, "bal": octs_to_u32(bal)}
    for l in range(dm.nlevels - 1):
        xf = np.random.default_rng(60 + l).uniform(-1, 1, 3 * int(dm.N[l]))
        xc = np.random.default_rng(70 + l).uniform(-1, 1, 3 * int(dm.N[l + 1]))
        xf.tofile(os.path.join(tmp, f"level{l}_in.f64"))  # inputs are regenerated from the seeds
        xc.tofile(os.path.join(tmp, f"coarse{l}_in.f64"))
    run("elastic_transfer", os.path.join(tmp, "bal_e.u32"), depth, nlevels, tmp)
    for l in range(dm.nlevels):
        rec[f"bdy{l}"] = np.fromfile(os.path.join(tmp, f"bdy{l}.u8"), np.uint8)
    for l in range(dm.nlevels - 1):
        rec[f"restrict{l}"] = np.fromfile(os.path.join(tmp, f"restrict{l}.f64"))
        rec[f"prolong{l}"] = np.fromfile(os.path.join(tmp, f"prolong{l}.f64"))
    np.savez_compressed(os.path.join(OUT, f"elastic_transfer_{name}.npz"), **rec)


def dirichlet_fixture(tmp, name):
    """The reference's boundary flags (assignBoundaryFlags) and its Dirichlet
    Laplacian / Jacobian MatMult and GetDiagonal on the mesh case."""
    z = np.load(os.path.join(OUT, f"mesh_{name}.npz"))
    z["bal"].astype(np.uint32).tofile(os.path.join(tmp, "bal_d.u32"))
    z["x"].tofile(os.path.join(tmp, "x_d.f64"))
    run("dirichlet", os.path.join(tmp, "bal_d.u32"), int(z["depth"]), os.path.join(tmp, "x_d.f64"), tmp)
    rd = lambda f, dt=np.float64: np.fromfile(os.path.join(tmp, f), dt)  # noqa: E731
    np.savez_compressed(os.path.join(OUT, f"dirichlet_{name}.npz"), bdy=rd("bdy.u8", np.uint8), x=z["x"],
                        yL=rd("yL.f64"), yJ=rd("yJ.f64"), dL=rd("dL.f64"), dJ=rd("dJ.f64"))


def jac3_fixture(tmp):
    """Jacobian3MatMult (examples/src/backend/omgJac.C:2235) on the coarse
    levels of the transfer case's hierarchy, from the next finer level's
    coefficients: the sphere coefficients (a = 1e4 inside r < 0.25) on the
    finest level, their per-level means below."""
    name, nlevels = TRANSFER_CASE
    z = np.load(os.path.join(OUT, f"transfer_{name}.npz"))
    depth, bal = int(z["depth"]), z["bal"]
    nl = int(z["nlevels"])
    bal.tofile(os.path.join(tmp, "bal_j.u32"))
    dm = O.DAMG(bal.view(np.uint32).reshape(-1, 4).astype(np.uint32).view(O.OCT_DTYPE).reshape(-1), depth, nlevels)
    assert dm.nlevels == nl
    rec = {"depth": depth, "nlevels": nl, "bal": bal}
    e0 = z["elem0"]
    s0 = 2.0 ** -(e0[:, 3].astype(np.float64) - 1)
    coef = I.sphere_coefficients(e0[:, :3] / 2.0 ** depth + 0.5 * s0[:, None]).reshape(-1)
    for l in range(nl - 1):
        rec[f"coef{l}"] = coef
        coef.tofile(os.path.join(tmp, f"coef{l}.f64"))
        x = np.random.default_rng(50 + l).uniform(-1, 1, int(dm.N[l + 1]))
        rec[f"jin{l + 1}"] = x
        x.tofile(os.path.join(tmp, f"jin{l + 1}.f64"))
        coef = O.coarse_coef(dm.level_mesh(l), coef, dm.level_mesh(l + 1)).reshape(-1)
    run("jac3", os.path.join(tmp, "bal_j.u32"), depth, nl, tmp)
    for l in range(1, nl):
        rec[f"jout{l}"] = np.fromfile(os.path.join(tmp, f"jout{l}.f64"))
    np.savez_compressed(os.path.join(OUT, f"jac3_{name}.npz"), **rec)


IO_CASES = ["corner_points_d5", "uniform600_d7", "gauss1k_d8"]
DUMP_BIN = os.path.join(ROOT, "oracle", "_ref", "dendro_ref_dumpmesh")


def io_fixture(tmp, name):
    """The reference's file writers and readers (src/oct/OctFunctions.C:313-439)
    on the mesh case's points and balanced octree, and its mesh dump
    (examples/src/drivers/dumpMesh.C, one rank) of that octree."""
    z = np.load(os.path.join(OUT, f"mesh_{name}.npz"))
    bal, depth = z["bal"], int(z["depth"])
    pts = MESH_CASES[name]()[0]
    vals = np.random.default_rng(21).uniform(-1, 1, len(pts))
    bal.astype(np.uint32).tofile(os.path.join(tmp, "octs.u32"))
    pts.astype(np.float64).tofile(os.path.join(tmp, "pts.f64"))
    vals.tofile(os.path.join(tmp, "vals.f64"))
    run("io", os.path.join(tmp, "octs.u32"), depth, os.path.join(tmp, "pts.f64"), os.path.join(tmp, "vals.f64"), tmp)
    rd = lambda f, dt=np.uint8: np.fromfile(os.path.join(tmp, f), dt)  # noqa: E731
    assert np.array_equal(rd("octs_rt.u32", np.uint32).reshape(-1, 4), bal)
    assert np.array_equal(rd("pts_rt.f64", np.float64).reshape(-1, 3), pts)
    assert np.array_equal(rd("data_vals_rt.f64", np.float64), vals)
    shutil.copy(os.path.join(tmp, "octs.ot"), os.path.join(tmp, "m0_1.ot"))
    r = subprocess.run([DUMP_BIN, os.path.join(tmp, "m")], cwd=REF_CWD, capture_output=True, text=True, timeout=600)
    if r.returncode:
        raise RuntimeError(f"reference dumpMesh failed ({r.returncode}): {r.stderr[-2000:]}")
    np.savez_compressed(os.path.join(OUT, f"io_{name}.npz"), depth=depth, bal=bal, pts=pts, vals=vals,
                        ot=rd("octs.ot"), pts_file=rd("pts.pts"), data_file=rd("data.pts"),
                        nl=rd("m_NL_0_1.out"), el=rd("m_EL_0_1.out"), m=rd("m_M_0_1.out"))


CFG1 = "gauss131k_d10"  # 131,072 points N(0.5, 0.1) (seed 0), maxDepth 10
CFG1_PROJECTIONS = 4


def digest(a):
    """sha256 of an array's uint32 bytes (C order)."""
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def projections(y, k=CFG1_PROJECTIONS, seed=77):
    """y projected on k seeded unit vectors (a size-independent check of y)."""
    g = np.random.default_rng(seed).normal(size=(k, len(y)))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    return np.array([math.fsum(gi * y) for gi in g])


def cfg1_fixture(tmp):
    """The reference at the full size of the small configuration: its balance of
    the oracle's linear octree, its DA maps and one Jacobian2MatMult with
    constant coefficients (x = U[-1, 1], seed 1), kept as digests (sha256 of the
    integer arrays; norm, sum and seeded projections of y) because the arrays
    themselves run to tens of megabytes."""
    pts, depth = I.workload_points(CFG1)
    lin = O.points2octree(pts, depth, 1)
    octs_to_u32(lin).tofile(os.path.join(tmp, "lin.u32"))
    run("balance", os.path.join(tmp, "lin.u32"), depth, tmp)
    bal = read_octs(os.path.join(tmp, "bal.u32"))
    bal.tofile(os.path.join(tmp, "bal_in.u32"))
    run("mesh", os.path.join(tmp, "bal_in.u32"), depth, tmp)
    elem = np.fromfile(os.path.join(tmp, "elem.u32"), np.uint32).reshape(-1, 14)
    node_xyz = np.fromfile(os.path.join(tmp, "node_xyz.u32"), np.uint32).reshape(-1, 3)
    N = len(node_xyz)
    x = I.uniform_rhs(N, 1)
    x.tofile(os.path.join(tmp, "x.f64"))
    run("matvec", os.path.join(tmp, "bal_in.u32"), depth, os.path.join(tmp, "x.f64"), "none",
        os.path.join(tmp, "y.f64"))
    y = np.fromfile(os.path.join(tmp, "y.f64"))
    np.savez_compressed(os.path.join(OUT, f"cfg1_{CFG1}.npz"), depth=depth, n_lin=len(lin), n_bal=len(bal),
                        E=len(elem), N=N, bal_sha=digest(bal), maps_sha=digest(elem[:, 3:]),
                        node_sha=digest(node_xyz), y_norm=np.linalg.norm(y), y_sum=math.fsum(y),
                        y_proj=projections(y))


def table_digest(a):
    """Checksums of each (child number, type) table: sum, sum of squares,
    sum of magnitudes and a position-weighted sum."""
    m = a.shape[-1]
    w = (7.0 * np.arange(m)[:, None] + 3.0 * np.arange(m)[None, :] + 1.0) / (10.0 * m)
    return np.stack([a.sum(axis=(2, 3)), (a * a).sum(axis=(2, 3)), np.abs(a).sum(axis=(2, 3)),
                     (a * w).sum(axis=(2, 3))], -1)


def vector_digest(a):
    """Checksums of each (child number, type) vector: sum, sum of squares, sum of
    magnitudes and a position-weighted sum."""
    m = a.shape[-1]
    w = (7.0 * np.arange(m) + 1.0) / (10.0 * m)
    return np.stack([a.sum(-1), (a * a).sum(-1), np.abs(a).sum(-1), (a * w).sum(-1)], -1)


def stencil_digests():
    """Checksums of the reference's Laplacian, mass, grad-div and same-level
    restriction tables (Stencils/*Type2Stencils.inp)."""
    rec = {}
    for tag, fname, m in (("lap", "LapType2Stencils.inp", 8), ("mass", "MassType2Stencils.inp", 8),
                          ("gd", "GDType2Stencils.inp", 24), ("rmat2", "RmatType2Stencils.inp", 8)):
        a = np.array(open(os.path.join(STENCILS, fname)).read().split(), float).reshape(8, 18, m, m)
        rec[tag] = table_digest(a)
    # RHSType2Stencil [child][type][vertex] (ComputeRHS_omgNeumann's load table)
    r = np.array(open(os.path.join(STENCILS, "RHSType2Stencils.inp")).read().split(), float).reshape(8, 18, 8)
    rec["rhs"] = vector_digest(r)
    # type-1 tables [coarse child][type][fine child][8][8], digested per (type, fine child)
    for tag, fname in (("lap1", "LapType1Stencils.inp"), ("mass1", "MassType1Stencils.inp")):
        a = np.array(open(os.path.join(STENCILS, fname)).read().split(), float).reshape(8, 18 * 8, 8, 8)
        rec[tag] = table_digest(a)
    np.savez_compressed(os.path.join(OUT, "stencil_digests.npz"), **rec)


def main():
    if not os.path.exists(REF_BIN):
        sys.exit("build the reference first: python oracle/ref_build/build_ref.py")
    if "--stencils-only" in sys.argv:
        stencil_digests()
        return
    if "--dirichlet-only" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            for name in MESH_CASES:
                dirichlet_fixture(tmp, name)
        return
    if "--jac3-only" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            jac3_fixture(tmp)
        stencil_digests()
        return
    if "--elastic-only" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            elastic_transfer_fixture(tmp)
        return
    if "--cfg1-only" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            cfg1_fixture(tmp)
        return
    if "--io-only" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            for name in IO_CASES:
                io_fixture(tmp, name)
        return
    with tempfile.TemporaryDirectory() as tmp:
        p2o_fixture(tmp)
        for name in MESH_CASES:
            mesh_fixture(tmp, name)
        transfer_fixture(tmp)
        jac3_fixture(tmp)
        for name in MESH_CASES:
            dirichlet_fixture(tmp, name)
        for name in IO_CASES:
            io_fixture(tmp, name)
        cfg1_fixture(tmp)
        elastic_transfer_fixture(tmp)
    stencil_digests()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
