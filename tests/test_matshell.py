"""The reference-side PETSc binding (include/dendro_b200_matshell.hpp):
compiled against the project's single-rank PETSc stand-ins
(oracle/ref_build/shim) into a driver that wraps the GPU operators in a
MatShell and drives them through MatMult and MatGetDiagonal, as
CreateJacobian2 / CreateElasticityMat (examples/src/backend/omgNeumann.C:
643-745, elasticityJac.C) do.  The products are compared with the
reference's own Jacobian2MatMult / ElasticityMatMult outputs
(tests/golden/mesh_*.npz) and the diagonals with the oracle's."""
import os
import subprocess

import numpy as np
import pytest

from tests.golden_data import MESH_CASES, load, rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_driver(out_dir):
    from dendro_b200 import build
    so = build.build()
    exe = os.path.join(out_dir, "matshell_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "oracle", "ref_build", "shim"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "matshell", "matshell_driver.cpp"), "-L", os.path.dirname(so),
           "-ldendro_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{os.path.dirname(so)}",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_matshell_binding_compiles(tmp_path):
    assert os.path.exists(build_driver(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", MESH_CASES)
def test_matshell_through_matmult(gpu, oracle, tmp_path, name):
    from tests.golden_data import u32_to_octs
    exe = build_driver(str(tmp_path))
    g = load("mesh_" + name)
    d = int(g["depth"])
    octs = str(tmp_path / "bal.u32")
    g["bal"].astype(np.uint32).tofile(octs)
    M = oracle.Mesh(u32_to_octs(g["bal"]), d)

    def run(*args):
        r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]

    x, coef = str(tmp_path / "x.f64"), str(tmp_path / "coef.f64")
    g["x"].tofile(x)
    g["coef"].tofile(coef)
    y, dg = str(tmp_path / "y.f64"), str(tmp_path / "d.f64")
    for cpath, yref, cf in (("none", g["y"], None), (coef, g["yc"], g["coef"])):
        run("lapmass", octs, d, x, cpath, y, dg)
        assert rel(np.fromfile(y), yref) < 1e-12
        assert rel(np.fromfile(dg), M.diagonal(cf)) < 1e-12
    x3 = str(tmp_path / "x3.f64")
    g["x3"].tofile(x3)
    run("elastic", octs, d, x3, float(g["mu"]), float(g["lam"]), y, dg)
    assert rel(np.fromfile(y), g["y3"]) < 1e-12


@pytest.mark.gpu
def test_transfer_shell_through_matmult(gpu, tmp_path):
    """R as a MatShell (src/omg/omg.C:2278-2283): MatMult restricts, MatMultTranspose
    prolongs, the ADD forms add to another Vec; against the reference's own
    restrictMatVecType1 / prolongMatVecType1 outputs."""
    exe = build_driver(str(tmp_path))
    g = load("transfer_gauss1k_d8")
    d, nl = int(g["depth"]), int(g["nlevels"])
    octs = str(tmp_path / "bal.u32")
    g["bal"].astype(np.uint32).tofile(octs)
    for l in range(nl - 1):
        xf, xc, out = str(tmp_path / "xf.f64"), str(tmp_path / "xc.f64"), str(tmp_path / f"t{l}")
        g[f"xf{l}"].tofile(xf)
        g[f"xc{l}"].tofile(xc)
        r = subprocess.run([exe, "transfer", octs, str(d), str(nl), str(l), xf, xc, out],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        assert rel(np.fromfile(out + ".R"), g[f"restrict{l}"]) < 1e-12
        assert rel(np.fromfile(out + ".P"), g[f"prolong{l}"]) < 1e-12
        assert rel(np.fromfile(out + ".RA") - 1.0, g[f"restrict{l}"]) < 1e-12
        assert rel(np.fromfile(out + ".PA") - 1.0, g[f"prolong{l}"]) < 1e-12
