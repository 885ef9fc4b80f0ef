"""GPU product against outputs of the reference itself (tests/golden/)."""
import numpy as np
import pytest

from tests.golden_data import MESH_CASES, depth_of, load, octs_to_u32, p2o_cases, rel, u32_to_octs

pytestmark = pytest.mark.gpu
TOL = 1e-12  # FP64 operators: relative 2-norm


def test_p2o_tiny_bitexact(gpu):
    g, keys = p2o_cases()
    for k in keys:
        d = depth_of(k)
        lin = gpu.points2Octree(g[k + "_pts"], d, 1)
        assert np.array_equal(octs_to_u32(lin.to_numpy()), g[k + "_p2o"]), k
        assert np.array_equal(octs_to_u32(gpu.balanceOctree(lin).to_numpy()), g[k + "_bal"]), k


@pytest.mark.parametrize("name", MESH_CASES)
def test_balance_coarsen_mesh_operators(gpu, name):
    import torch
    g = load("mesh_" + name)
    d = int(g["depth"])
    lin = gpu.Octree.from_octants(u32_to_octs(g["lin"]), d)
    bal = gpu.balanceOctree(lin)
    assert np.array_equal(octs_to_u32(bal.to_numpy()), g["bal"])
    assert np.array_equal(octs_to_u32(gpu.coarsenOctree(bal).to_numpy()), g["coarse"])
    da = gpu.DA(bal)
    ex = da.export()
    el = g["elem"]
    assert np.array_equal(ex["nlist"], el[:, 6:]) and np.array_equal(ex["hmask"], el[:, 5])
    assert np.array_equal(ex["cnum"], el[:, 4]) and np.array_equal(ex["level"], el[:, 3])
    assert np.array_equal(ex["node_xyz"], g["node_xyz"])
    x = torch.tensor(g["x"], device="cuda")
    assert rel(gpu.Jacobian2(da).mult(x).cpu().numpy(), g["y"]) < TOL
    assert rel(gpu.Jacobian2(da, g["coef"]).mult(x).cpu().numpy(), g["yc"]) < TOL
    x3 = torch.tensor(g["x3"], device="cuda")
    y3 = gpu.Elasticity(da, float(g["mu"]), float(g["lam"])).mult(x3).cpu().numpy()
    assert rel(y3, g["y3"]) < TOL


def test_transfer(gpu):
    g = load("transfer_gauss1k_d8")
    d, nl = int(g["depth"]), int(g["nlevels"])
    m = gpu.DAMG(gpu.Octree.from_octants(u32_to_octs(g["bal"]), d), nlevels=nl)
    assert m.nlevels == nl
    for l in range(nl):
        assert np.array_equal(m.level_da(l).export()["nlist"], g[f"elem{l}"][:, 6:])
    for l in range(nl - 1):
        assert rel(m.restrict(l, g[f"xf{l}"]), g[f"restrict{l}"]) < TOL
        xf0 = np.zeros(int(m.N[l]))
        assert rel(m.prolong(l, g[f"xc{l}"], xf0), g[f"prolong{l}"]) < TOL
