"""GPU mesh (ot::DA) maps against the oracle: bit-exact node map in anchor space."""
import numpy as np
import pytest

from tests.cases import points

pytestmark = pytest.mark.gpu

MESH_CASES = ["gauss2k_d8", "gauss20k_d10", "lognormal20k_d12", "uniform8k_d9_m4", "single_point",
              "corner_points_d5"]


def oracle_mesh(oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    return bal, d, oracle.Mesh(bal, d)


@pytest.mark.parametrize("name", MESH_CASES)
def test_mesh_maps_bitexact(gpu, oracle, name):
    bal, d, ref = oracle_mesh(oracle, name)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    assert (da.E, da.N) == (ref.E, ref.N)
    g = da.export()
    assert np.array_equal(g["node_xyz"], ref.node_xyz)
    assert np.array_equal(g["nlist"], ref.nlist)
    assert np.array_equal(g["hmask"], ref.hmask)
    assert np.array_equal(g["cnum"], ref.cnum)
    assert np.array_equal(g["etype"], ref.etype)
    assert np.array_equal(g["level"], ref.elev)
    assert np.array_equal(g["node_bdy"], ref.node_bdy)
    # element anchors are the embedded input octants
    assert np.array_equal(g["elem_xyz"], np.stack([bal["x"], bal["y"], bal["z"]], 1))


def test_unbalanced_octree_rejected(gpu, oracle):
    pts, d, m = points("gauss20k_d10")
    lin = oracle.points2octree(pts, d, m)
    bal = oracle.balance(lin, d)
    if len(bal) == len(lin):
        pytest.skip("input already balanced")
    with pytest.raises(gpu.DendroError):
        gpu.DA(gpu.Octree.from_octants(lin, d))
