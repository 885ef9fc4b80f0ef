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


def test_single_octant_mesh(gpu, oracle, tmp_path):
    """The root octant alone (an empty point set): one element, its 8 nodes;
    operator, diagonal and a solve against the oracle.  The hierarchy keeps its
    first coarsening (the root again) before it stops, as the oracle's and the
    reference's DAMGCreateAndSetDA do: two identical levels."""
    import numpy as np
    from dendro_b200 import inputs as I
    d = 6
    root = oracle.points2octree(np.zeros((0, 3)), d, 1)
    ref = oracle.Mesh(root, d)
    da = gpu.DA(gpu.Octree.from_octants(root, d))
    assert (da.E, da.N) == (ref.E, ref.N) == (1, 8)
    x = I.uniform_rhs(ref.N, 5)
    A = gpu.Jacobian2(da)
    assert np.linalg.norm(A.mult(x) - ref.matvec(x)) <= 1e-12 * np.linalg.norm(ref.matvec(x))
    assert np.linalg.norm(A.getDiagonal().cpu().numpy() - ref.diagonal()) <= 1e-12 * np.linalg.norm(ref.diagonal())
    m = gpu.DAMG(gpu.Octree.from_octants(root, d))
    assert m.nlevels == oracle.DAMG(root, d, 30).nlevels == 2
    xs, rep = m.solve(x)
    assert rep["converged"]
    assert np.linalg.norm(ref.matvec(xs) - x) <= 1e-8 * np.linalg.norm(x)
    da.dumpMesh(str(tmp_path / "m"))
    assert np.fromfile(tmp_path / "m_M_0_1.out", np.uint32).tolist() == [1, 0, 0, 1, 2, 3, 4, 5, 6, 7]
