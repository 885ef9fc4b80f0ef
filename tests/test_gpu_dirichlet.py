"""Dirichlet Laplacian / Jacobian operators and diagonals on the GPU against
the reference's own MatMult / GetDiagonal (golden fixtures) and the oracle."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points
from tests.golden_data import MESH_CASES, load, rel, u32_to_octs

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("name", MESH_CASES)
def test_dirichlet_operators_match_reference(gpu, name):
    g, m = load("dirichlet_" + name), load("mesh_" + name)
    da = gpu.DA(gpu.Octree.from_octants(u32_to_octs(m["bal"]), int(m["depth"])))
    assert np.array_equal(da.export()["node_bdy"] != 0, g["bdy"] != 0)
    for cls, y, d in ((gpu.DirichletLaplacian, "yL", "dL"), (gpu.DirichletJacobian, "yJ", "dJ")):
        A = cls(da)  # default flags: the domain-boundary nodes, as assignBoundaryFlags
        assert rel(A.mult(g["x"]), g[y]) < TOL, y
        assert rel(A.getDiagonal().cpu().numpy(), g[d]) < TOL, d


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12"])
def test_dirichlet_operators_match_oracle(gpu, oracle, name):
    """With flags of the caller's choosing (a seeded random set of nodes)."""
    import torch
    pts, d, mx = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, mx), d)
    ref = oracle.Mesh(bal, d)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    bdy = (np.random.default_rng(11).uniform(size=ref.N) < 0.1).astype(np.uint8)
    x = I.uniform_rhs(ref.N, 12)
    for cls, mass in ((gpu.DirichletLaplacian, False), (gpu.DirichletJacobian, True)):
        A = cls(da, bdy)
        y = A.mult(torch.tensor(x, device="cuda")).cpu().numpy()
        assert rel(y, ref.dirichlet_matvec(x, bdy, mass)) < TOL
        assert rel(A.getDiagonal().cpu().numpy(), ref.dirichlet_diagonal(bdy, mass)) < TOL
