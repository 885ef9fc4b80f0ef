"""GPU: the dof-3 multigrid (DAMGCreateAndSetDA with dof 3, linear elasticity
on every level with that level's boundary nodes Dirichlet, as
examples/src/drivers/newElasSolver.C:279-361 sets it up) against the
oracle's restatement of the same hierarchy: level sizes, the transfers per
component, one V(2,2) cycle, and PCG to 1e-8 (iterations within one of the
oracle's, FP64 true residual, error against the oracle's solution)."""
import numpy as np
import pytest

from tests.cases import points
from tests.golden_data import rel

pytestmark = pytest.mark.gpu
MU, LAM = 1.0 / (2.0 * 1.3), 0.3 / (1.3 * 0.4)  # E = 1, nu = 0.3


@pytest.mark.parametrize("name,nlevels", [("gauss2k_d8", 3), ("lognormal20k_d12", 5), ("corner_points_d5", 2)])
def test_elasticity_multigrid(gpu, oracle, name, nlevels):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    tree = gpu.Octree.from_octants(bal, d)
    mg = gpu.DAMG(tree, nlevels=nlevels, dof=3, mu=MU, lam=LAM)
    H = oracle.DAMG(bal, d, nlevels, dof=3, mu=MU, lam=LAM)
    assert mg.nlevels == H.nlevels and list(mg.N) == [int(v) for v in H.N]
    rng = np.random.default_rng(5)
    meshes = [H.level_mesh(l) for l in range(H.nlevels)]
    for l in range(mg.nlevels - 1):
        rf = rng.uniform(-1, 1, 3 * int(mg.N[l]))
        rc = mg.restrict(l, rf)
        assert rc.shape == (3 * int(mg.N[l + 1]),)
        # per component: the oracle's scalar restriction P^T of each component
        ptr, col, val = oracle.prolongation(meshes[l], meshes[l + 1])
        rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
        for c in range(3):
            want = np.zeros(int(mg.N[l + 1]))
            np.add.at(want, col, val * rf[c::3][rows])
            assert rel(rc[c::3], want) < 1e-12, (l, c)
    b = rng.uniform(-1, 1, 3 * int(mg.N[0]))
    import torch

    from dendro_b200.learned import vcycle
    z = vcycle(mg, torch.tensor(b, device="cuda"))
    assert rel(z.cpu().numpy(), H.vcycle(b)) < 1e-10
    x, rep = mg.solve(b)
    x_orc, it_orc, _ = H.pcg(b, 1e-8, 300)
    mesh = H.level_mesh(0)
    res = np.linalg.norm(mesh.elasticity_matvec(x, MU, LAM) - b) / np.linalg.norm(b)
    assert rep["converged"] and res <= 1e-8, (rep, res)
    assert abs(rep["iterations"] - it_orc) <= 1, (rep["iterations"], it_orc)
    assert rel(x, x_orc) < 1e-6


def test_elastic_transfer_golden(gpu):
    """The dof-3 hierarchy's transfers against the reference's own, run in its
    elasticity solver's set-up order (tests/golden/elastic_transfer_*.npz)."""
    from tests.golden_data import elastic_inputs, load, u32_to_octs
    g = load("elastic_transfer_gauss1k_d8")
    d, nl = int(g["depth"]), int(g["nlevels"])
    mg = gpu.DAMG(gpu.Octree.from_octants(u32_to_octs(g["bal"]), d), nlevels=nl, dof=3, mu=MU, lam=LAM)
    assert mg.nlevels == nl
    for l, (xf, xc) in enumerate(elastic_inputs(g, mg.N)):
        assert rel(mg.restrict(l, xf), g[f"restrict{l}"]) < 1e-12
        assert rel(mg.prolong(l, xc, np.zeros(3 * int(mg.N[l]))), g[f"prolong{l}"]) < 1e-12
