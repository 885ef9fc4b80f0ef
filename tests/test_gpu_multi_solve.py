"""GPU: many right-hand sides solved together (dg_damg_solve_multi) against
the single-right-hand-side solve column by column: every column converged,
its FP64 true residual at the tolerance (oracle operator), its solution
within 1e-6 of the single solve's, in the FP64 and the FP32 inner cycle."""
import numpy as np
import pytest

from tests.cases import points

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nrhs,inner", [("lognormal20k_d12", 32, 1), ("gauss20k_d10", 64, 0),
                                             ("corner_points_d5", 32, 1)])
def test_multi_solve_matches_single(gpu, oracle, name, nrhs, inner):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    tree = gpu.Octree.from_octants(bal, d)
    mg = gpu.DAMG(tree, inner_prec=inner)
    N = int(mg.N[0])
    B = np.random.default_rng(6).uniform(-1, 1, (N, nrhs))
    X, rep = mg.solve_multi(B)
    assert rep["converged"] and rep["rel_residual"] <= 1e-8
    mesh = oracle.Mesh(bal, d)
    single = gpu.DAMG(tree, inner_prec=inner)
    for j in range(0, nrhs, max(1, nrhs // 8)):
        res = np.linalg.norm(mesh.matvec(X[:, j]) - B[:, j]) / np.linalg.norm(B[:, j])
        assert res <= 1.01e-8, (j, res)
        xs, _ = single.solve(B[:, j])
        assert np.linalg.norm(X[:, j] - xs) <= 1e-6 * np.linalg.norm(xs), j


def test_multi_solve_rejects_bad_counts(gpu, oracle):
    pts, d, m = points("corner_points_d5")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    mg = gpu.DAMG(gpu.Octree.from_octants(bal, d))
    with pytest.raises(gpu.DendroError):
        mg.solve_multi(np.zeros((int(mg.N[0]), 48)))
