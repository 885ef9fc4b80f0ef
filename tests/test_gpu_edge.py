"""The smallest mesh, the root octant alone (one element in a tile of 32):
every operator launch shape, the multi-right-hand-side kernels, the Dirichlet
and elasticity operators (all 8 nodes on the domain boundary) and a
mixed-precision solve replayed from a CUDA graph, against the oracle."""
import numpy as np
import pytest

from dendro_b200 import inputs as I

pytestmark = pytest.mark.gpu

D = 6


def root_mesh(gpu, oracle):
    root = oracle.points2octree(np.zeros((0, 3)), D, 1)
    return root, oracle.Mesh(root, D), gpu.DA(gpu.Octree.from_octants(root, D))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_every_launch_shape_on_one_element(gpu, oracle):
    import torch
    _, ref, da = root_mesh(gpu, oracle)
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 2)
    y_ref = ref.matvec(x, coef)
    A = gpu.Jacobian2(da, coef)
    xd = torch.tensor(x, device="cuda")
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        A.set_kernel(v, 1)
        assert rel(A.mult(xd).cpu().numpy(), y_ref) < 1e-12, v
        assert rel(A.mult(xd.float()).double().cpu().numpy(), y_ref) < 2e-6, v
    gpu.deviceCheck()


@pytest.mark.parametrize("nrhs", [16, 32, 64, 96])
def test_multi_rhs_on_one_element(gpu, oracle, nrhs):
    import torch
    _, ref, da = root_mesh(gpu, oracle)
    X = np.random.default_rng(8).uniform(-1, 1, (ref.N, nrhs))
    Yr = np.stack([ref.matvec(X[:, j]) for j in range(nrhs)], 1)
    Y = gpu.Jacobian2(da).mult_multi(torch.tensor(X, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    assert (np.linalg.norm(Y - Yr, axis=0) / np.linalg.norm(Yr, axis=0)).max() < 2e-6


def test_boundary_operators_on_one_element(gpu, oracle):
    _, ref, da = root_mesh(gpu, oracle)
    assert ref.node_bdy.all()
    x = I.uniform_rhs(ref.N, 3)
    for A in (gpu.DirichletLaplacian(da), gpu.DirichletJacobian(da)):
        assert np.array_equal(A.mult(x), x)  # every row is a Dirichlet row
        assert np.array_equal(A.getDiagonal().cpu().numpy(), np.ones(ref.N))
    x3 = I.uniform_rhs(3 * ref.N, 4)
    assert np.array_equal(gpu.Elasticity(da, 0.4, 0.6).mult(x3), x3)


def test_mixed_graph_solve_on_one_element(gpu, oracle):
    root, ref, _ = root_mesh(gpu, oracle)
    m = gpu.DAMG(gpu.Octree.from_octants(root, D), inner_prec=1, use_graph=True)
    b = I.uniform_rhs(ref.N, 6)
    for _ in range(2):  # the second solve replays the captured V-cycle
        x, rep = m.solve(b)
        assert rep["converged"]
        assert np.linalg.norm(ref.matvec(x) - b) <= 1.01e-8 * np.linalg.norm(b)
