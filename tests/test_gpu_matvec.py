"""GPU elemental operators against the oracle (FP64: 1e-12 relative)."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu

TOL64 = 1e-12   # FP64 matvec vs the reference-form oracle, relative 2-norm
TOL32 = 2e-6    # FP32 matvec vs the FP64 oracle, relative 2-norm


def setup(gpu, oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    ref = oracle.Mesh(bal, d)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    return ref, da


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name", ["gauss2k_d8", "gauss20k_d10", "lognormal20k_d12", "corner_points_d5"])
def test_lapmass_f64(gpu, oracle, name):
    import torch
    ref, da = setup(gpu, oracle, name)
    x = I.uniform_rhs(ref.N, 1)
    y_ref = ref.matvec(x)
    A = gpu.Jacobian2(da)
    y = A.mult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert rel(y, y_ref) < TOL64
    y_host = A.mult(x)
    assert rel(y_host, y_ref) < TOL64


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12"])
def test_lapmass_variable_coef_f64(gpu, oracle, name):
    import torch
    ref, da = setup(gpu, oracle, name)
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 3)
    y_ref = ref.matvec(x, coef)
    y = gpu.Jacobian2(da, coef).mult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert rel(y, y_ref) < TOL64


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12", "corner_points_d5"])
def test_every_launch_shape(gpu, oracle, name):
    """Each operator kernel the autotuner may pick, fixed in turn, FP64 and FP32."""
    import torch
    ref, da = setup(gpu, oracle, name)
    da.compressMaps()  # the compressed-map shape reads its own map, not a fallback
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 5)
    y_ref = ref.matvec(x, coef)
    A = gpu.Jacobian2(da, coef)
    xd = torch.tensor(x, device="cuda")
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        A.set_kernel(v, 1)
        assert rel(A.mult(xd).cpu().numpy(), y_ref) < TOL64, v
        y32 = A.mult(xd.float()).double().cpu().numpy()
        assert rel(y32, y_ref) < TOL32, v


def test_lapmass_f32(gpu, oracle):
    import torch
    ref, da = setup(gpu, oracle, "lognormal20k_d12")
    x = I.uniform_rhs(ref.N, 1)
    y_ref = ref.matvec(x)
    y = gpu.Jacobian2(da).mult(torch.tensor(x, device="cuda", dtype=torch.float32)).double().cpu().numpy()
    assert rel(y, y_ref) < TOL32


def test_diagonal(gpu, oracle):
    ref, da = setup(gpu, oracle, "lognormal20k_d12")
    coef = I.sphere_coefficients(da.elementCenters())
    d = gpu.Jacobian2(da, coef).getDiagonal().cpu().numpy()
    assert rel(d, ref.diagonal(coef)) < TOL64


def test_constant_and_symmetry(gpu, oracle):
    """A 1 integrates to the unit-cube volume; (Ax, y) == (x, Ay)."""
    import torch
    _, da = setup(gpu, oracle, "gauss20k_d10")
    A = gpu.Jacobian2(da)
    one = torch.ones(da.N, dtype=torch.float64, device="cuda")
    assert abs(A.mult(one).sum().item() - 1.0) < 1e-12
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(da.N, dtype=torch.float64, device="cuda", generator=g)
    y = torch.rand(da.N, dtype=torch.float64, device="cuda", generator=g)
    a, b = torch.dot(A.mult(x), y).item(), torch.dot(x, A.mult(y)).item()
    assert abs(a - b) < 1e-12 * abs(a)


@pytest.mark.parametrize("name", ["gauss2k_d8", "lognormal20k_d12"])
def test_elasticity_f64(gpu, oracle, name):
    import torch
    ref, da = setup(gpu, oracle, name)
    mu, lam = 1.0 / (2.0 * 1.3), 0.3 / (1.3 * 0.4)
    x = I.uniform_rhs(3 * ref.N, 5)
    y_ref = ref.elasticity_matvec(x, mu, lam)
    y = gpu.Elasticity(da, mu, lam).mult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert rel(y, y_ref) < TOL64


def test_elasticity_diagonal_matches_unit_vectors(gpu, oracle):
    import torch
    ref, da = setup(gpu, oracle, "corner_points_d5")
    mu, lam = 0.4, 0.6
    A = gpu.Elasticity(da, mu, lam)
    d = A.getDiagonal().cpu().numpy()
    n = 3 * ref.N
    cols = np.array([ref.elasticity_matvec(np.eye(n)[j], mu, lam)[j] for j in range(n)])
    assert rel(d, cols) < TOL64


def test_host_entry_point_pipelined(gpu, oracle):
    """y = A x through the host entry point on a mesh of more than 2^20
    elements (copies pipelined against launches over groups of tiles) against
    the oracle: pageable and page-locked buffers, new buffers and new values
    in the same buffers."""
    import torch
    pts = I.clamp_unit(I.lognormal_cloud(400000, 7), 12)
    bal = gpu.balanceOctree(gpu.points2Octree(pts, 12, 1))
    da = gpu.DA(bal)
    assert da.E >= 1 << 20
    coef = I.sphere_coefficients(da.elementCenters())
    A = gpu.Jacobian2(da, coef)
    ref = oracle.Mesh(bal.to_numpy(), 12)
    for seed in (3, 4):
        x = I.uniform_rhs(da.N, seed)
        y_ref = ref.matvec(x, coef)
        y_page = A.mult(x)                       # first call tunes, later calls pipeline
        xp = torch.tensor(x).pin_memory()
        yp = torch.empty(da.N, dtype=torch.float64).pin_memory()
        A.mult(xp.numpy(), yp.numpy())
        for y in (y_page, yp.numpy(), A.mult(x)):
            assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 1e-12
    x = I.uniform_rhs(da.N, 5)
    xp.copy_(torch.from_numpy(x))
    A.mult(xp.numpy(), yp.numpy())
    y_ref = ref.matvec(x, coef)
    assert np.linalg.norm(yp.numpy() - y_ref) / np.linalg.norm(y_ref) < 1e-12
