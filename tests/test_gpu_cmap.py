"""Compressed element map (the DA's compressLut option, include/oda/oda.txx:1125-1300):
the decoded map is bit-exact against the DA's map, and the operator reading it matches
the oracle (FP64 1e-12, FP32 2e-6 relative)."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu


def setup(gpu, oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    return oracle.Mesh(bal, d), gpu.DA(gpu.Octree.from_octants(bal, d))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def cmap_shape(A):
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        if "compressed map" in A.kernel_name(0):
            return v
    raise AssertionError("no compressed-map launch shape")


@pytest.mark.parametrize("name", ["gauss2k_d8", "gauss20k_d10", "lognormal20k_d12", "uniform8k_d9_m4",
                                  "single_point", "corner_points_d5"])
@pytest.mark.parametrize("qbits", [16, 4, 1])
def test_decode_bitexact(gpu, oracle, name, qbits):
    ref, da = setup(gpu, oracle, name)
    nbytes = da.compressMaps(qbits)
    assert np.array_equal(da.decompressMaps(), da.export()["nlist"])
    assert np.array_equal(da.decompressMaps(), ref.nlist)
    wide = da.compressedMapBytes()[1]
    tiles = (da.E + 31) // 32
    assert 0 <= wide <= tiles
    assert nbytes >= 9 * da.E + 8 * tiles
    if qbits == 16 and da.E >= 1000:
        assert wide == 0 and nbytes < 16 * da.E   # against 32 bytes per element raw


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12", "corner_points_d5"])
@pytest.mark.parametrize("qbits", [16, 1])
def test_operator_on_compressed_map(gpu, oracle, name, qbits):
    import torch
    ref, da = setup(gpu, oracle, name)
    da.compressMaps(qbits)
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 7)
    y_ref = ref.matvec(x, coef)
    A = gpu.Jacobian2(da, coef)
    v = cmap_shape(A)
    A.set_kernel(v, 0)
    A.set_kernel(v, 1)
    xd = torch.tensor(x, device="cuda")
    assert rel(A.mult(xd).cpu().numpy(), y_ref) < 1e-12
    assert rel(A.mult(xd.float()).double().cpu().numpy(), y_ref) < 2e-6
    # constant coefficients (no coefficient arrays)
    B = gpu.Jacobian2(da)
    B.set_kernel(v, 0)
    assert rel(B.mult(xd).cpu().numpy(), ref.matvec(x)) < 1e-12


def test_shape_without_map_falls_back(gpu, oracle):
    """The compressed-map shape fixed on a mesh without the map runs the element kernel."""
    import torch
    ref, da = setup(gpu, oracle, "gauss20k_d10")
    other, da2 = setup(gpu, oracle, "gauss20k_d10")
    da2.compressMaps()
    v = cmap_shape(gpu.Jacobian2(da2))
    A = gpu.Jacobian2(da)
    A.set_kernel(v, 0)
    x = I.uniform_rhs(ref.N, 9)
    assert rel(A.mult(torch.tensor(x, device="cuda")).cpu().numpy(), ref.matvec(x)) < 1e-12
