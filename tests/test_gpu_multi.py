"""Multi-right-hand-side operator (mma.sync on the warp tiles, split 3 / 1;
tcgen05 with tensor-memory accumulators on octet pairs, split 5 / 4; the
octet form on the CUDA cores, split 0) against the oracle's FP64 operator
applied column by column."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu

TOL_SPLIT3 = 2e-6   # three TF32 products: FP32-level, relative 2-norm per column
TOL_SPLIT1 = 2e-3   # one TF32 product (10-bit mantissa inputs)


def setup(gpu, oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    return oracle.Mesh(bal, d), gpu.DA(gpu.Octree.from_octants(bal, d))


# 16 and 48 right-hand sides take the 16-per-pass kernel, multiples of 32 the
# 32-wide block kernel (DG_MRHS_KERNEL=block64: 64-wide where they divide)
@pytest.mark.parametrize("name,nrhs,coef", [("lognormal20k_d12", 32, True), ("gauss20k_d10", 16, False),
                                             ("corner_points_d5", 48, True), ("lognormal20k_d12", 64, True),
                                             ("gauss20k_d10", 96, False), ("uniform8k_d9_m4", 64, False),
                                             ("gauss20k_d10", 128, True), ("single_point", 64, True)])
def test_multi_rhs_matches_oracle(gpu, oracle, name, nrhs, coef):
    import torch
    ref, da = setup(gpu, oracle, name)
    c = I.sphere_coefficients(da.elementCenters()) if coef else None
    A = gpu.Jacobian2(da, c)
    X = np.random.default_rng(6).uniform(-1, 1, (ref.N, nrhs))
    Yr = np.stack([ref.matvec(X[:, j], c) for j in range(nrhs)], 1)
    Xd = torch.tensor(X, dtype=torch.float32, device="cuda")
    forms = ((3, TOL_SPLIT3), (1, TOL_SPLIT1)) + (((0, TOL_SPLIT3),) if nrhs % 32 == 0 else ()) + \
        (((5, TOL_SPLIT3), (4, TOL_SPLIT1)) if nrhs % 64 == 0 else ())
    for split, tol in forms:
        Y = A.mult_multi(Xd, split=split).double().cpu().numpy()
        err = np.linalg.norm(Y - Yr, axis=0) / np.linalg.norm(Yr, axis=0)
        assert err.max() < tol, (split, err.max())


def test_multi_rhs_rejects_bad_shapes(gpu, oracle):
    import torch
    ref, da = setup(gpu, oracle, "corner_points_d5")
    A = gpu.Jacobian2(da)
    with pytest.raises(gpu.DendroError):
        A.mult_multi(torch.zeros((ref.N, 20), dtype=torch.float32, device="cuda"))
    with pytest.raises(gpu.DendroError):  # the tensor-memory form takes multiples of 64
        A.mult_multi(torch.zeros((ref.N, 32), dtype=torch.float32, device="cuda"), split=4)


def test_tensor_memory_form_wait_limit_reports_timeout(gpu, oracle):
    """A one-cycle limit makes every CTA of the tcgen05 form give up on its
    first accumulator wait: it records DG_ETIMEOUT, waits for the MMAs it
    issued, frees its tensor memory and returns; the check reports it once,
    and with the default limit restored the same launch is correct."""
    import torch
    ref, da = setup(gpu, oracle, "lognormal20k_d12")
    A = gpu.Jacobian2(da)
    X = torch.tensor(np.random.default_rng(8).uniform(-1, 1, (ref.N, 64)), dtype=torch.float32, device="cuda")
    Y0 = A.mult_multi(X, split=4).clone()
    gpu.deviceCheck()
    try:
        gpu.setDeviceWaitLimit(1)
        A.mult_multi(X, split=4)
        with pytest.raises(gpu.DendroError) as err:
            gpu.deviceCheck()
        assert err.value.status == 5  # DG_ETIMEOUT
    finally:
        gpu.setDeviceWaitLimit(0)
    gpu.deviceCheck()  # cleared by the check that reported it
    Y = A.mult_multi(X, split=4)
    gpu.deviceCheck()
    assert torch.isfinite(Y).all()
    assert (torch.linalg.norm(Y - Y0) / torch.linalg.norm(Y0)).item() < 1e-6
