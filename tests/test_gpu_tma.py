"""Operator launch shapes whose tile records arrive by bulk copies (TMA):
parity against the oracle on meshes whose element counts put the copy
windows at every 16-byte offset, with and without coefficients, and the
bounded wait for the copies reporting DG_ETIMEOUT without faulting."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.test_gpu_matvec import TOL32, TOL64, rel, setup

pytestmark = pytest.mark.gpu

MESHES = ["gauss2k_d8", "gauss20k_d10", "lognormal20k_d12", "uniform8k_d9_m4", "dup_points_d6",
          "single_point", "corner_points_d5"]


def bulk_copy_shapes(gpu, A):
    out = []
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        if "bulk copy" in A.kernel_name(0):
            out.append(v)
    assert out, "no bulk-copy launch shape registered"
    return out


@pytest.mark.parametrize("coef", [False, True])
def test_bulk_copy_shapes_match_oracle(gpu, oracle, coef):
    import torch
    residues = set()
    for name in MESHES:
        ref, da = setup(gpu, oracle, name)
        residues.add(da.E % 4)
        c = I.sphere_coefficients(da.elementCenters()) if coef else None
        x = I.uniform_rhs(ref.N, 7)
        y_ref = ref.matvec(x, c)
        A = gpu.Jacobian2(da, c)
        xd = torch.tensor(x, device="cuda")
        for v in bulk_copy_shapes(gpu, A):
            A.set_kernel(v, 0)
            A.set_kernel(v, 1)
            assert rel(A.mult(xd).cpu().numpy(), y_ref) < TOL64, (name, v)
            y32 = A.mult(xd.float()).double().cpu().numpy()
            assert rel(y32, y_ref) < TOL32, (name, v)
        gpu.deviceCheck()
    # the second coefficient array starts E elements in: more than one
    # 16-byte offset of its copy window is exercised
    assert len(residues) > 1, residues


def test_wait_limit_reports_timeout(gpu, oracle):
    """A one-cycle limit makes every warp give up on its first stage: the kernel
    records DG_ETIMEOUT, lets its copies land and returns; the check reports it
    once, and with the default limit restored the same launch is correct."""
    import torch
    ref, da = setup(gpu, oracle, "lognormal20k_d12")
    x = I.uniform_rhs(ref.N, 9)
    y_ref = ref.matvec(x)
    A = gpu.Jacobian2(da)
    xd = torch.tensor(x, device="cuda")
    v = bulk_copy_shapes(gpu, A)[0]
    A.set_kernel(v, 0)
    gpu.deviceCheck()
    try:
        gpu.setDeviceWaitLimit(1)
        A.mult(xd)
        with pytest.raises(gpu.DendroError) as err:
            gpu.deviceCheck()
        assert err.value.status == 5  # DG_ETIMEOUT
    finally:
        gpu.setDeviceWaitLimit(0)
    gpu.deviceCheck()  # cleared by the check that reported it
    y = A.mult(xd).cpu().numpy()
    gpu.deviceCheck()
    assert rel(y, y_ref) < TOL64
    assert np.isfinite(y).all()
