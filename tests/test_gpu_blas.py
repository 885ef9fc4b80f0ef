"""GPU FP64 inner product (VecDot stand-in) against numpy."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 255, 4097, 1_000_003])
def test_vec_dot(gpu, n):
    import torch
    rng = np.random.default_rng(n)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    got = gpu.vecDot(torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda"))
    ref = float(np.dot(x, y))
    assert abs(got - ref) <= 1e-12 * max(1.0, np.abs(x) @ np.abs(y))


def test_vec_dot_deterministic(gpu):
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(3_000_000, dtype=torch.float64, device="cuda", generator=g)
    a = [gpu.vecDot(x, x) for _ in range(3)]
    assert a[0] == a[1] == a[2]


@pytest.mark.parametrize("n", [1, 7, 100003])
def test_vec_dot_unaligned_views(gpu, n):
    """Views that start 8 bytes past a 16-byte boundary."""
    import torch
    rng = np.random.default_rng(n + 1)
    a = torch.tensor(rng.standard_normal(n + 1), device="cuda")
    b = torch.tensor(rng.standard_normal(n + 1), device="cuda")
    ref = float(a[1:].cpu().numpy() @ b[1:].cpu().numpy())
    got = gpu.vecDot(a[1:], b[1:])
    assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)) * np.sqrt(n)
