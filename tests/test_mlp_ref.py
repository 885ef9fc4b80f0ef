"""CPU: the FP64 numpy MLP reference's gradient against finite differences."""
import numpy as np

from oracle import mlp_ref


def test_reference_gradient_finite_differences():
    rng = np.random.default_rng(0)
    p = mlp_ref.init_params(1)
    F = rng.normal(0, 1, (64, 6))
    T = rng.normal(0, 1, 64)
    loss, g = mlp_ref.loss_and_grad(p, F, T)
    idx = rng.choice(len(p), 40, replace=False)
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (mlp_ref.loss_and_grad(p + e, F, T)[0] - mlp_ref.loss_and_grad(p - e, F, T)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])
    assert mlp_ref.N_PARAMS == 4673
