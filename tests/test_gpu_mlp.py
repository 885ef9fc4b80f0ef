"""Learned smoother: GPU forward/backward against the FP64 numpy reference,
training with the Adam kernel, and use inside the FP64 flexible PCG."""
import numpy as np
import pytest

from oracle import mlp_ref
from tests.cases import points

pytestmark = pytest.mark.gpu


def rand_features(n, seed):
    rng = np.random.default_rng(seed)
    F = rng.normal(0, 1, (n, 6)).astype(np.float32)
    F[:, 2] = rng.uniform(0, 1, n)
    F[:, 3] = rng.uniform(0, 1, n)
    return F


def test_forward_matches_fp64_reference(gpu):
    import torch
    from dendro_b200.learned import MLP, init_params
    p = init_params(3)
    F = rand_features(5000, 1)
    y_ref, _ = mlp_ref.forward(p.astype(np.float64), F.astype(np.float64))
    net = MLP(p)
    y = net.forward(torch.tensor(F, device="cuda"), exact=True).cpu().numpy()
    assert np.linalg.norm(y - y_ref) <= 1e-5 * np.linalg.norm(y_ref)
    y16 = net.forward(torch.tensor(F, device="cuda"), exact=False).cpu().numpy()  # BF16 weights
    assert np.linalg.norm(y16 - y_ref) <= 2e-2 * np.linalg.norm(y_ref)


def test_gradient_matches_fp64_reference(gpu):
    import torch
    from dendro_b200.learned import MLP, init_params
    p = init_params(5)
    F = rand_features(4096, 2)
    T = np.random.default_rng(3).normal(0, 1, 4096).astype(np.float32)
    loss_ref, g_ref = mlp_ref.loss_and_grad(p.astype(np.float64), F, T)
    net = MLP(p)
    loss, g = net.gradient(torch.tensor(F, device="cuda"), torch.tensor(T, device="cuda"), exact=True)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= 2e-4 * np.linalg.norm(g_ref)
    for name, sl in (("W1", slice(0, 384)), ("W2", slice(448, 4544)), ("w3", slice(4608, 4672))):
        assert np.linalg.norm(g[sl] - g_ref[sl]) <= 5e-4 * np.linalg.norm(g_ref[sl]), name


def test_adam_training_fits_a_teacher(gpu):
    import torch
    from dendro_b200.learned import MLP, init_params
    teacher = init_params(11)
    F = rand_features(32768, 4)
    T, _ = mlp_ref.forward(teacher.astype(np.float64), F.astype(np.float64))
    Fd, Td = torch.tensor(F, device="cuda"), torch.tensor(T.astype(np.float32), device="cuda")
    net = MLP(init_params(12))
    first = net.gradient(Fd, Td)[0]
    for _ in range(300):
        last = net.train_step(Fd, Td, 3e-3)
    assert last < 0.1 * first, (first, last)


def test_learned_smoother_in_flexible_pcg(gpu, oracle):
    """An untrained network as post-smoother: the FP64 residual judges it,
    Jacobi takes over when it stalls, and the solve still reaches 1e-8."""
    from dendro_b200 import inputs as I
    from dendro_b200.learned import MLP, init_params
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    mg = gpu.DAMG(gpu.Octree.from_octants(bal, d), inner_prec=1, use_graph=True)
    mg.setSmoother(MLP(init_params(7)), sweeps=2, fallback_ratio=0.7)
    b = I.uniform_rhs(int(mg.N[0]), 3)
    x, rep = mg.solve(b)
    assert rep["converged"]
    fm = oracle.Mesh(bal, d)
    assert np.linalg.norm(fm.matvec(x) - b) <= 1.01e-8 * np.linalg.norm(b)


def test_trained_smoother_gain_is_measured(gpu, oracle):
    """Train briefly on pairs from the plain solver, then compare iterations
    with and without the learned post-smoother on the same system."""
    from dendro_b200 import inputs as I
    from dendro_b200 import learned as Lrn
    net, hist = Lrn.train(n_pairs=60, steps_per_pair=2, batch=16384, mesh_points=(15000,), log=None)
    assert np.mean(hist[-10:]) < 0.5 * np.mean(hist[:3])
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    b = I.uniform_rhs(len(bal), 9)
    res = {}
    for tag in ("jacobi", "learned"):
        mg = gpu.DAMG(gpu.Octree.from_octants(bal, d), inner_prec=1)
        if tag == "learned":
            mg.setSmoother(net)
        bb = I.uniform_rhs(int(mg.N[0]), 9)
        _, rep = mg.solve(bb)
        assert rep["converged"]
        res[tag] = rep
    print("iterations jacobi", res["jacobi"]["iterations"], "learned", res["learned"]["iterations"],
          "fallbacks", res["learned"]["smoother_fallbacks"])
