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


def test_trained_smoother_gain_is_measured(gpu):
    """The committed trained network (the benchmark's) as the finest-level
    post-smoother of the FP32 V-cycle in flexible PCG, against the same cycle
    with damped Jacobi post-smoothing (2 sweeps) and with none, on a 262,144-
    point log-normal octree (maxDepth 14, the training distribution):
      * the network has learned something: it needs fewer iterations to 1e-8
        than the cycle without post-smoothing;
      * its solve time against Jacobi's is the product of the measured
        iteration ratio and per-cycle cost ratio (within 25 %), so the
        measured gain (or loss) is explained by those two numbers, which the
        test reports: the network costs more per application than the two
        Jacobi sweeps it replaces and does not cut the iteration count below
        theirs, so it does not pay on this hardware."""
    import torch

    from dendro_b200 import inputs as I
    from dendro_b200.learned import MLP, WEIGHTS, vcycle
    pts = I.clamp_unit(I.lognormal_cloud(262144, 11), 14)
    bal = gpu.balanceOctree(gpu.points2Octree(pts, 14, 1))
    net = MLP(np.load(WEIGHTS))
    out = {}
    for tag, kw in (("jacobi", {}), ("none", {"nu_post": 0}), ("learned", {})):
        mg = gpu.DAMG(bal, inner_prec=1, use_graph=True, **kw)
        if tag == "learned":
            mg.setSmoother(net)
        b = torch.tensor(I.uniform_rhs(int(mg.N[0]), 9), device="cuda")
        mg.solve(b)
        reps = [mg.solve(b)[1] for _ in range(3)]
        rep = min(reps, key=lambda r: r["solve_ms"])
        assert rep["converged"], (tag, rep)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            vcycle(mg, b)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(10):
            vcycle(mg, b)
        e1.record()
        torch.cuda.synchronize()
        out[tag] = dict(iterations=rep["iterations"], solve_ms=rep["solve_ms"], cycle_ms=e0.elapsed_time(e1) / 10,
                        fallbacks=rep["smoother_fallbacks"])
        del mg
    print("learned smoother:", out)
    assert out["learned"]["iterations"] < out["none"]["iterations"]
    model = (out["learned"]["iterations"] * out["learned"]["cycle_ms"]) / (
        out["jacobi"]["iterations"] * out["jacobi"]["cycle_ms"])
    measured = out["learned"]["solve_ms"] / out["jacobi"]["solve_ms"]
    assert abs(measured / model - 1) < 0.25, (measured, model)
