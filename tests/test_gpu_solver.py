"""GPU multigrid hierarchy, transfer operators and PCG solve against the oracle."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu


def hierarchy(gpu, oracle, name, nlevels):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    ref = oracle.DAMG(bal, d, nlevels)
    got = gpu.DAMG(gpu.Octree.from_octants(bal, d), nlevels=nlevels)
    return ref, got


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12"])
def test_level_sizes_and_transfer(gpu, oracle, name):
    ref, got = hierarchy(gpu, oracle, name, 4)
    assert got.nlevels == ref.nlevels
    assert np.array_equal(got.E, ref.E) and np.array_equal(got.N, ref.N)
    for l in range(ref.nlevels - 1):
        fm, cm = ref.level_mesh(l), ref.level_mesh(l + 1)
        ptr, col, val = oracle.prolongation(fm, cm)
        P = np.zeros((fm.N, cm.N))
        for f in range(fm.N):
            P[f, col[ptr[f]:ptr[f + 1]]] += val[ptr[f]:ptr[f + 1]]
        xc = I.uniform_rhs(cm.N, 10 + l)
        xf0 = I.uniform_rhs(fm.N, 20 + l)
        assert np.linalg.norm(got.prolong(l, xc, xf0) - (xf0 + P @ xc)) < 1e-12 * np.linalg.norm(P @ xc)
        assert np.linalg.norm(got.restrict(l, xf0) - P.T @ xf0) < 1e-12 * np.linalg.norm(P.T @ xf0)


def test_pcg_solution_matches_oracle(gpu, oracle):
    ref, got = hierarchy(gpu, oracle, "gauss20k_d10", 4)
    b = I.uniform_rhs(int(ref.N[0]), 1)
    xr, itr, _ = ref.pcg(b, 1e-10, 100)
    x, rep = got.solve(b)
    assert rep["converged"] and rep["rel_residual"] <= 1e-8
    fm = ref.level_mesh(0)
    assert np.linalg.norm(fm.matvec(x) - b) <= 1.01e-8 * np.linalg.norm(b)
    assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
    assert abs(rep["iterations"] - len(_) + 1) <= 3 or rep["iterations"] <= itr


def test_pcg_variable_coefficients(gpu, oracle):
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    got = gpu.DAMG(gpu.Octree.from_octants(bal, d))
    coef = I.sphere_coefficients(got.level_da(0).elementCenters())
    got.setKSP(coef)
    b = I.uniform_rhs(int(got.N[0]), 3)
    x, rep = got.solve(b)
    assert rep["converged"]
    fm = oracle.Mesh(bal, d)
    assert np.linalg.norm(fm.matvec(x, coef) - b) <= 1.01e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("inner_prec,use_graph", [(0, True), (1, False), (1, True), (2, True)])
def test_pcg_precision_and_graph(gpu, oracle, inner_prec, use_graph):
    """FP32 (or BF16-coefficient) inner V-cycle inside FP64 flexible PCG, with
    and without the CUDA-graph preconditioner: the FP64 true residual reaches 1e-8."""
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    got = gpu.DAMG(gpu.Octree.from_octants(bal, d), inner_prec=inner_prec, use_graph=use_graph)
    coef = I.sphere_coefficients(got.level_da(0).elementCenters())
    got.setKSP(coef)
    b = I.uniform_rhs(int(got.N[0]), 3)
    x, rep = got.solve(b)
    x2, rep2 = got.solve(b)  # second solve replays the captured graph
    assert rep["converged"] and rep2["converged"]
    fm = oracle.Mesh(bal, d)
    for xx in (x, x2):
        assert np.linalg.norm(fm.matvec(xx, coef) - b) <= 1.01e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("inner_prec,tol", [(0, 1e-11), (1, 2e-5)])
def test_vcycle_matches_oracle(gpu, oracle, inner_prec, tol):
    """One V(2,2) application (fused tile-local sweeps and residuals on the
    GPU) against the oracle's V-cycle on the same hierarchy."""
    import torch
    from dendro_b200.learned import vcycle
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    ref = oracle.DAMG(bal, d, 4)
    got = gpu.DAMG(gpu.Octree.from_octants(bal, d), nlevels=4, inner_prec=inner_prec, use_graph=False)
    b = I.uniform_rhs(int(ref.N[0]), 4)
    zr = ref.vcycle(b)
    z = vcycle(got, torch.tensor(b, device="cuda")).cpu().numpy()
    assert np.linalg.norm(z - zr) <= tol * np.linalg.norm(zr)


def test_solve_with_unaligned_device_vectors(gpu, oracle):
    """Device b and x that start 8 bytes past a 16-byte boundary (views into
    larger tensors) take the staged path and give the same solution."""
    import torch
    pts, d, m = points("gauss20k_d10")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    mg = gpu.DAMG(gpu.Octree.from_octants(bal, d), inner_prec=1, use_graph=True)
    n = int(mg.N[0])
    b = I.uniform_rhs(n, 12)
    x0, rep0 = mg.solve(torch.tensor(b, device="cuda"))
    bb = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    bb[1:] = torch.tensor(b, device="cuda")
    xx = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    _, rep1 = mg.solve(bb[1:], xx[1:])
    assert rep0["converged"] and rep1["converged"]
    assert float(torch.linalg.norm(x0 - xx[1:])) <= 1e-12 * float(torch.linalg.norm(x0))


def test_transfer_codes_bit_identical(gpu, oracle, monkeypatch):
    """The 8-bit weight codes of P and R give the FP64 weights' results bit for bit."""
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    coded = gpu.DAMG(gpu.Octree.from_octants(bal, d), nlevels=4)
    monkeypatch.setenv("DG_TRANSFER_CODES", "0")
    plain = gpu.DAMG(gpu.Octree.from_octants(bal, d), nlevels=4)
    for l in range(coded.nlevels - 1):
        xf = I.uniform_rhs(int(coded.N[l]), 30 + l)
        xc = I.uniform_rhs(int(coded.N[l + 1]), 40 + l)
        assert np.array_equal(coded.restrict(l, xf), plain.restrict(l, xf))
        xf0 = I.uniform_rhs(int(coded.N[l]), 50 + l)
        assert np.array_equal(coded.prolong(l, xc, xf0.copy()), plain.prolong(l, xc, xf0.copy()))
