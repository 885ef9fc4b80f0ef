"""Coarse operators from the next finer level's coefficients (Jacobian3,
coarse_op = 1) on the GPU: each level's J against the reference's own
Jacobian3MatMult (golden fixture) and against the oracle, one FP64 V-cycle
against the oracle's, and solves that converge in FP64 and mixed precision."""
import os

import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu

TOL = 1e-12      # one operator application, relative 2-norm
# one V-cycle: with the 1e4 coefficient jump the coarsest level's direct
# solve (Gauss-Jordan inverse here, Cholesky in the oracle) amplifies the
# rounding of the assembled matrix by its condition number
TOL_VC = 1e-9


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_level_operator_matches_reference(gpu):
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "jac3_gauss1k_d8.npz"))
    depth, nl = int(g["depth"]), int(g["nlevels"])
    from dendro_b200._lib import OCT_DTYPE
    bal = g["bal"].astype(np.uint32).view(OCT_DTYPE).reshape(-1)
    dm = gpu.DAMG(gpu.Octree.from_octants(bal, depth), nlevels=nl, coarse_op=1)
    assert dm.nlevels == nl
    dm.setKSP(g["coef0"].reshape(-1, 2))
    for l in range(1, nl):
        assert rel(dm.levelApply(l, g[f"jin{l}"]), g[f"jout{l}"]) < TOL, l


def hierarchies(gpu, oracle, name, nlevels, inner_prec=0):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    got = gpu.DAMG(gpu.Octree.from_octants(bal, d), nlevels=nlevels, coarse_op=1, inner_prec=inner_prec)
    coef = I.sphere_coefficients(got.level_da(0).elementCenters())
    got.setKSP(coef)
    ref = oracle.DAMG(bal, d, nlevels, coef)
    ref.set_coarse_op(1)
    assert np.array_equal(got.N, ref.N)
    return ref, got, coef


def level_coef(ref, coef, l, oracle):
    """Averaged coefficients of oracle level l from the finest level's."""
    c = np.ascontiguousarray(coef, np.float64).reshape(-1)
    for k in range(l):
        c = oracle.coarse_coef(ref.level_mesh(k), c, ref.level_mesh(k + 1))
    return c


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12"])
def test_level_operators_and_vcycle_match_oracle(gpu, oracle, name):
    import torch
    from dendro_b200.learned import vcycle
    ref, got, coef = hierarchies(gpu, oracle, name, 4)
    differs = False
    for l in range(got.nlevels):
        x = I.uniform_rhs(int(got.N[l]), 60 + l)
        y = ref.level_apply(l, x)
        assert rel(got.levelApply(l, x), y) < TOL, l
        if l > 0:
            # the type-1 elements make J differ from the averaged-coefficient operator
            ya = ref.level_mesh(l).matvec(x, level_coef(ref, coef, l, oracle))
            differs |= rel(ya, y) > 1e-6
    assert differs
    b = I.uniform_rhs(int(got.N[0]), 7)
    z = vcycle(got, torch.tensor(b, device="cuda")).cpu().numpy()
    assert rel(z, ref.vcycle(b)) < TOL_VC


@pytest.mark.parametrize("inner_prec", [0, 1])
def test_solve_converges(gpu, oracle, inner_prec):
    ref, got, coef = hierarchies(gpu, oracle, "lognormal20k_d12", 30, inner_prec)
    b = I.uniform_rhs(int(got.N[0]), 3)
    x, rep = got.solve(b)
    assert rep["converged"] and rep["rel_residual"] <= 1e-8
    fm = ref.level_mesh(0)
    assert np.linalg.norm(fm.matvec(x, coef) - b) <= 1.01e-8 * np.linalg.norm(b)
    _, it_ref, _ = ref.pcg(b, 1e-8, 200)
    assert abs(rep["iterations"] - it_ref) <= 2
