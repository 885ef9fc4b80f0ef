"""GPU product at the full size of the small configuration (131,072 Gaussian
points N(0.5, 0.1), seed 0, maxDepth 10, 2:1 balanced: 699,987 elements,
475,159 nodes), as examples/src/drivers/tstMatVec.C:165-275 and the
reference's solve driver run it: the octree bit-exact against the oracle and
the reference's own balance (digest), the DA maps against the reference's
(digest), the FP64 operator within 1e-12 of the oracle and of the reference's
Jacobian2MatMult, and the 4-level V(2,2) PCG to 1e-8 within one iteration of
the oracle's (whose coarsest level, 17,845 nodes, is solved directly on both
sides)."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.golden_data import (CFG1, check_y_digest, digest, load, maps_table, octs_to_u32, reference_matvec,
                               rel)

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def cfg1(gpu, oracle):
    pts, d = I.workload_points(CFG1)
    bal_gpu = gpu.balanceOctree(gpu.points2Octree(pts, d, 1))
    bal_ref = oracle.balance(oracle.points2octree(pts, d, 1), d)
    return d, bal_gpu, bal_ref


def test_cfg1_octree_and_maps(gpu, oracle, cfg1):
    g = load("cfg1_" + CFG1)
    d, bal, bal_ref = cfg1
    octs = bal.to_numpy()
    assert np.array_equal(octs_to_u32(octs), octs_to_u32(bal_ref))
    assert digest(octs_to_u32(octs)) == str(g["bal_sha"])
    da = gpu.DA(bal)
    assert (da.E, da.N) == (int(g["E"]), int(g["N"]))
    ex = da.export()
    assert digest(maps_table(ex["level"], ex["cnum"], ex["hmask"], ex["nlist"])) == str(g["maps_sha"])
    assert digest(ex["node_xyz"]) == str(g["node_sha"])


def test_cfg1_operator(gpu, oracle, cfg1):
    """Every launch shape the autotuner can pick, against the oracle, and the
    tuned one against the reference's own operator on this mesh."""
    import torch
    g = load("cfg1_" + CFG1)
    d, bal, bal_ref = cfg1
    da = gpu.DA(bal)
    x = I.uniform_rhs(da.N, 1)
    y_orc = oracle.Mesh(bal_ref, d).matvec(x)
    A = gpu.Jacobian2(da)
    xd = torch.tensor(x, device="cuda")
    y = A.mult(xd).cpu().numpy()
    assert rel(y, y_orc) < TOL
    check_y_digest(y, g)
    y_ref = reference_matvec(octs_to_u32(bal_ref), d, x)
    if y_ref is not None:
        assert rel(y, y_ref) < TOL
    for v in range(A.kernel_count()):
        A.set_kernel(v, 0)
        assert rel(A.mult(xd).cpu().numpy(), y_orc) < TOL, v


def test_cfg1_pcg_vcycle(gpu, oracle, cfg1):
    """PCG with the 4-level V(2,2) damped-Jacobi cycle (omega 2/3) to relative
    residual 1e-8: converged, the FP64 true residual below the tolerance, the
    iteration count within one of the oracle's, and -- at equal counts -- the
    solution within 1e-6 of the oracle's."""
    d, bal, bal_ref = cfg1
    m = gpu.DAMG(bal, nlevels=4)
    assert m.nlevels == 4
    H = oracle.DAMG(bal_ref, d, 4)
    assert list(H.N) == [int(v) for v in m.N]
    b = I.uniform_rhs(int(m.N[0]), 1)
    x, rep = m.solve(b)
    x_orc, it_orc, _ = H.pcg(b, 1e-8, 100)
    assert it_orc > 0
    res = np.linalg.norm(H.level_mesh(0).matvec(x) - b) / np.linalg.norm(b)
    assert rep["converged"] and res <= 1e-8, (rep, res)
    assert abs(rep["iterations"] - it_orc) <= 1, (rep["iterations"], it_orc)
    if rep["iterations"] == it_orc:  # the same iterates up to rounding
        assert rel(x, x_orc) < 1e-6, rel(x, x_orc)
