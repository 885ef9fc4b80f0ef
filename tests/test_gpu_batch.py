"""Batched form: independent meshes concatenated into one hierarchy."""
import numpy as np
import pytest

from dendro_b200 import inputs as I

pytestmark = pytest.mark.gpu


def clouds(k, depth=9):
    out = []
    for i in range(k):
        rng = np.random.default_rng(100 + i)
        n = int(np.exp(rng.uniform(np.log(2000), np.log(20000))))
        sigma = rng.uniform(0.05, 0.2)
        c = rng.uniform(0.3, 0.7, 3)
        out.append(I.clamp_unit(rng.normal(c, sigma, (n, 3)), depth))
    return out, depth


def test_batch_matvec_and_solve(gpu, oracle):
    import torch
    pts, d = clouds(5)
    trees = [gpu.balanceOctree(gpu.points2Octree(p, d, 1)) for p in pts]
    m = gpu.DAMG(trees, nlevels=30)
    assert m.count == 5
    eo, no = m.batch_offsets(0)
    meshes = [oracle.Mesh(t.to_numpy(), d) for t in trees]
    assert [mm.N for mm in meshes] == list(np.diff(no))
    da = m.level_da(0)
    ex = da.export()
    for i, mm in enumerate(meshes):  # node map of each mesh, shifted by its node offset
        assert np.array_equal(ex["nlist"][eo[i]:eo[i + 1]] - no[i], mm.nlist)
    coef = np.concatenate([I.sphere_coefficients(gpu.DA(t).elementCenters()) for t in trees])
    x = I.uniform_rhs(int(no[-1]), 4)
    y = gpu.Jacobian2(da, coef).mult(torch.tensor(x, device="cuda")).cpu().numpy()
    for i, mm in enumerate(meshes):
        yi = mm.matvec(x[no[i]:no[i + 1]], coef[2 * eo[i]:2 * eo[i + 1]])
        assert np.linalg.norm(y[no[i]:no[i + 1]] - yi) <= 1e-12 * np.linalg.norm(yi)
    m.setKSP(coef)
    b = I.uniform_rhs(int(no[-1]), 5)
    xs, rep = m.solve(b)
    assert rep["converged"]
    for i, mm in enumerate(meshes):
        bi = b[no[i]:no[i + 1]]
        ri = mm.matvec(xs[no[i]:no[i + 1]], coef[2 * eo[i]:2 * eo[i + 1]]) - bi
        assert np.linalg.norm(ri) <= 1.01e-8 * np.linalg.norm(bi), i


def test_batch_of_uneven_meshes_takes_the_deepest_hierarchy(gpu, oracle):
    """Meshes of very different sizes: the batch has the deepest mesh's level
    count (shallower hierarchies coarsened further) and every mesh converges."""
    from dendro_b200 import inputs as I
    clouds, d = I.batch_clouds(count=4, first_seed=200, depth=10, n_lo=500, n_hi=60000)
    trees = [gpu.balanceOctree(gpu.points2Octree(p, d, 1)) for p in clouds]
    natural = [gpu.DAMG(t).nlevels for t in trees]
    m = gpu.DAMG(trees, inner_prec=1, use_graph=True)
    assert m.nlevels == max(natural)
    _, no = m.batch_offsets(0)
    b = I.uniform_rhs(int(no[-1]), 11)
    x, rep = m.solve(b)
    assert rep["converged"]
    for i, t in enumerate(trees):
        mm = oracle.Mesh(t.to_numpy(), d)
        bi = b[no[i]:no[i + 1]]
        assert np.linalg.norm(mm.matvec(x[no[i]:no[i + 1]]) - bi) <= 1.01e-8 * np.linalg.norm(bi), i
