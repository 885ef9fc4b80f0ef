"""GPU octree construction, balance and coarsening: bit-exact against the oracle."""
import numpy as np
import pytest

from tests.cases import CASES, points

pytestmark = pytest.mark.gpu


def same(a, b):
    return len(a) == len(b) and np.array_equal(a.view(np.uint32).reshape(-1, 4), b.view(np.uint32).reshape(-1, 4))


@pytest.mark.parametrize("name", sorted(CASES))
def test_points2octree_bitexact(gpu, oracle, name):
    pts, d, m = points(name)
    ref = oracle.points2octree(pts, d, m)
    got = gpu.points2Octree(pts, d, m).to_numpy()
    assert same(got, ref), (len(got), len(ref))


@pytest.mark.parametrize("name", sorted(CASES))
def test_balance_bitexact(gpu, oracle, name):
    pts, d, m = points(name)
    lin = oracle.points2octree(pts, d, m)
    ref = oracle.balance(lin, d)
    got = gpu.balanceOctree(gpu.Octree.from_octants(lin, d)).to_numpy()
    assert same(got, ref), (len(got), len(ref))
    assert oracle.is_sorted_linear(got)


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12", "uniform8k_d9_m4"])
def test_coarsen_bitexact(gpu, oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    ref = oracle.coarsen(bal, d)
    got = gpu.coarsenOctree(gpu.Octree.from_octants(bal, d)).to_numpy()
    assert same(got, ref)


def test_device_points_input(gpu, oracle):
    import torch
    pts, d, m = points("gauss20k_d10")
    ref = oracle.points2octree(pts, d, m)
    got = gpu.points2Octree(torch.tensor(pts, device="cuda"), d, m).to_numpy()
    assert same(got, ref)


def test_points_outside_unit_cube_rejected(gpu):
    with pytest.raises(gpu.DendroError):
        gpu.points2Octree(np.array([[0.5, 1.5, 0.2], [0.1, 0.1, 0.1]]), 8, 1)


def test_unsorted_octants_rejected(gpu, oracle):
    pts, d, m = points("gauss2k_d8")
    lin = oracle.points2octree(pts, d, m)
    with pytest.raises(gpu.DendroError):
        gpu.Octree.from_octants(lin[::-1].copy(), d)


def test_empty_point_set(gpu, oracle):
    """No points: the complete octree is the root octant alone, as the oracle's."""
    ref = oracle.points2octree(np.zeros((0, 3)), 6, 1)
    t = gpu.points2Octree(np.zeros((0, 3)), 6, 1)
    assert same(t.to_numpy(), ref)
    assert same(gpu.balanceOctree(t).to_numpy(), oracle.balance(ref, 6))


def deep_points(d):
    from dendro_b200 import inputs as I
    # two points one finest cell apart force leaves at level d
    return np.concatenate([np.array([[0.5, 0.5, 0.5], [0.5 + 2.0 ** -d, 0.5, 0.5]]),
                           I.clamp_unit(np.random.default_rng(3).uniform(0, 1, (200, 3)), d)])


def test_deepest_supported_octree(gpu, oracle):
    """Octrees go to maxDepth 19 (bit-exact); maxDepth 20 is refused with
    DG_EDEPTH, and so is a mesh of a depth-19 octree (its embedded keys would
    need 65 bits)."""
    d = 19
    pts = deep_points(d)
    lin = oracle.points2octree(pts, d, 1)
    assert (lin["lf"] & 31).max() == d
    got = gpu.points2Octree(pts, d, 1)
    assert same(got.to_numpy(), lin)
    gb = gpu.balanceOctree(got)
    assert same(gb.to_numpy(), oracle.balance(lin, d))
    for call in (lambda: gpu.points2Octree(pts, 20, 1), lambda: gpu.DA(gb)):
        with pytest.raises(gpu.DendroError) as err:
            call()
        assert err.value.status == 7  # DG_EDEPTH


def test_deepest_supported_mesh(gpu, oracle):
    """Meshes go to maxDepth 18 (embedded depth 19): octree, balance, mesh and
    operator match the oracle with leaves at the deepest level."""
    from dendro_b200 import inputs as I
    d = 18
    pts = deep_points(d)
    lin = oracle.points2octree(pts, d, 1)
    assert (lin["lf"] & 31).max() == d
    bal = oracle.balance(lin, d)
    gb = gpu.balanceOctree(gpu.points2Octree(pts, d, 1))
    assert same(gb.to_numpy(), bal)
    ref = oracle.Mesh(bal, d)
    da = gpu.DA(gb)
    assert (da.E, da.N) == (ref.E, ref.N)
    x = I.uniform_rhs(ref.N, 4)
    y, yr = gpu.Jacobian2(da).mult(x), ref.matvec(x)
    assert np.linalg.norm(y - yr) <= 1e-12 * np.linalg.norm(yr)
