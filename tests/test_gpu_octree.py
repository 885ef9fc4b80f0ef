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
