"""The octree validators (tests/octree_checks.py) against the oracle's octrees, and with
mistakes planted in those octrees (an octant removed, two swapped, a 2:1 violation)."""
import numpy as np
import pytest

from tests import octree_checks as V
from tests.cases import points


@pytest.mark.parametrize("name", ["gauss2k_d8", "lognormal20k_d12", "uniform8k_d9_m4", "corner_points_d5"])
def test_validators_accept_oracle_octrees(oracle, name):
    pts, d, m = points(name)
    lin = oracle.points2octree(pts, d, m)
    bal = oracle.balance(lin, d)
    assert V.is_sorted_linear(lin, d) and V.is_complete(lin, d)
    assert V.is_complete(bal, d) and V.is_balanced(bal, d)
    coarse = oracle.coarsen(bal, d)
    assert V.is_complete(coarse, d)


def test_validators_reject_planted_mistakes(oracle):
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    lin = oracle.points2octree(pts, d, m)
    k = len(bal) // 2
    assert not V.is_complete(np.delete(bal, k), d)               # a hole
    swapped = bal.copy()
    swapped[[k, k + 1]] = swapped[[k + 1, k]]
    assert not V.is_sorted_linear(swapped, d)                     # out of order
    assert not V.is_sorted_linear(np.concatenate([bal[:k + 1], bal[k:]]), d)   # an overlap
    # the unbalanced linear octree fails 2:1 where balancing added octants
    if len(lin) != len(bal):
        assert V.is_complete(lin, d) and not V.is_balanced(lin, d)
