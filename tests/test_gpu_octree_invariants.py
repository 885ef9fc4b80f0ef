"""The GPU's octrees checked with the reference's invariant predicates (isSorted, isLinear,
isComplete, isBalanced; include/test/testUtils.h:29-100) on the CPU, also at the
benchmark's size (1M points, maxDepth 14), where no oracle octree is built in the tests."""
import pytest

from dendro_b200 import inputs as I
from tests import octree_checks as V
from tests.cases import points

pytestmark = pytest.mark.gpu


def check_chain(gpu, pts, d, m=1):
    lin = gpu.points2Octree(pts, d, m)
    a = lin.to_numpy()
    assert V.is_sorted_linear(a, d) and V.is_complete(a, d)
    bal = gpu.balanceOctree(lin)
    b = bal.to_numpy()
    assert V.is_complete(b, d) and V.is_balanced(b, d)
    c = gpu.coarsenOctree(bal).to_numpy()
    assert V.is_complete(c, d)
    return len(a), len(b), len(c)


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12", "uniform8k_d9_m4", "dup_points_d6",
                                  "single_point", "corner_points_d5"])
def test_case_octrees(gpu, name):
    pts, d, m = points(name)
    check_chain(gpu, pts, d, m)


@pytest.mark.parametrize("name", ["gauss131k_d10", "lognormal1m_d14"])
def test_benchmark_octrees(gpu, name):
    pts, d = I.workload_points(name)
    n_lin, n_bal, n_coarse = check_chain(gpu, pts, d)
    assert n_bal >= n_lin > n_coarse
