"""The prolongation weights are dyadic: every one is k / 128 with k in 1..128.

The GPU hierarchy stores P's and R's weights as these 8-bit k (checked again
for every level when the hierarchy is built, falling back to the FP64 / FP32
weights when one has no code); this pins the premise on the oracle's
prolongation (Dendro's type-1 transfers, src/omg/ProlongMatVec.C).
"""
import numpy as np
import pytest

from tests.cases import points


@pytest.mark.parametrize("name", ["gauss20k_d10", "lognormal20k_d12"])
def test_transfer_weights_have_exact_codes(oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    ref = oracle.DAMG(bal, d, 4)
    for l in range(ref.nlevels - 1):
        ptr, col, val = oracle.prolongation(ref.level_mesh(l), ref.level_mesh(l + 1))
        k = np.asarray(val) * 128.0
        assert len(k) > 0
        assert np.array_equal(k, np.round(k))
        assert k.min() >= 1 and k.max() <= 128
