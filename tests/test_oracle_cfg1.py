"""CPU: the oracle restatement at the full size of the small configuration
(131,072 Gaussian points, seed 0, maxDepth 10; 699,987 elements, 475,159
nodes) against the reference itself: its balanced octree, DA maps and
operator output as digests (tests/golden/cfg1_gauss131k_d10.npz), and --
when the compiled reference is present -- its Jacobian2MatMult directly."""
import numpy as np

from dendro_b200 import inputs as I
from tests.golden_data import (CFG1, check_y_digest, digest, load, maps_table, octs_to_u32, reference_matvec,
                               rel)


def test_cfg1_octree_mesh_operator(oracle):
    g = load("cfg1_" + CFG1)
    pts, d = I.workload_points(CFG1)
    assert d == int(g["depth"])
    lin = oracle.points2octree(pts, d, 1)
    assert len(lin) == int(g["n_lin"])
    bal = oracle.balance(lin, d)
    assert digest(octs_to_u32(bal)) == str(g["bal_sha"])
    M = oracle.Mesh(bal, d)
    assert (M.E, M.N) == (int(g["E"]), int(g["N"]))
    assert digest(maps_table(M.elev, M.cnum, M.hmask, M.nlist)) == str(g["maps_sha"])
    assert digest(M.node_xyz) == str(g["node_sha"])
    x = I.uniform_rhs(M.N, 1)
    y = M.matvec(x)
    check_y_digest(y, g)
    y_ref = reference_matvec(octs_to_u32(bal), d, x)
    if y_ref is not None:
        assert rel(y, y_ref) < 1e-12
