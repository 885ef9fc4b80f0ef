"""Octree invariants as CPU validators of GPU outputs (test infrastructure).

The reference checks its octrees with the predicates of include/test/testUtils.h:29-100
(isSorted, isLinear, isComplete, isBalanced; src/test/testUtils.C).  These are numpy
restatements over octant arrays with fields x, y, z (anchor at maxDepth resolution) and
lf (level in the low 5 bits): Morton order with coarser first for equal anchors
(TreeNode.txx:160-188), no octant overlapping the next, volumes adding up to the
domain, and 2:1 balance across faces, edges and corners (incCorner).
"""
import numpy as np


def _spread(v):
    """Bits of v (< 2^21) moved to every third position."""
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton(x, y, z):
    """Morton key with z the most significant bit of each triple."""
    return _spread(x) | (_spread(y) << np.uint64(1)) | (_spread(z) << np.uint64(2))


def _fields(octs):
    x = octs["x"].astype(np.int64)
    y = octs["y"].astype(np.int64)
    z = octs["z"].astype(np.int64)
    lev = (octs["lf"] & 31).astype(np.int64)
    return x, y, z, lev


def is_sorted_linear(octs, max_depth):
    """Sorted (Morton, coarser first) and linear (no octant contains the next)."""
    if len(octs) < 2:
        return True
    x, y, z, lev = _fields(octs)
    m = morton(x, y, z)
    vol = np.uint64(1) << (np.uint64(3) * (max_depth - lev).astype(np.uint64))
    return bool(np.all(m[1:] >= m[:-1] + vol[:-1]))


def is_complete(octs, max_depth):
    """Linear and covering the domain: the volumes add up to 8^maxDepth."""
    _, _, _, lev = _fields(octs)
    total = sum(int(v) for v in (np.uint64(1) << (np.uint64(3) * (max_depth - lev).astype(np.uint64))))
    return is_sorted_linear(octs, max_depth) and total == 8 ** max_depth


def is_balanced(octs, max_depth):
    """2:1 across faces, edges and corners, for a complete linear octree: from every
    octant, the leaf just outside it in each of the 26 directions is at most one
    level coarser (a finer neighbour sees this octant from its own side)."""
    x, y, z, lev = _fields(octs)
    size = np.int64(1) << (max_depth - lev)
    keys = morton(x, y, z)
    top = np.int64(1) << max_depth
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                if dx == dy == dz == 0:
                    continue
                q = [np.where(d < 0, a - 1, np.where(d > 0, a + size, a)) for d, a in ((dx, x), (dy, y), (dz, z))]
                inside = np.ones(len(x), bool)
                for c in q:
                    inside &= (c >= 0) & (c < top)
                if not inside.any():
                    continue
                qm = morton(q[0][inside], q[1][inside], q[2][inside])
                j = np.searchsorted(keys, qm, side="right") - 1
                if np.any(lev[j] < lev[inside] - 1):
                    return False
    return True
