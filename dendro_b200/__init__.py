"""dendro_b200: B200-native matrix-free octree finite elements.

Host-side mirror of the reference's interfaces on this path:

* ``points2Octree`` / ``balanceOctree`` / ``coarsenOctree`` (namespace ``ot``,
  src/oct/Construct.C:727, src/oct/Balance.C:31, src/oct/Coarsen.C:53);
* ``DA`` (``ot::DA``, include/oda/oda.h:500);
* ``Jacobian2`` / ``Elasticity`` operators (the MatShell callbacks of
  examples/src/backend/omgNeumann.C:533 and elasticityJac.C:212);
* ``DAMG`` (``ot::DAMG``: DAMGCreateAndSetDA / DAMGSetKSP / DAMGSolve,
  include/omg/omg.h:470-492);
* ``dendro_b200.halo``: one mesh and its hierarchy over several ranks
  (``ot::DA`` / ``ot::DAMG`` with npes > 1).

All work runs in libdendro_b200.so (CUDA, sm_100a); importing this package
does not load it until first use, and every use fails loudly without it.
"""
from .api import (DA, DAMG, DirichletJacobian, DirichletLaplacian, Elasticity, Jacobian2,  # noqa: F401
                  Octree, balanceOctree, coarsenOctree,
                  deviceCheck, points2Octree, readDataPtsFromFile, readNodesFromFile, readPtsFromFile,
                  setDeviceWaitLimit, vecDot, writeDataPtsToFile, writeNodesToFile, writePtsToFile)
from ._lib import DendroError, OCT_DTYPE  # noqa: F401
