// Companion of the reference's examples/src/drivers/dumpMesh.C in the
// single-rank oracle build (test infrastructure only):
//  * ot::RegisterEvents (src/sys/sys.C:19) registers the reference's
//    block-diagonal PETSc preconditioner and its logging events; the mesh
//    dump uses neither, so it is a no-op here;
//  * every TreeNode constructor reads the Hilbert rotation tables, which
//    dumpMesh.C's main does not set up; they are set up before main, as the
//    reference's own drivers do first thing (examples/src/drivers/testPartition.C:35).
#include "petsc.h"

void initializeHilbetTable(int dim);

namespace ot {
PetscErrorCode RegisterEvents() { return 0; }
}  // namespace ot

namespace {
struct HilbertTables {
  HilbertTables() {
    initializeHilbetTable(2);
    initializeHilbetTable(3);
  }
} hilbert_tables;
}  // namespace
