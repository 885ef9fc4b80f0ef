// PETSc MatShell binding of the dendro_b200 operators: the code a Dendro
// maintainer adds on the reference side so that a PETSc Mat runs the GPU
// operator.  It replaces CreateJacobian2 / Jacobian2MatMult /
// Jacobian2MatGetDiagonal (examples/src/backend/omgNeumann.C:396-557,
// 643-745) and CreateElasticityMat / ElasticityMatMult /
// ElasticityMatGetDiagonal (examples/src/backend/elasticityJac.C:100-230):
// the callbacks take the MatShell's context, a dg_mat*, and work on host Vec
// arrays (copied to the GPU and back per call).
//
// Include after the PETSc headers (petscmat.h, petscvec.h); link with
// -ldendro_b200 -lcudart.  Errors come back as PETSC_ERR_LIB with the
// library's message on stderr, as the reference's CHKERRQ paths report.
#pragma once

#include <cstdio>

#include <cuda_runtime.h>

#include "dendro_b200.h"

namespace dendro_b200 {

inline PetscErrorCode dg_to_petsc(dg_status st, const char* where) {
  if (st == DG_OK) return 0;
  char msg[512];
  dg_last_error(msg, sizeof msg);
  std::fprintf(stderr, "%s: %s (%s)\n", where, dg_status_string(st), msg);
  return PETSC_ERR_LIB;
}

// MATOP_MULT: out = A in.
inline PetscErrorCode DgMatMult(Mat A, Vec in, Vec out) {
  dg_mat* J = nullptr;
  MatShellGetContext(A, &J);
  PetscScalar *x = nullptr, *y = nullptr;
  VecGetArray(in, &x);
  VecGetArray(out, &y);
  const PetscErrorCode rc = dg_to_petsc(dg_mat_mult_host(J, x, y), "DgMatMult");
  VecRestoreArray(in, &x);
  VecRestoreArray(out, &y);
  return rc;
}

// MATOP_GET_DIAGONAL: d = diag(A) (the Jacobi smoother's diagonal).
inline PetscErrorCode DgMatGetDiagonal(Mat A, Vec d) {
  dg_mat* J = nullptr;
  MatShellGetContext(A, &J);
  const int64_t n = dg_mat_size(J);
  double* dd = nullptr;
  if (cudaMalloc(&dd, sizeof(double) * size_t(n)) != cudaSuccess) return PETSC_ERR_MEM;
  PetscErrorCode rc = dg_to_petsc(dg_mat_get_diagonal(J, dd, nullptr), "DgMatGetDiagonal");
  PetscScalar* h = nullptr;
  VecGetArray(d, &h);
  if (!rc && cudaMemcpy(h, dd, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = PETSC_ERR_LIB;
  VecRestoreArray(d, &h);
  cudaFree(dd);
  return rc;
}

// MATOP_DESTROY: the operator goes with the Mat (as DestroyUserContexts,
// omgNeumann.C:300-322, frees the Jacobian's context).
inline PetscErrorCode DgMatDestroy(Mat A) {
  dg_mat* J = nullptr;
  MatShellGetContext(A, &J);
  dg_mat_destroy(J);
  return 0;
}

// MatCreateShell over an operator, with the three callbacks set; the Mat
// takes ownership of J.
inline PetscErrorCode DgCreateMatShell(MPI_Comm comm, dg_mat* J, Mat* A) {
  const PetscInt n = PetscInt(dg_mat_size(J));
  PetscErrorCode rc = MatCreateShell(comm, n, n, PETSC_DETERMINE, PETSC_DETERMINE, J, A);
  if (rc) return rc;
  MatShellSetOperation(*A, MATOP_MULT, (void (*)(void))DgMatMult);
  MatShellSetOperation(*A, MATOP_GET_DIAGONAL, (void (*)(void))DgMatGetDiagonal);
  MatShellSetOperation(*A, MATOP_DESTROY, (void (*)(void))DgMatDestroy);
  return 0;
}

}  // namespace dendro_b200
