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

// ---- the intergrid transfer as a MatShell ----
// DAMGSetUp wraps R between level l and the next coarser one in a MatShell
// (src/omg/omg.C:2278-2283, context TransferOpData, include/omg/omg.h:
// 386-412): MATOP_MULT restricts (coarse = R fine), MATOP_MULT_TRANSPOSE
// prolongs (fine = P coarse, P = R^T), the ADD forms add the product to
// another Vec, MATOP_DESTROY frees the context.  PCMG calls them through
// MatRestrict / MatInterpolate(Add).  Vec arrays are host arrays, copied to
// the GPU and back per call; the hierarchy stays owned by the caller.
struct DgTransferCtx {
  dg_damg* m;
  int level;
  int64_t nf, nc;  // fine and coarse Vec lengths (dof x nodes)
};

// c = R f
inline PetscErrorCode DgRestrictMult(Mat R, Vec f, Vec c) {
  DgTransferCtx* t = nullptr;
  MatShellGetContext(R, &t);
  PetscScalar *pf = nullptr, *pc = nullptr;
  VecGetArray(f, &pf);
  VecGetArray(c, &pc);
  const PetscErrorCode rc = dg_to_petsc(dg_damg_restrict(t->m, t->level, pf, pc, 0), "DgRestrictMult");
  VecRestoreArray(f, &pf);
  VecRestoreArray(c, &pc);
  return rc;
}

// f = P c (R^T c): the library adds P c into f, so f is zeroed first
inline PetscErrorCode DgProlongMult(Mat R, Vec c, Vec f) {
  DgTransferCtx* t = nullptr;
  MatShellGetContext(R, &t);
  PetscScalar *pc = nullptr, *pf = nullptr;
  VecGetArray(c, &pc);
  VecGetArray(f, &pf);
  for (int64_t i = 0; i < t->nf; ++i) pf[i] = 0.0;
  const PetscErrorCode rc = dg_to_petsc(dg_damg_prolong(t->m, t->level, pc, pf, 0), "DgProlongMult");
  VecRestoreArray(c, &pc);
  VecRestoreArray(f, &pf);
  return rc;
}

// out = add + R f (MatMultAdd)
inline PetscErrorCode DgRestrictMultAdd(Mat R, Vec f, Vec add, Vec out) {
  DgTransferCtx* t = nullptr;
  MatShellGetContext(R, &t);
  double* tmp = new double[size_t(t->nc)];
  PetscScalar *pf = nullptr, *pa = nullptr, *po = nullptr;
  VecGetArray(f, &pf);
  PetscErrorCode rc = dg_to_petsc(dg_damg_restrict(t->m, t->level, pf, tmp, 0), "DgRestrictMultAdd");
  VecRestoreArray(f, &pf);
  if (!rc) {
    VecGetArray(add, &pa);
    VecGetArray(out, &po);
    for (int64_t i = 0; i < t->nc; ++i) po[i] = pa[i] + tmp[i];
    VecRestoreArray(add, &pa);
    VecRestoreArray(out, &po);
  }
  delete[] tmp;
  return rc;
}

// out = add + P c (MatMultTransposeAdd, PCMG's MatInterpolateAdd)
inline PetscErrorCode DgProlongMultAdd(Mat R, Vec c, Vec add, Vec out) {
  DgTransferCtx* t = nullptr;
  MatShellGetContext(R, &t);
  PetscScalar *pc = nullptr, *pa = nullptr, *po = nullptr;
  VecGetArray(add, &pa);
  VecGetArray(out, &po);
  if (po != pa)
    for (int64_t i = 0; i < t->nf; ++i) po[i] = pa[i];
  VecGetArray(c, &pc);
  const PetscErrorCode rc = dg_to_petsc(dg_damg_prolong(t->m, t->level, pc, po, 0), "DgProlongMultAdd");
  VecRestoreArray(c, &pc);
  VecRestoreArray(add, &pa);
  VecRestoreArray(out, &po);
  return rc;
}

inline PetscErrorCode DgTransferDestroy(Mat R) {
  DgTransferCtx* t = nullptr;
  MatShellGetContext(R, &t);
  delete t;
  return 0;
}

// MatCreateShell over R from `level` (0 = finest) to level + 1 of m, with
// the five callbacks set; rows are the coarse Vec's entries, columns the
// fine one's.  dof is the hierarchy's (1, or 3 for elasticity).
inline PetscErrorCode DgCreateRestrictionShell(MPI_Comm comm, dg_damg* m, int level, int dof, Mat* R) {
  const int L = dg_damg_levels(m);
  if (level < 0 || level + 1 >= L) return PETSC_ERR_ARG_OUTOFRANGE;
  int64_t* E = new int64_t[size_t(L)];
  int64_t* N = new int64_t[size_t(L)];
  PetscErrorCode rc = dg_to_petsc(dg_damg_level_sizes(m, E, N), "DgCreateRestrictionShell");
  DgTransferCtx* t = rc ? nullptr : new DgTransferCtx{m, level, int64_t(dof) * N[level], int64_t(dof) * N[level + 1]};
  delete[] E;
  delete[] N;
  if (rc) return rc;
  rc = MatCreateShell(comm, PetscInt(t->nc), PetscInt(t->nf), PETSC_DETERMINE, PETSC_DETERMINE, t, R);
  if (rc) {
    delete t;
    return rc;
  }
  MatShellSetOperation(*R, MATOP_MULT, (void (*)(void))DgRestrictMult);
  MatShellSetOperation(*R, MATOP_MULT_TRANSPOSE, (void (*)(void))DgProlongMult);
  MatShellSetOperation(*R, MATOP_MULT_ADD, (void (*)(void))DgRestrictMultAdd);
  MatShellSetOperation(*R, MATOP_MULT_TRANSPOSE_ADD, (void (*)(void))DgProlongMultAdd);
  MatShellSetOperation(*R, MATOP_DESTROY, (void (*)(void))DgTransferDestroy);
  return 0;
}

}  // namespace dendro_b200
