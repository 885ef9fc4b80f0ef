/* Minimal stand-in for the PETSc declarations the reference's octree / mesh /
 * operator sources use (oracle build only, test infrastructure). */
#ifndef DG_SHIM_PETSCSYS_H
#define DG_SHIM_PETSCSYS_H
#include "petsc.h"
#endif
