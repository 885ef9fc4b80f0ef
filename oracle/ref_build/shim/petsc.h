/* Minimal single-process stand-in for the parts of PETSc that the reference's
 * octree / mesh / operator / transfer sources touch, so that they compile
 * and run unmodified as one rank.  Vec is a host array, Mat a shell with a
 * function table, KSP / PC / logging / viewers are inert.  Written for the
 * oracle build only (test infrastructure, never part of the product). */
#ifndef DG_SHIM_PETSC_H
#define DG_SHIM_PETSC_H

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

#include "mpi.h"

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef double PetscLogDouble;
typedef int PetscLogEvent;
typedef int PetscClassId;
typedef int PetscCookie;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef PetscBool PetscTruth;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2, MAX_VALUES = 3, NOT_SET_VALUES = 0 } InsertMode;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3, NORM_1_AND_2 = 4 } NormType;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { SAME_NONZERO_PATTERN = 0, DIFFERENT_NONZERO_PATTERN, SAME_PRECONDITIONER, SUBSET_NONZERO_PATTERN } MatStructure;
typedef enum { MAT_INITIAL_MATRIX, MAT_REUSE_MATRIX } MatReuse;
typedef enum { SCATTER_FORWARD = 0, SCATTER_REVERSE = 1 } ScatterMode;
typedef enum {
  MATOP_MULT = 1, MATOP_MULT_ADD, MATOP_MULT_TRANSPOSE, MATOP_MULT_TRANSPOSE_ADD, MATOP_GET_DIAGONAL,
  MATOP_DESTROY, MATOP_GET_ROW, MATOP_VIEW, MATOP_ZERO_ENTRIES, MATOP_LAST
} MatOperation;
typedef enum { PC_LEFT, PC_RIGHT, PC_SYMMETRIC } PCSide;
typedef enum { KSP_NORM_DEFAULT = -1, KSP_NORM_NONE = 0, KSP_NORM_PRECONDITIONED = 1, KSP_NORM_UNPRECONDITIONED = 2,
               KSP_NORM_NATURAL = 3 } KSPNormType;
typedef enum { PC_MG_MULTIPLICATIVE, PC_MG_ADDITIVE, PC_MG_FULL, PC_MG_KASKADE } PCMGType;
typedef enum { PC_MG_CYCLE_V = 1, PC_MG_CYCLE_W = 2 } PCMGCycleType;
typedef enum { KSP_CONVERGED_ITERATING = 0 } KSPConvergedReason;
typedef enum { MAT_SHIFT_NONE, MAT_SHIFT_NONZERO, MAT_SHIFT_POSITIVE_DEFINITE, MAT_SHIFT_INBLOCKS } MatFactorShiftType;
typedef const char* MatType;
typedef const char* VecType;
typedef const char* KSPType;
typedef const char* PCType;
typedef const char* PetscRandomType;

#define PETSC_NULL 0
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_COMM_SELF MPI_COMM_SELF
#define PETSC_ERR_ARG_WRONG 62
#define PETSC_ERR_SUP 56
#define PETSC_ERR_MEM 55
#define PETSC_ERR_LIB 76
#define PETSC_ERR_USER 83
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_VIEWER_STDOUT_WORLD ((PetscViewer)0)
#define PETSC_VIEWER_STDOUT_SELF ((PetscViewer)0)
#define PETSC_VIEWER_DRAW_(c) ((PetscViewer)0)
#define PETSC_ERR_ARG_NULL 85
#define PETSC_ERR_ORDER 73
#define PETSC_ERR_ARG_INCOMP 75
#define MATDAAD "daad"
#define MATMFFD "mffd"

#define VECMPI "mpi"
#define VECSEQ "seq"
#define VECSTANDARD "standard"
#define MATMPIAIJ "mpiaij"
#define MATSEQAIJ "seqaij"
#define MATAIJ "aij"
#define MATMPIBAIJ "mpibaij"
#define MATSEQBAIJ "seqbaij"
#define MATBAIJ "baij"
#define MATSHELL "shell"
#define KSPCG "cg"
#define KSPFGMRES "fgmres"
#define KSPGMRES "gmres"
#define KSPRICHARDSON "richardson"
#define KSPPREONLY "preonly"
#define PCMG "mg"
#define PCNONE "none"
#define PCLU "lu"
#define PCJACOBI "jacobi"
#define PCSHELL "shell"
#define PCREDUNDANT "redundant"
#define PCCHOLESKY "cholesky"
#define PETSCRAND48 "rand48"

#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)
#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define CHKERRABORT(c, e) do { if (e) MPI_Abort(c, e); } while (0)
#define CHKMEMQ
#define SETERRQ(c, n, s) do { fprintf(stderr, "%s\n", s); return (n); } while (0)
#define SETERRQ1(c, n, s, a) do { fprintf(stderr, s, a); return (n); } while (0)
#define PetscLogEventBegin(...) 0
#define PetscLogEventEnd(...) 0
#define PetscLogFlops(x) 0
#define PetscLogEventRegister(...) 0
#define PetscMax(a, b) ((a) > (b) ? (a) : (b))
#define PetscMin(a, b) ((a) < (b) ? (a) : (b))
#define PetscAbsScalar(a) fabs(a)
#define PetscAbsReal(a) fabs(a)
#define PetscSqrtScalar(a) sqrt(a)
#define PetscRealPart(a) (a)
#define PetscMalloc(n, p) ((*(void**)(p) = malloc(n)) ? 0 : 55)
#define PetscFree(p) (free(p), (p) = 0, 0)
#define PetscNew(T, p) ((*(p) = (T*)calloc(1, sizeof(T))) ? 0 : 55)
#define PetscMemzero(p, n) (memset((p), 0, (n)), 0)
#define PetscMemcpy(d, s, n) (memcpy((d), (s), (n)), 0)

struct _p_PetscObject { int dummy; };
typedef _p_PetscObject* PetscObject;
struct _p_PetscViewer { int dummy; };
typedef _p_PetscViewer* PetscViewer;
struct _p_PetscRandom { unsigned long seed; };
typedef _p_PetscRandom* PetscRandom;
struct _p_MatNullSpace { int dummy; };
typedef _p_MatNullSpace* MatNullSpace;
struct _p_IS { int dummy; };
typedef _p_IS* IS;
struct _p_VecScatter { int dummy; };
typedef _p_VecScatter* VecScatter;

struct _p_Vec {
  std::vector<double> a;
  double* placed = 0;
  double* data() { return placed ? placed : a.data(); }
};
typedef _p_Vec* Vec;

typedef PetscErrorCode (*DgShimMatFn)(void);
struct _p_Mat {
  void* ctx = 0;
  int m = 0, n = 0;
  DgShimMatFn op[MATOP_LAST] = {0};
  std::vector<double>* dense = 0;
};
typedef _p_Mat* Mat;
struct _p_PC { void* ctx = 0; int setupcalled = 0; };
typedef _p_PC* PC;
struct _p_KSP { _p_PC pc; };
typedef _p_KSP* KSP;

/* ---- options database (string map) ---- */
static inline std::map<std::string, std::string>& dg_shim_opts() {
  static std::map<std::string, std::string> m;
  return m;
}
static inline PetscErrorCode PetscInitialize(int*, char***, const char*, const char*) { return 0; }
static inline PetscErrorCode PetscFinalize() { return 0; }
static inline PetscErrorCode PetscOptionsSetValue(const char* k, const char* v) { dg_shim_opts()[k] = v ? v : ""; return 0; }
static inline PetscErrorCode PetscOptionsClearValue(const char* k) { dg_shim_opts().erase(k); return 0; }
static inline PetscErrorCode PetscOptionsHasName(const char*, const char* k, PetscBool* f) {
  *f = dg_shim_opts().count(k) ? PETSC_TRUE : PETSC_FALSE; return 0; }
static inline PetscErrorCode PetscOptionsGetInt(const char*, const char* k, PetscInt* v, PetscBool* f) {
  auto it = dg_shim_opts().find(k); if (f) *f = PETSC_FALSE;
  if (it != dg_shim_opts().end()) { *v = atoi(it->second.c_str()); if (f) *f = PETSC_TRUE; } return 0; }
static inline PetscErrorCode PetscOptionsGetReal(const char*, const char* k, PetscReal* v, PetscBool* f) {
  auto it = dg_shim_opts().find(k); if (f) *f = PETSC_FALSE;
  if (it != dg_shim_opts().end()) { *v = atof(it->second.c_str()); if (f) *f = PETSC_TRUE; } return 0; }
static inline PetscErrorCode PetscOptionsGetString(const char*, const char* k, char* v, size_t n, PetscBool* f) {
  auto it = dg_shim_opts().find(k); if (f) *f = PETSC_FALSE;
  if (it != dg_shim_opts().end()) { strncpy(v, it->second.c_str(), n); if (f) *f = PETSC_TRUE; } return 0; }
static inline PetscErrorCode PetscOptionsGetTruth(const char* p, const char* k, PetscBool* v, PetscBool* f) {
  PetscInt i = *v; PetscErrorCode e = PetscOptionsGetInt(p, k, &i, f); *v = i ? PETSC_TRUE : PETSC_FALSE; return e; }
#define PetscOptionsGetBool PetscOptionsGetTruth
static inline PetscErrorCode PetscStrcmp(const char* a, const char* b, PetscBool* f) {
  *f = (a && b && !strcmp(a, b)) ? PETSC_TRUE : PETSC_FALSE; return 0; }
static inline PetscErrorCode PetscPrintf(MPI_Comm, const char* fmt, ...) {
  va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap); return 0; }
static inline PetscErrorCode PetscSynchronizedPrintf(MPI_Comm, const char* fmt, ...) {
  va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap); return 0; }
static inline PetscErrorCode PetscSynchronizedFlush(MPI_Comm) { return 0; }
static inline PetscErrorCode PetscGetTime(PetscLogDouble* t) { *t = MPI_Wtime(); return 0; }
static inline PetscErrorCode PetscTime(PetscLogDouble* t) { *t = MPI_Wtime(); return 0; }
static inline PetscErrorCode PetscObjectGetComm(PetscObject, MPI_Comm* c) { *c = MPI_COMM_WORLD; return 0; }
template <class T> static inline PetscErrorCode PetscObjectTypeCompare(T, const char*, PetscBool* f) { *f = PETSC_FALSE; return 0; }
#define PetscTypeCompare PetscObjectTypeCompare
static inline PetscErrorCode PetscClassIdRegister(const char*, PetscClassId* c) { *c = 0; return 0; }
static inline PetscErrorCode PetscCookieRegister(const char*, PetscCookie* c) { *c = 0; return 0; }

/* ---- Vec ---- */
static inline PetscErrorCode VecCreate(MPI_Comm, Vec* v) { *v = new _p_Vec(); return 0; }
static inline PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) { *v = new _p_Vec(); (*v)->a.assign(n, 0.0); return 0; }
static inline PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt n, PetscInt, Vec* v) { *v = new _p_Vec(); (*v)->a.assign(n, 0.0); return 0; }
static inline PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N) { v->a.assign(n >= 0 ? n : N, 0.0); return 0; }
static inline PetscErrorCode VecSetType(Vec, VecType) { return 0; }
static inline PetscErrorCode VecSetFromOptions(Vec) { return 0; }
static inline PetscErrorCode VecGetArray(Vec v, PetscScalar** a) { *a = v->data(); return 0; }
static inline PetscErrorCode VecRestoreArray(Vec, PetscScalar**) { return 0; }
static inline PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
static inline PetscErrorCode VecGetSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
static inline PetscErrorCode VecGetOwnershipRange(Vec v, PetscInt* a, PetscInt* b) { *a = 0; *b = (PetscInt)v->a.size(); return 0; }
static inline PetscErrorCode VecZeroEntries(Vec v) { for (size_t i = 0; i < v->a.size(); ++i) v->data()[i] = 0; return 0; }
static inline PetscErrorCode VecSet(Vec v, PetscScalar s) { for (size_t i = 0; i < v->a.size(); ++i) v->data()[i] = s; return 0; }
static inline PetscErrorCode VecDuplicate(Vec v, Vec* w) { *w = new _p_Vec(); (*w)->a.assign(v->a.size(), 0.0); return 0; }
static inline PetscErrorCode VecDuplicateVecs(Vec v, PetscInt m, Vec** w) {
  *w = new Vec[m]; for (int i = 0; i < m; ++i) VecDuplicate(v, *w + i); return 0; }
static inline PetscErrorCode VecDestroy(Vec* v) { delete *v; *v = 0; return 0; }
static inline PetscErrorCode VecDestroy(Vec v) { delete v; return 0; }
static inline PetscErrorCode VecDestroyVecs(Vec* v, PetscInt m) { for (int i = 0; i < m; ++i) delete v[i]; delete[] v; return 0; }
static inline PetscErrorCode VecDestroyVecs(PetscInt m, Vec** v) { return VecDestroyVecs(*v, m); }
static inline PetscErrorCode VecCopy(Vec x, Vec y) { for (size_t i = 0; i < x->a.size(); ++i) y->data()[i] = x->data()[i]; return 0; }
static inline PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) { for (size_t i = 0; i < x->a.size(); ++i) y->data()[i] += a * x->data()[i]; return 0; }
static inline PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x) { for (size_t i = 0; i < x->a.size(); ++i) y->data()[i] = x->data()[i] + a * y->data()[i]; return 0; }
static inline PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y) {
  for (size_t i = 0; i < x->a.size(); ++i) w->data()[i] = a * x->data()[i] + y->data()[i]; return 0; }
static inline PetscErrorCode VecScale(Vec x, PetscScalar a) { for (size_t i = 0; i < x->a.size(); ++i) x->data()[i] *= a; return 0; }
static inline PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* d) {
  double s = 0; for (size_t i = 0; i < x->a.size(); ++i) s += x->data()[i] * y->data()[i]; *d = s; return 0; }
static inline PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* r) {
  double s = 0; for (size_t i = 0; i < x->a.size(); ++i) {
    double v = fabs(x->data()[i]); if (t == NORM_INFINITY) s = v > s ? v : s; else if (t == NORM_1) s += v; else s += v * v; }
  *r = (t == NORM_2 || t == NORM_FROBENIUS) ? sqrt(s) : s; return 0; }
static inline PetscErrorCode VecPointwiseMult(Vec w, Vec x, Vec y) { for (size_t i = 0; i < x->a.size(); ++i) w->data()[i] = x->data()[i] * y->data()[i]; return 0; }
static inline PetscErrorCode VecPointwiseDivide(Vec w, Vec x, Vec y) { for (size_t i = 0; i < x->a.size(); ++i) w->data()[i] = x->data()[i] / y->data()[i]; return 0; }
static inline PetscErrorCode VecReciprocal(Vec x) { for (size_t i = 0; i < x->a.size(); ++i) x->data()[i] = 1.0 / x->data()[i]; return 0; }
static inline PetscErrorCode VecPlaceArray(Vec v, const PetscScalar* a) { v->placed = (double*)a; return 0; }
static inline PetscErrorCode VecResetArray(Vec v) { v->placed = 0; return 0; }
static inline PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt* ix, const PetscScalar* y, InsertMode m) {
  for (int i = 0; i < n; ++i) { if (m == ADD_VALUES) v->data()[ix[i]] += y[i]; else v->data()[ix[i]] = y[i]; } return 0; }
static inline PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
static inline PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
static inline PetscErrorCode VecView(Vec, PetscViewer) { return 0; }
static inline PetscErrorCode VecSetRandom(Vec v, PetscRandom r) {
  unsigned long s = r ? r->seed : 1; for (size_t i = 0; i < v->a.size(); ++i) { s = s * 6364136223846793005ul + 1442695040888963407ul; v->data()[i] = double(s >> 11) / double(1ul << 53); } return 0; }
static inline PetscErrorCode PetscRandomCreate(MPI_Comm, PetscRandom* r) { *r = new _p_PetscRandom(); (*r)->seed = 1; return 0; }
static inline PetscErrorCode PetscRandomSetType(PetscRandom, PetscRandomType) { return 0; }
static inline PetscErrorCode PetscRandomSetSeed(PetscRandom r, unsigned long s) { r->seed = s; return 0; }
static inline PetscErrorCode PetscRandomSeed(PetscRandom) { return 0; }
static inline PetscErrorCode PetscRandomSetFromOptions(PetscRandom) { return 0; }
static inline PetscErrorCode PetscRandomDestroy(PetscRandom* r) { delete *r; *r = 0; return 0; }
static inline PetscErrorCode PetscRandomDestroy(PetscRandom r) { delete r; return 0; }

/* ---- Mat ---- */
static inline PetscErrorCode MatCreateShell(MPI_Comm, PetscInt m, PetscInt n, PetscInt, PetscInt, void* ctx, Mat* A) {
  *A = new _p_Mat(); (*A)->ctx = ctx; (*A)->m = m; (*A)->n = n; return 0; }
static inline PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void)) { A->op[op] = (DgShimMatFn)f; return 0; }
static inline PetscErrorCode MatShellGetContext(Mat A, void* ctx) { *(void**)ctx = A->ctx; return 0; }
static inline PetscErrorCode MatShellSetContext(Mat A, void* ctx) { A->ctx = ctx; return 0; }
static inline PetscErrorCode MatMult(Mat A, Vec x, Vec y) {
  return A->op[MATOP_MULT] ? ((PetscErrorCode(*)(Mat, Vec, Vec))A->op[MATOP_MULT])(A, x, y) : 0; }
static inline PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y) {
  return A->op[MATOP_MULT_TRANSPOSE] ? ((PetscErrorCode(*)(Mat, Vec, Vec))A->op[MATOP_MULT_TRANSPOSE])(A, x, y) : 0; }
static inline PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z) {
  return A->op[MATOP_MULT_ADD] ? ((PetscErrorCode(*)(Mat, Vec, Vec, Vec))A->op[MATOP_MULT_ADD])(A, x, y, z) : 0; }
static inline PetscErrorCode MatMultTransposeAdd(Mat A, Vec x, Vec y, Vec z) {
  return A->op[MATOP_MULT_TRANSPOSE_ADD] ? ((PetscErrorCode(*)(Mat, Vec, Vec, Vec))A->op[MATOP_MULT_TRANSPOSE_ADD])(A, x, y, z) : 0; }
static inline PetscErrorCode MatInterpolate(Mat A, Vec x, Vec y) { return MatMultTranspose(A, x, y); }
static inline PetscErrorCode MatGetDiagonal(Mat A, Vec d) {
  return A->op[MATOP_GET_DIAGONAL] ? ((PetscErrorCode(*)(Mat, Vec))A->op[MATOP_GET_DIAGONAL])(A, d) : 0; }
static inline PetscErrorCode MatDestroy(Mat* A) { delete *A; *A = 0; return 0; }
static inline PetscErrorCode MatDestroy(Mat A) { delete A; return 0; }
static inline PetscErrorCode MatCreate(MPI_Comm, Mat* A) { *A = new _p_Mat(); return 0; }
static inline PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt, PetscInt) { A->m = m; A->n = n; return 0; }
static inline PetscErrorCode MatSetType(Mat, MatType) { return 0; }
static inline PetscErrorCode MatSetFromOptions(Mat) { return 0; }
static inline PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt*) { return 0; }
static inline PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*) { return 0; }
static inline PetscErrorCode MatSeqBAIJSetPreallocation(Mat, PetscInt, PetscInt, const PetscInt*) { return 0; }
static inline PetscErrorCode MatMPIBAIJSetPreallocation(Mat, PetscInt, PetscInt, const PetscInt*, PetscInt, const PetscInt*) { return 0; }
static inline PetscErrorCode MatSetValues(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*, const PetscScalar*, InsertMode) { return 0; }
static inline PetscErrorCode MatSetValuesLocal(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*, const PetscScalar*, InsertMode) { return 0; }
static inline PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
static inline PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
static inline PetscErrorCode MatZeroEntries(Mat) { return 0; }
static inline PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n) { if (m) *m = A->m; if (n) *n = A->n; return 0; }
static inline PetscErrorCode MatGetLocalSize(Mat A, PetscInt* m, PetscInt* n) { if (m) *m = A->m; if (n) *n = A->n; return 0; }
static inline PetscErrorCode MatGetVecs(Mat A, Vec* r, Vec* l) {
  if (r) { *r = new _p_Vec(); (*r)->a.assign(A->n, 0.0); } if (l) { *l = new _p_Vec(); (*l)->a.assign(A->m, 0.0); } return 0; }
#define MatCreateVecs MatGetVecs
static inline PetscErrorCode MatView(Mat, PetscViewer) { return 0; }
static inline PetscErrorCode MatSetNullSpace(Mat, MatNullSpace) { return 0; }
static inline PetscErrorCode MatNullSpaceCreate(MPI_Comm, PetscBool, PetscInt, const Vec*, MatNullSpace* s) { *s = 0; return 0; }
static inline PetscErrorCode MatNullSpaceDestroy(MatNullSpace*) { return 0; }
static inline PetscErrorCode MatNullSpaceDestroy(MatNullSpace) { return 0; }
static inline PetscErrorCode MatSetOption(Mat, int, PetscBool) { return 0; }

/* ---- KSP / PC: inert (the oracle restates the solver separately) ---- */
#define DG_SHIM_NOOP(name) template <class... A> static inline PetscErrorCode name(A...) { return 0; }
DG_SHIM_NOOP(KSPSetType) DG_SHIM_NOOP(KSPSetOperators) DG_SHIM_NOOP(KSPSetFromOptions) DG_SHIM_NOOP(KSPSetUp)
DG_SHIM_NOOP(KSPSolve) DG_SHIM_NOOP(KSPSetTolerances) DG_SHIM_NOOP(KSPSetOptionsPrefix) DG_SHIM_NOOP(KSPAppendOptionsPrefix)
DG_SHIM_NOOP(KSPSetInitialGuessNonzero) DG_SHIM_NOOP(KSPSetInitialGuessKnoll) DG_SHIM_NOOP(KSPSetNormType)
DG_SHIM_NOOP(KSPSetPCSide) DG_SHIM_NOOP(KSPSetNullSpace)  DG_SHIM_NOOP(KSPRichardsonSetScale)
 DG_SHIM_NOOP(KSPGetIterationNumber) DG_SHIM_NOOP(KSPGetConvergedReason)
DG_SHIM_NOOP(KSPView) DG_SHIM_NOOP(PCSetType) DG_SHIM_NOOP(PCSetOperators) DG_SHIM_NOOP(PCMGSetLevels)
DG_SHIM_NOOP(PCMGSetType) DG_SHIM_NOOP(PCMGSetCycleType) DG_SHIM_NOOP(PCMGSetInterpolation) DG_SHIM_NOOP(PCMGSetRestriction)
 DG_SHIM_NOOP(PCMGSetX) DG_SHIM_NOOP(PCMGSetRhs) DG_SHIM_NOOP(PCMGSetR)
DG_SHIM_NOOP(PCMGSetNumberSmoothUp) DG_SHIM_NOOP(PCMGSetNumberSmoothDown) DG_SHIM_NOOP(PCSetFromOptions)
DG_SHIM_NOOP(PCSetOptionsPrefix) DG_SHIM_NOOP(PCAppendOptionsPrefix) DG_SHIM_NOOP(PCGetOptionsPrefix)
DG_SHIM_NOOP(KSPGetOptionsPrefix) DG_SHIM_NOOP(PCShellSetSetUp) DG_SHIM_NOOP(PCShellSetName) DG_SHIM_NOOP(PCShellSetDestroy)
DG_SHIM_NOOP(PCShellSetContext) DG_SHIM_NOOP(PCShellSetApply) DG_SHIM_NOOP(PCFactorSetShiftType)
DG_SHIM_NOOP(PCFactorSetShiftPd) DG_SHIM_NOOP(PCSetUp) DG_SHIM_NOOP(PCApply) DG_SHIM_NOOP(PCGetOperators)
DG_SHIM_NOOP(PCRedundantGetPC) DG_SHIM_NOOP(PCRedundantGetKSP) DG_SHIM_NOOP(KSPSetDM) DG_SHIM_NOOP(PetscViewerASCIIOpen)
DG_SHIM_NOOP(PetscViewerDestroy) DG_SHIM_NOOP(PetscViewerASCIISetTab) 
   
DG_SHIM_NOOP(PetscObjectReference) DG_SHIM_NOOP(PetscObjectDereference) DG_SHIM_NOOP(PCShellGetContext)
static inline PetscErrorCode KSPMonitorDefault(KSP, PetscInt, PetscReal, void*) { return 0; }
static inline PetscErrorCode KSPConvergedSkip(KSP, PetscInt, PetscReal, KSPConvergedReason*, void*) { return 0; }
static inline PetscErrorCode KSPDefaultConverged(KSP, PetscInt, PetscReal, KSPConvergedReason*, void*) { return 0; }
static inline PetscErrorCode PCMGResidualDefault(Mat, Vec, Vec, Vec) { return 0; }
#define PCMGDefaultResidual PCMGResidualDefault
template <class... A> static inline PetscErrorCode KSPSetConvergenceTest(A...) { return 0; }
template <class... A> static inline PetscErrorCode KSPMonitorSet(A...) { return 0; }
template <class... A> static inline PetscErrorCode PCMGSetResidual(A...) { return 0; }
static inline PetscErrorCode KSPCreate(MPI_Comm, KSP* k) { *k = new _p_KSP(); return 0; }
static inline PetscErrorCode KSPDestroy(KSP* k) { delete *k; *k = 0; return 0; }
static inline PetscErrorCode KSPDestroy(KSP k) { delete k; return 0; }
static inline PetscErrorCode KSPGetPC(KSP k, PC* p) { *p = &k->pc; return 0; }
static inline PetscErrorCode PCMGGetSmoother(PC, PetscInt, KSP* k) { static _p_KSP s; *k = &s; return 0; }
static inline PetscErrorCode PCMGGetSmootherUp(PC, PetscInt, KSP* k) { static _p_KSP s; *k = &s; return 0; }
static inline PetscErrorCode PCMGGetSmootherDown(PC, PetscInt, KSP* k) { static _p_KSP s; *k = &s; return 0; }
static inline PetscErrorCode PCMGGetCoarseSolve(PC, KSP* k) { static _p_KSP s; *k = &s; return 0; }

#endif
