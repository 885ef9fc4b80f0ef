/* Single-process stand-in for the MPI interface the reference uses, so that
 * its octree / mesh / operator sources compile and run as one rank.  Every
 * collective degenerates to a copy from the send to the receive buffer.
 * Written for the oracle build only (test infrastructure). */
#ifndef DG_SHIM_MPI_H
#define DG_SHIM_MPI_H

#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Group;
typedef int MPI_Request;
typedef int MPI_Errhandler;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_GROUP_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_SUCCESS 0
#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_MAX_PROCESSOR_NAME 64

#define MPI_OP_NULL 0
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_LOR 6
#define MPI_BAND 7
#define MPI_BOR 8
#define MPI_MAXLOC 9
#define MPI_MINLOC 10

/* predefined datatypes: handle = index into the size table */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR 1
#define MPI_SIGNED_CHAR 1
#define MPI_UNSIGNED_CHAR 2
#define MPI_BYTE 3
#define MPI_SHORT 4
#define MPI_UNSIGNED_SHORT 5
#define MPI_INT 6
#define MPI_UNSIGNED 7
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 9
#define MPI_LONG_LONG_INT 10
#define MPI_LONG_LONG 10
#define MPI_UNSIGNED_LONG_LONG 11
#define MPI_FLOAT 12
#define MPI_DOUBLE 13
#define MPI_LONG_DOUBLE 14
#define MPI_DOUBLE_INT 15
#define MPI_FLOAT_INT 16
#define MPI_2INT 17
#define MPI_C_BOOL 18
#define MPI_CXX_BOOL 18
#define MPI_WCHAR 19
#define MPI_C_COMPLEX 20
#define MPI_C_DOUBLE_COMPLEX 21
#define MPI_DOUBLE_COMPLEX 21
#define MPI_COMPLEX 20
#define MPI_SHIM_FIRST_DERIVED 32

#ifdef __cplusplus
extern "C++" {
#endif

static inline size_t* dg_shim_type_sizes(void) {
  static size_t t[4096] = {0, 1, 1, 1, 2, 2, 4, 4, 8, 8, 8, 8, 4, 8, 16, 12, 8, 8, 1, 4, 8, 16};
  return t;
}
static inline int* dg_shim_type_next(void) {
  static int n = MPI_SHIM_FIRST_DERIVED;
  return &n;
}
static inline size_t dg_shim_size(MPI_Datatype t) { return dg_shim_type_sizes()[t]; }
static inline void dg_shim_copy(const void* s, void* r, int count, MPI_Datatype t) {
  if (s == MPI_IN_PLACE || s == r || count <= 0) return;
  memmove(r, s, (size_t)count * dg_shim_size(t));
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Init_thread(int*, char***, int, int* p) { if (p) *p = 0; return 0; }
static inline int MPI_Initialized(int* f) { *f = 1; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Finalized(int* f) { *f = 0; return 0; }
static inline int MPI_Abort(MPI_Comm, int c) { exit(c); return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int, MPI_Comm* n) { *n = color == MPI_UNDEFINED ? MPI_COMM_NULL : c; return 0; }
static inline int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* r) { *r = a == b ? MPI_IDENT : MPI_CONGRUENT; return 0; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return 0; }
static inline int MPI_Group_incl(MPI_Group, int n, const int*, MPI_Group* g) { *g = n > 0 ? 1 : MPI_GROUP_NULL; return 0; }
static inline int MPI_Group_free(MPI_Group* g) { *g = MPI_GROUP_NULL; return 0; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm* n) { *n = g ? c : MPI_COMM_NULL; return 0; }
static inline int MPI_Get_processor_name(char* n, int* l) { strcpy(n, "localhost"); *l = 9; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* t) {
  int id = (*dg_shim_type_next())++;
  dg_shim_type_sizes()[id] = (size_t)count * dg_shim_size(old);
  *t = id;
  return 0;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) { *t = MPI_DATATYPE_NULL; return 0; }
static inline int MPI_Type_size(MPI_Datatype t, int* s) { *s = (int)dg_shim_size(t); return 0; }
static inline int MPI_Op_create(void*, int, MPI_Op* op) { *op = 100; return 0; }
static inline int MPI_Op_free(MPI_Op* op) { *op = MPI_OP_NULL; return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Gatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d, MPI_Datatype, int, MPI_Comm) {
  dg_shim_copy(s, (char*)r + (size_t)d[0] * dg_shim_size(t), n, t); return 0; }
static inline int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d, MPI_Datatype, MPI_Comm) {
  dg_shim_copy(s, (char*)r + (size_t)d[0] * dg_shim_size(t), n, t); return 0; }
static inline int MPI_Alltoall(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) { dg_shim_copy(s, r, n, t); return 0; }
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*, const int* rd,
                                MPI_Datatype, MPI_Comm) {
  dg_shim_copy((const char*)s + (size_t)sd[0] * dg_shim_size(st), (char*)r + (size_t)rd[0] * dg_shim_size(st), sc[0], st);
  return 0;
}
/* Point-to-point: one pending self-message mailbox per (tag) is enough for the
 * single-rank paths, which never message themselves in the code exercised. */
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Ssend(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status* st) { if (st) st->count = 0; return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Issend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Sendrecv(const void* s, int sn, MPI_Datatype st, int, int, void* r, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
  dg_shim_copy(s, r, sn, st); return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Test(MPI_Request*, int* f, MPI_Status*) { *f = 1; return 0; }
static inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype, int* c) { *c = s ? s->count : 0; return 0; }
static inline int MPI_Probe(int, int, MPI_Comm, MPI_Status* s) { if (s) s->count = 0; return 0; }
static inline int MPI_Iprobe(int, int, MPI_Comm, int* f, MPI_Status*) { *f = 0; return 0; }

#ifdef __cplusplus
}
#endif

#endif
