/*
 * dendro_b200 -- C ABI of the B200 matrix-free octree finite-element path.
 *
 * Plain pointers and sizes only.  Every entry point returns a dg_status
 * (0 = OK) and never traps; a failed call leaves a message retrievable with
 * dg_last_error().  Handles are opaque, owned by the library, and are not to
 * be shared between host threads; calls on different handles are reentrant.
 *
 * Each declaration names the reference (hsundar/dendro) interface it stands
 * in for, by file:line within that project.
 */
#ifndef DENDRO_B200_H
#define DENDRO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Errors: PetscErrorCode / CHKERRQ (include/oda/oda.h:26-28) and the
 * assert(false) paths (include/oda/odaUtils.txx:89-91) become status codes. */
typedef enum dg_status {
  DG_OK = 0,
  DG_EINVAL = 1,          /* bad argument, size or pointer kind */
  DG_ENOMEM = 2,          /* device allocation failed */
  DG_ECUDA = 3,           /* a CUDA runtime call failed */
  DG_ENOTCONVERGED = 4,   /* iteration cap reached before the tolerance */
  DG_ETIMEOUT = 5,        /* a bounded device wait ran out */
  DG_EUNBALANCED = 6,     /* octree not linear / complete / 2:1 balanced */
  DG_EDEPTH = 7,          /* maxDepth outside the supported range */
  DG_ENOTIMPL = 8
} dg_status;

/* Octant record: anchor and level|flags with the reference's flag bits
 * (ot::TreeNode, include/oct/TreeNode.h:40,77-78: level mask 31,
 * BOUNDARY 64, NODE 128). */
typedef struct dg_octant {
  uint32_t x, y, z, level_flags;
} dg_octant;

typedef struct dg_octree dg_octree; /* device-resident sorted linear octree */
typedef struct dg_da dg_da;         /* device-resident mesh (ot::DA)         */
typedef struct dg_mat dg_mat;       /* operator on a mesh (PETSc MatShell)   */
typedef struct dg_damg dg_damg;     /* multigrid hierarchy (ot::DAMG)        */
typedef struct dg_mlp dg_mlp;       /* learned post-smoother (no reference counterpart) */
typedef struct dg_halo dg_halo;     /* one rank's part of a partitioned mesh (ot::DA, npes > 1) */
typedef struct dg_parcsr dg_parcsr; /* one rank's rows of a sparse matrix between partitioned levels */

const char* dg_status_string(dg_status s);
/* Copies the last error message of the calling thread into buf. */
void dg_last_error(char* buf, size_t n);
/* Number of CUDA devices visible (0 on a host without a GPU). */
int dg_device_count(void);

/* ------------------------------------------------------------- octree --- */

/* ot::points2Octree / points2OctreeSeq (src/oct/Construct.C:727,880):
 * quantise n points in [0,1)^3 (xyz interleaved FP64) at maxDepth, sort by
 * Morton key and emit the coarsest leaves holding <= maxNumPts points.
 * pts_on_device: 1 when pts is a device pointer, 0 for host memory. */
dg_status dg_points2octree(const double* pts, int64_t n, int pts_on_device, uint32_t max_depth,
                           uint32_t max_num_pts, dg_octree** out);

/* Wrap an existing sorted linear octree (e.g. read from an .ot file). */
dg_status dg_octree_from_octants(const dg_octant* octs, int64_t n, int on_device, uint32_t max_depth,
                                 dg_octree** out);

/* ot::balanceOctree with incCorner = true (src/oct/Balance.C:31): the
 * coarsest 2:1 (face, edge and corner) balanced refinement. */
dg_status dg_balance_octree(const dg_octree* in, dg_octree** out);

/* ot::coarsenOctree, sequential form (src/oct/Coarsen.C:53-104). */
dg_status dg_coarsen_octree(const dg_octree* in, dg_octree** out);

int64_t dg_octree_size(const dg_octree* t);
uint32_t dg_octree_max_depth(const dg_octree* t);
/* Copy the octants to host memory (n = dg_octree_size entries). */
dg_status dg_octree_export(const dg_octree* t, dg_octant* host_out);
void dg_octree_destroy(dg_octree* t);

/* ------------------------------------------------------------ files --- */
/* The reference drivers' file formats, on the host (no GPU needed for the
 * point files).  Point files: readPtsFromFile / writePtsToFile
 * (src/oct/OctFunctions.C:313-341, 370-385): uint32 count, then xyz FP64
 * interleaved; the writer leaves the file empty for no points, and an empty
 * file reads as no points.  dg_read_pts with pts == NULL only returns the
 * count; otherwise capacity (in points) must hold it. */
dg_status dg_write_pts(const char* path, const double* pts, int64_t n);
dg_status dg_read_pts(const char* path, double* pts, int64_t capacity, int64_t* n);
/* Points with one value each: readDataPtsFromFile / writeDataPtsToFile
 * (OctFunctions.C:343-368, 387-401): the count, the coordinates, the values. */
dg_status dg_write_data_pts(const char* path, const double* pts, const double* vals, int64_t n);
dg_status dg_read_data_pts(const char* path, double* pts, double* vals, int64_t capacity, int64_t* n);
/* Octree files (.ot): writeNodesToFile / readNodesFromFile
 * (OctFunctions.C:403-439): "3 maxDepth", the count, "x y z level" per octant
 * (flags are not written).  The reader rejects a file that is not a sorted
 * linear octree (DG_EUNBALANCED), as dg_octree_from_octants does. */
dg_status dg_octree_write(const dg_octree* t, const char* path);
dg_status dg_octree_read(const char* path, dg_octree** out);

/* ---------------------------------------------------------------- mesh --- */

/* ot::DA::DA (include/oda/oda.h:500; src/oda/oda.C:175 -> DA_FactoryPart0..3,
 * src/oda/private/odaFactory.C:100-880) on one GPU: embeds the balanced
 * octree at maxDepth+1 with positive-boundary pseudo-octants
 * (addBoundaryNodesType1, src/oct/OctFunctions.C:636), flags non-hanging
 * anchors (flagNodesType3, OctFunctions.C:1501) and builds the element->node
 * map with hanging masks, child numbers and element types (buildNodeList,
 * src/oda/private/odaBuildNlist.C:47-856).  The input octree is not consumed. */
/* Meshes take octrees of maxDepth <= 18 (DG_EDEPTH above). */
dg_status dg_da_create(const dg_octree* balanced, dg_da** out);

/* Build a mesh from maps computed elsewhere (host arrays): nlist [E][8] node
 * ids, level [E] (embedded level), cnum [E], hmask [E], node anchors
 * [N][3] (embedded coordinates), element anchors [E][3]. */
dg_status dg_da_create_from_maps(int64_t E, int64_t N, uint32_t max_depth, const uint32_t* nlist,
                                 const uint8_t* level, const uint8_t* cnum, const uint8_t* hmask,
                                 const uint32_t* node_xyz, const uint32_t* elem_xyz, dg_da** out);

/* Sizes: elements (getElementSize), nodes (getNodeSize + getBoundaryNodeSize,
 * include/oda/oda.h:668-684) and positive-boundary pseudo-octants. */
dg_status dg_da_sizes(const dg_da* da, int64_t* elements, int64_t* nodes, int64_t* pseudo_octants);
uint32_t dg_da_max_depth(const dg_da* da); /* embedded depth (maxDepth + 1) */
/* Parent octants with at least one leaf child: the units of the octet
 * operator kernels (no reference counterpart; 0 for batched meshes). */
int64_t dg_da_octets(const dg_da* da);

/* Load vector of the Neumann problem (ComputeRHS_omgNeumann,
 * examples/src/backend/omgNeumann.C:749-785): force [E] sampled at the
 * element centres (the order of dg_da_element_centers), b [N] =
 * sum over elements of force_e h^3/8 RHSType2Stencil[childNum][elemType]
 * at the element's nodes.  Host or device arrays (on_device). */
dg_status dg_da_load_vector(const dg_da* da, const double* force, double* b, int on_device);

/* Compressed element map: the DA's compressLut option (the remainder and
 * quotient arrays m_ucpLutRemainders / m_uspLutQuotients, include/oda/oda.h:
 * 332-341, decoded by getNodeIndices, include/oda/oda.txx:1125-1300) in a
 * warp-tile form: per tile of 32 elements the smallest node id, per element a
 * byte remainder of each node's offset from it and a 16-bit quotient where the
 * offset needs one (a tile whose quotients exceed quotient_bits bits keeps
 * 32-bit quotients).  quotient_bits is 16 normally (1..16; smaller values make
 * wide tiles for tests).  Once built, the operator's autotuner also times the
 * element kernel that reads this map ("element, compressed map"). */
dg_status dg_da_compress_maps(dg_da* da, int quotient_bits);
/* Bytes of the compressed map (0 when not built); *wide_tiles (may be NULL)
 * receives the number of tiles with 32-bit quotients. */
int64_t dg_da_compressed_map_bytes(const dg_da* da, int64_t* wide_tiles);
/* The element map decoded from the compressed form on the device, into host
 * nlist [E][8] (the layout of dg_da_export). */
dg_status dg_da_decompress_maps(const dg_da* da, uint32_t* nlist);

/* Copy the maps to host memory; any pointer may be NULL.  nlist [E][8]
 * (getNodeIndices, include/oda/oda.txx:1111), hmask [E]
 * (getHangingNodeIndex, src/oda/oda.C:784), cnum [E] (getChildNumber,
 * oda.txx:1087), etype [E] (GET_ETYPE_BLOCK, include/oda/odaUtils.h:334),
 * level [E] (getLevel), node anchors [N][3], element anchors [E][3],
 * node_bdy [N] (1 on the domain boundary). */
dg_status dg_da_export(const dg_da* da, uint32_t* nlist, uint8_t* hmask, uint8_t* cnum, uint8_t* etype,
                       uint8_t* level, uint32_t* node_xyz, uint32_t* elem_xyz, uint8_t* node_bdy);

/* Element centres in [0,1]^3, xyz interleaved (CalculateCenters,
 * examples/src/backend/omgNeumann.C:788-820); out is host memory [E][3]. */
dg_status dg_da_element_centers(const dg_da* da, double* host_out);
/* The files of examples/src/drivers/dumpMesh.C for one rank of one:
 * <prefix>_NL_0_1.out (node count; per node, in order of first visit over
 * the elements, anchor x y z and global id), <prefix>_EL_0_1.out (maxDepth,
 * element count; per element anchor x y z, level - 1, global id) and
 * <prefix>_M_0_1.out (element count; per element its id and 8 node ids);
 * 4-byte integers, embedded coordinates.  Byte-identical to the reference's
 * output on the same balanced octree. */
dg_status dg_da_dump_mesh(const dg_da* da, const char* prefix);
void dg_da_destroy(dg_da* da);

/* ----------------------------------------------------------- operators --- */

typedef enum dg_prec {
  DG_PREC_F64 = 0,        /* FP64 vectors and arithmetic                      */
  DG_PREC_F32 = 1,        /* FP32 vectors, FP32 coefficients and accumulation */
  DG_PREC_F32_BF16COEF = 2 /* FP32 vectors, BF16-stored coefficients          */
} dg_prec;

/* CreateJacobian2 / Jacobian2MatMult (examples/src/backend/omgNeumann.C:533,
 * 643-745): -div(a grad u) + b u with per-element coefficients
 * coef[2*e] = a_e, coef[2*e+1] = b_e (host memory), or a = b = 1 when coef is
 * NULL (Jacobian1, examples/src/backend/odaJac.C:271-290). */
dg_status dg_mat_create_lapmass(dg_da* da, const double* coef, dg_mat** out);

/* ElasticityMatMult (examples/src/backend/elasticityJac.C:130-230): 3 dof per
 * node, mu h/2 (L x I3) + (mu+lambda) h/2 GD, Dirichlet rows set to the input
 * and Dirichlet columns skipped.  dirichlet: host [N] flags, or NULL for all
 * domain-boundary nodes. */
dg_status dg_mat_create_elasticity(dg_da* da, double mu, double lambda, const uint8_t* dirichlet,
                                   dg_mat** out);

/* MatMult (MATOP_MULT of the MatShell, omgNeumann.C:700-710): y = A x with
 * device pointers on the given CUDA stream (NULL = default stream). */
/* CreateDirichletLaplacian / CreateDirichletJacobian with their MatMult and
 * GetDiagonal (examples/src/backend/omgJac.C:61-269, 859-1160): unit
 * coefficients, h/2 L (with_mass = 0) or h/2 L + h^3/8 M (with_mass = 1); the
 * rows of the nodes flagged in dirichlet [N] are the identity and their
 * columns are dropped.  dirichlet == NULL: the domain-boundary nodes
 * (assignBoundaryFlags, src/oda/odaUtils.C:1054). */
dg_status dg_mat_create_dirichlet(dg_da* da, int with_mass, const uint8_t* dirichlet, dg_mat** out);
dg_status dg_mat_mult(dg_mat* A, const double* x, double* y, void* stream);
/* y += A x for the scalar operator (PETSc MatMultAdd with y as both the
 * addend and the result), FP64, one launch and no clearing pass: the
 * dependent elements of a partitioned mesh add into the local vector. */
dg_status dg_mat_mult_add(dg_mat* A, const double* x, double* y, void* stream);
/* FP32 inner-solver form of the same operator. */
dg_status dg_mat_mult_f32(dg_mat* A, const float* x, float* y, void* stream);
/* y += A x in FP32 (the FP32 coefficient copy): the dependent elements of a
 * partitioned mesh in the FP32 inner V-cycle. */
dg_status dg_mat_mult_add_f32(dg_mat* A, const float* x, float* y, void* stream);
/* MATOP_GET_DIAGONAL (Jacobian2MatGetDiagonal, omgNeumann.C:442-465). */
dg_status dg_mat_get_diagonal(dg_mat* A, double* d, void* stream);
/* Same as dg_mat_mult with host x and y: copies in, applies, copies out and
 * synchronises (the call a PETSc MatShell callback makes on host Vec arrays).
 * On scalar meshes of more than 2^20 elements, after the first call, the
 * copies run in chunks overlapped with the operator when x and y are both
 * page-locked (cudaHostAlloc / cudaHostRegister); with pageable buffers the
 * call copies x in, applies the operator and copies y out, one after another. */
dg_status dg_mat_mult_host(dg_mat* A, const double* x, double* y);
/* Synchronise `stream`; DG_ETIMEOUT when a bounded device wait of an
 * operator kernel (the bulk-copy staged launch shape waits for its copies)
 * has run out since the last check, which clears it.  The results of the
 * launches concerned are not valid.  When, after such a timeout, the copies
 * still in flight did not land within a second bounded wait either, the
 * error message says so: a copy may then have written into shared memory
 * that a later block of any kernel owned, and every result computed since the
 * last check is void.  dg_mat_mult_host and dg_damg_solve make
 * the same check.  No reference counterpart: PETSc's MatMult reports errors
 * through its return code (Jacobian2MatMult, omgNeumann.C:533-556, returns 0). */
dg_status dg_device_check(void* stream);
/* Test hook: the clock64 cycles such a wait lasts before it gives up
 * (<= 0 restores the default of 2^31 cycles, about one second). */
dg_status dg_set_device_wait_limit(int64_t cycles);
int64_t dg_mat_size(const dg_mat* A); /* rows = dof * nodes */
/* Launch shape of the scalar operator kernel that the autotuner picked on the
 * first application in the given precision ("untuned" before it). */
const char* dg_mat_kernel_name(const dg_mat* A, int prec);
/* Number of launch shapes the autotuner chooses from, and a way to fix one
 * (0 <= variant < count) for a mesh and precision instead of timing them
 * (no reference counterpart; testing and benchmarking). */
int dg_mat_kernel_count(void);
/* Y = A X for nrhs right-hand sides at once (no reference counterpart: the
 * reference's Jacobian2MatMult, omgNeumann.C:533, takes one Vec).  X and Y are
 * device arrays, node-major [N][nrhs] FP32, 16-byte aligned; nrhs a multiple
 * of 16.  The element contraction runs on the tensor cores with TF32 inputs
 * and FP32 accumulation; split = 3 splits each input into a TF32 high part and
 * a TF32 remainder (three products, FP32-level accuracy), split = 1 uses one
 * TF32 product (both with mma.sync on the warp tiles); split = 5 and split = 4
 * are the same two precisions on the 5th-generation tensor cores (tcgen05.mma
 * with accumulators in tensor memory: per pair of element parents their
 * assembled 27 x 27 lattice matrix times the lattice rows of X; nrhs a
 * multiple of 64); split = 0 runs the octet form on the CUDA cores instead (a
 * warp per element parent and 32 right-hand sides, exact FP32 products;
 * nrhs a multiple of 32).  Scalar Laplacian + mass operators only. */
dg_status dg_mat_mult_multi(dg_mat* A, const float* X, float* Y, int nrhs, int split, void* stream);
dg_status dg_mat_set_kernel(dg_mat* A, int prec, int variant);
void dg_mat_destroy(dg_mat* A);

/* ------------------------------------------------------------ multigrid --- */

typedef struct dg_damg_config {
  int nlevels;          /* requested levels; fewer when a level drops below 500 octants */
  int nu_pre, nu_post;  /* damped-Jacobi sweeps (bin/options:187-194) */
  double omega;         /* Richardson scale (bin/options: 0.667) */
  double rtol;          /* ||b - A x||_2 <= rtol ||b||_2 */
  int maxit;            /* outer iteration cap */
  int inner_prec;       /* dg_prec of the V-cycle (F64, or F32 inside FP64 outer) */
  int use_graph;        /* capture the V-cycle in a CUDA graph */
  int coarse_op;        /* operators below the finest level: 0 from the level's averaged coefficients
                           (Jacobian2 with ASSIGN_MAT_PROP_FINE_TO_COARSE, omgNeumann.C:73-113); 1 from the
                           next finer level's coefficients (Jacobian3, examples/src/backend/omgJac.C:2139-2340:
                           a coarse element whose 8 children's coefficients differ takes the sum of the
                           children's operators, the type-1 stencils); the Jacobi diagonal is the averaged
                           operator's either way, as the reference's B matrix */
  int dof;              /* degrees of freedom per node (DAMGCreateAndSetDA's dof, include/omg/omg.h:470-473):
                           1 the Laplacian + mass operator; 3 linear elasticity (ElasticityMatMult,
                           examples/src/backend/elasticityJac.C:130-230) on every level with that level's
                           boundary nodes as Dirichlet nodes, as examples/src/drivers/newElasSolver.C:279-361
                           sets it up (FP64 V-cycle, single mesh, coarse_op 0) */
  double mu, lambda;    /* Lame parameters of the dof-3 operator (SetElasticityContexts defaults: 1, 1) */
} dg_damg_config;

typedef struct dg_solve_report {
  int iterations;
  int converged;
  double rel_residual;  /* FP64 ||b - A x||_2 / ||b||_2 at exit */
  double solve_ms;      /* device time of the solve */
  int smoother_fallbacks; /* learned smoother replaced by damped Jacobi during the solve */
} dg_solve_report;

void dg_damg_default_config(dg_damg_config* cfg);

/* DAMGCreateAndSetDA (include/omg/omg.h:470; src/omg/omg.C:1306-1420): level
 * hierarchy by coarsenOctree + balanceOctree, a mesh per level, and the
 * transfer operators of createInterpolationType1 (omg.C:2234-2290). */
dg_status dg_damg_create(const dg_octree* finest_balanced, const dg_damg_config* cfg, dg_damg** out);
/* Many independent meshes as one hierarchy (the batched form): every mesh gets
 * the same number of levels (the smallest natural count over the meshes),
 * level l of all meshes is concatenated into one mesh with per-mesh node-id
 * offsets, transfers are block diagonal and the coarsest level is solved with
 * one dense block per mesh.  One kernel launch then serves all meshes; the
 * solve stops when every mesh reaches rtol on its own ||b_i||.  Vectors and
 * coefficients are the per-mesh arrays concatenated in mesh order. */
dg_status dg_damg_create_batch(const dg_octree* const* finest_balanced, int count, const dg_damg_config* cfg,
                               dg_damg** out);
int dg_damg_batch_count(const dg_damg* m);
/* Element and node offsets of each mesh on a level (count + 1 entries each). */
dg_status dg_damg_batch_offsets(const dg_damg* m, int level, int64_t* elem_off, int64_t* node_off);

/* DAMGSetKSP with CreateJacobian2 (omg.h:488; omgNeumann.C:643): finest-level
 * coefficients (host, 2 per element or NULL), coarse levels averaged as
 * SetPDECoefFromPts (omgNeumann.C:73-113,188-297). */
dg_status dg_damg_set_lapmass(dg_damg* m, const double* coef);
/* DAMGSolve (omg.h:492; omg.C:1121-1169): CG with V(nu_pre, nu_post)
 * preconditioning.  b and x are host arrays when on_device = 0. */
dg_status dg_damg_solve(dg_damg* m, const double* b, double* x, int on_device, dg_solve_report* rep);

/* Many right-hand sides on one mesh, solved together: B and X node-major
 * [N][nrhs] FP64 (nrhs 32, 64, 128 or 256), one flexible PCG per column in
 * FP64 around one V-cycle per iteration for all columns (the cycle in the
 * configuration's inner precision; its operator applications are the octet
 * multi-right-hand-side kernel).  Stops when every column's relative residual
 * is at or below rtol; rep: iterations, the largest relative residual, device
 * time.  One mesh, the scalar operator, coarse_op 0.  No reference
 * counterpart (the reference solves one Vec at a time, DAMGSolve,
 * include/omg/omg.h:492). */
dg_status dg_damg_solve_multi(dg_damg* m, const double* B, double* X, int nrhs, int on_device,
                              dg_solve_report* rep);
/* Relative residual target and iteration limit of later solves (the
 * reference sets them through PETSc, KSPSetTolerances / -ksp_rtol,
 * bin/options:50-53). */
dg_status dg_damg_set_tolerances(dg_damg* m, double rtol, int maxit);
int dg_damg_levels(const dg_damg* m);
dg_status dg_damg_level_sizes(const dg_damg* m, int64_t* elements, int64_t* nodes);
dg_da* dg_damg_level_da(dg_damg* m, int level); /* 0 = finest; owned by m */
/* P (fine level l from level l+1) applied to host or device vectors. */
dg_status dg_damg_prolong(dg_damg* m, int level, const double* xc, double* xf, int on_device);
dg_status dg_damg_restrict(dg_damg* m, int level, const double* rf, double* rc, int on_device);
/* The transfer matrices between level and level + 1 as CSR, copied to host
 * memory: which 0 = P (rows: the nodes of level, columns: the nodes of
 * level + 1; prolongMatVecType2, src/omg/ProlongMatVec.C:83-284), which 1 =
 * R = P^T (rows: the nodes of level + 1).  *nnz receives the entry count;
 * ptr [rows + 1], col and val [nnz] may be NULL (ask for nnz first). */
dg_status dg_damg_transfer_export(dg_damg* m, int level, int which, int64_t* nnz, uint32_t* ptr, uint32_t* col,
                                  double* val);
/* The level's element coefficients (a, b per element, host [2 E_level]): the
 * finest level's as set, the coarser ones averaged (omgNeumann.C:73-113). */
dg_status dg_damg_level_coef(dg_damg* m, int level, double* coef);
/* x = A_c^-1 b on the coarsest level (the dense inverse set up with the
 * operators); device pointers [N_coarsest], asynchronous on `stream`. */
dg_status dg_damg_coarse_solve(dg_damg* m, const double* b, double* x, void* stream);
void dg_damg_destroy(dg_damg* m);

/* PCApply of the multigrid preconditioner: one V-cycle on device vectors. */
/* y = J x on one level (0 = finest): the operator the V-cycle smooths and
 * takes residuals with on that level (MatMult of damg[l]->J). */
dg_status dg_damg_level_apply(dg_damg* m, int level, const double* x, double* y, int on_device);
dg_status dg_damg_vcycle(dg_damg* m, const double* b, double* x);

/* ------------------------------------------------- partitioned meshes --- */

/* par::partitionW (include/par/parUtils.txx:1011-1177) on a list held whole:
 * n items with integer weights (NULL: 1 each) into nranks contiguous ranges
 * of equal weight, the first W % nranks ranks one unit heavier; rank r gets
 * items first[r] .. first[r+1] - 1 (first has nranks + 1 entries).  Host only. */
dg_status dg_partition_weighted(int64_t n, const uint32_t* weights, int nranks, int64_t* first);

/* One rank's part of a mesh split over nranks ranks: the DA that the
 * reference builds per rank (ot::DA ctor, include/oda/oda.h:500-512, with
 * the scatter maps of prepareAprioriCommMessagesInDAtype2,
 * src/oda/private/odaFactory.C:199-460).  Elements are partitioned by
 * dg_partition_weighted (weights per element, NULL: 1 each); a node belongs
 * to the rank whose element range holds its anchor, so each rank owns a
 * contiguous range of node ids.  The rank keeps every element with a vertex
 * it owns: independent elements (all vertices owned) and dependent ones.
 * Local node ids: owned nodes first, then ghost nodes ascending by global id
 * (grouped by owner rank).  Inputs are the maps of dg_da_export (host
 * arrays; node ids in the Morton order of their anchors).  Host only: no GPU
 * is touched until the exchange calls below. */
dg_status dg_halo_create(int64_t E, int64_t N, uint32_t max_depth, const uint32_t* nlist, const uint8_t* level,
                         const uint8_t* cnum, const uint8_t* hmask, const uint32_t* node_xyz, const uint32_t* elem_xyz,
                         const uint32_t* weights, int nranks, int rank, dg_halo** out);
/* The same from a mesh on the GPU (exports its maps first). */
dg_status dg_halo_create_from_da(const dg_da* da, const uint32_t* weights, int nranks, int rank, dg_halo** out);
/* Sizes: owned and ghost nodes, the global id of the first owned node, the
 * independent and dependent elements and the local nodes the dependent
 * Any pointer may be NULL. */
dg_status dg_halo_sizes(const dg_halo* h, int64_t* n_owned, int64_t* n_ghost, int64_t* first_owned,
                        int64_t* n_independent, int64_t* n_dependent);
/* Element and node ranges of all ranks, [nranks + 1] each. */
dg_status dg_halo_ranges(const dg_halo* h, int64_t* elem_first, int64_t* node_first);
/* The exchange plan (m_uipSendProcs / m_uipSendCounts / m_uipScatterMap and
 * m_uipRecvProcs / m_uipRecvCounts, include/oda/oda.h:426-438): values sent
 * to and received from each rank [nranks]; the local ids of the owned nodes
 * sent, by destination rank then ascending; the ghosts' global ids. */
dg_status dg_halo_comm(const dg_halo* h, int64_t* send_counts, int64_t* recv_counts, uint32_t* send_idx,
                       uint32_t* ghosts);
/* A part's elements (which 0: independent, 1: dependent): global element ids
 * [E_part] and their local node ids [E_part][8] (part 0: owned nodes only). */
dg_status dg_halo_part(const dg_halo* h, int which, int64_t* elems, uint32_t* nlist);
/* The part's mesh on the current GPU (part 0 over the owned nodes, part 1
 * over all local nodes, so that dg_mat_mult_add adds its elements into a
 * local vector in place); DG_EINVAL for a part without elements. */
dg_status dg_halo_local_da(const dg_halo* h, int which, dg_da** out);
/* ReadFromGhostsBegin's send buffer (include/oda/oda.txx:479-500):
 * send[k] = x_local[send_idx[k]] for dof values per node; device pointers,
 * asynchronous on `stream`.  The received values, concatenated by source
 * rank, are x_local's ghost slots (x_local + dof * n_owned). */
dg_status dg_halo_pack(dg_halo* h, const double* x_local, double* send, int dof, void* stream);
/* The same for FP32 vectors (the FP32 inner V-cycle's exchanges). */
dg_status dg_halo_pack_f32(dg_halo* h, const float* x_local, float* send, int dof, void* stream);
/* WriteToGhostsEnd (include/oda/oda.txx:609-640): y_local[send_idx[k]] +=
 * recv[k] for k in order, recv being the peers' ghost slots concatenated by
 * source rank (what they send in WriteToGhostsBegin, oda.txx:566-605). */
dg_status dg_halo_accumulate(dg_halo* h, const double* recv, double* y_local, int dof, void* stream);
void dg_halo_destroy(dg_halo* h);

/* The rows of a sparse matrix that one rank owns, for products between two
 * partitioned levels: the multigrid transfers of a partitioned hierarchy
 * (prolongMatVecType2 / restrictMatVecType2, src/omg/ProlongMatVec.C:83-284,
 * src/omg/RestrictMatVec.C:486-619, whose coarse values the reference reads
 * with ReadFromGhosts and whose contributions it adds with WriteToGhosts).
 * M is CSR on the host [nrows x ncols]; rank r owns rows row_first[r] ..
 * row_first[r+1] - 1 and the input values of columns col_first[r] ..
 * col_first[r+1] - 1 (both [nranks + 1]).  Host only until the calls below. */
dg_status dg_parcsr_create(int64_t nrows, int64_t ncols, const uint32_t* ptr, const uint32_t* col, const double* val,
                           const int64_t* row_first, const int64_t* col_first, int nranks, int rank, dg_parcsr** out);
dg_status dg_parcsr_sizes(const dg_parcsr* pc, int64_t* n_rows, int64_t* n_cols_owned, int64_t* n_ghost,
                          int64_t* nnz);
/* The exchange plan: input values sent to / received from each rank, the
 * owned columns sent (by destination rank, then ascending) and the ghost
 * columns' global ids (ascending, so grouped by owner rank). */
dg_status dg_parcsr_comm(const dg_parcsr* pc, int64_t* send_counts, int64_t* recv_counts, uint32_t* send_idx,
                         uint32_t* ghosts);
/* send[k] = x_own[send_idx[k]] (device pointers, asynchronous on `stream`). */
dg_status dg_parcsr_pack(dg_parcsr* pc, const double* x_own, double* send, void* stream);
/* y = M x (add = 0) or y += M x (add = 1) over the owned rows, x given as the
 * owned input values and the received ghost values (device pointers). */
dg_status dg_parcsr_apply(dg_parcsr* pc, const double* x_own, const double* x_ghost, double* y, int add,
                          void* stream);
/* The same two in FP32 (vectors and an FP32 copy of M's entries; the
 * transfers' weights are dyadic, so the copy is exact). */
dg_status dg_parcsr_pack_f32(dg_parcsr* pc, const float* x_own, float* send, void* stream);
dg_status dg_parcsr_apply_f32(dg_parcsr* pc, const float* x_own, const float* x_ghost, float* y, int add,
                              void* stream);
void dg_parcsr_destroy(dg_parcsr* pc);

/* ------------------------------------------------------- learned smoother --- */
/* No reference counterpart (the reference smooths with damped Jacobi,
 * bin/options:187-194).  A per-node MLP 6 -> 64 -> 64 -> 1 (GELU), BF16
 * weights in the forward pass, FP32 accumulation, FP32 master parameters
 * packed as W1[64][6] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3.
 * Features of node i for a residual r (s = RMS of r): r_i/s, log2 d_i minus
 * its mean (d = operator diagonal), level, share of hanging references,
 * mean and max |r| over the surrounding elements / s.  It replaces the
 * post-smoothing of the finest level, x_i += y_i s / d_i, inside the FP32
 * inner V-cycle; the FP64 outer residual judges it and damped Jacobi takes
 * over for the rest of a solve when that residual falls by less than
 * fallback_ratio in one iteration. */
int dg_mlp_param_count(void);
dg_status dg_mlp_create(const float* params_host /* NULL: zeros */, dg_mlp** out);
dg_status dg_mlp_get_params(const dg_mlp* m, float* host);
dg_status dg_mlp_set_params(dg_mlp* m, const float* host);
/* out[i] = MLP(F[i][0..5]) for device F, out; exact_fp32 = 1 skips BF16 rounding. */
dg_status dg_mlp_forward(dg_mlp* m, const float* F, int64_t n, float* out, int exact_fp32, void* stream);
/* Gradient of mean (MLP(F_i) - T_i)^2 over n device rows (host grad, loss). */
dg_status dg_mlp_gradient(dg_mlp* m, const float* F, const float* T, int64_t n, int exact_fp32, float* grad_host,
                          double* loss_host);
/* One Adam step (beta 0.9/0.999) on that loss. */
dg_status dg_mlp_train_step(dg_mlp* m, const float* F, const float* T, int64_t n, float lr, double* loss_host);
void dg_mlp_destroy(dg_mlp* m);
/* Use the MLP (or NULL for damped Jacobi) as finest-level post-smoother. */
dg_status dg_damg_set_smoother(dg_damg* m, dg_mlp* mlp, int sweeps, double fallback_ratio);
/* Features of a finest-level residual r (device) into F [N][6] (device); *scale = s. */
dg_status dg_damg_features(dg_damg* m, const double* r, float* F, float* scale);

/* -------------------------------------------------------- vector kernels --- */

/* VecDot / VecNorm^2 as PETSc's KSPCG calls them (KSPSolve, src/omg/omg.C:1166,
 * with bin/options:50 -ksp_type cg): *result = sum_i x[i] y[i] in FP64 with a
 * fixed-order (deterministic) two-stage reduction.  x, y and result are device
 * pointers; the call synchronises the stream before returning. */
dg_status dg_vec_dot(const double* x, const double* y, int64_t n, double* result, void* stream);

/* The same inner product without any device allocation, for callers that
 * cannot allocate: a convergence test or monitor run every iteration inside
 * a solver whose device memory belongs to another allocator (a caching pool
 * that already holds the free HBM, or a process under an MPS memory cap), or
 * a loop that cannot take the device-wide synchronisation of cudaMalloc /
 * cudaFree.  It has no counterpart in the reference.  Limit: n <= 268435456.
 * The partial sums live in a fixed 512 KiB array inside the library's device
 * memory, held by every GPU that loads the library until the process exits.
 * The first call on each device looks up that array's address (with the
 * device current), so make that first call before any stream capture.  The
 * result is written asynchronously on `stream` (no synchronisation).  All
 * calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race on it and must be serialised by the caller.  The
 * looked-up address belongs to the device's current context: after
 * cudaDeviceReset on a device, do not call this function on that device
 * again in the same process (the cached address would be stale). */
dg_status dg_vec_dot_noalloc(const double* x, const double* y, int64_t n, double* result, void* stream);

/* One damped Jacobi update, x[i] += omega dinv[i] (b[i] - ax[i]) (the
 * V-cycle's smoother step, Richardson with Jacobi, bin/options:187-194), for
 * callers that apply the operator themselves (the partitioned hierarchy);
 * device pointers, asynchronous on `stream`. */
dg_status dg_vec_jacobi_update(double* x, const double* b, const double* ax, const double* dinv, double omega,
                               int64_t n, void* stream);
/* The same update in FP32. */
dg_status dg_vec_jacobi_update_f32(float* x, const float* b, const float* ax, const float* dinv, float omega,
                                   int64_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DENDRO_B200_H */
