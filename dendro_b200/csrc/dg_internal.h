// Internal device-side objects behind the opaque C-ABI handles.
#pragma once

#include <memory>
#include <vector>

#include "dg_common.cuh"

namespace dg {
// Tiles of `te` consecutive elements for the shared-memory operator kernels.
// Per tile: its distinct node ids (ascending; bit 31 set when another tile
// also references the node) and, grouped by node, the tile's references to
// them, each as position v * te + element of its (element, vertex) slot.
struct TileSet {
  int te = 0;                // elements per tile
  int64_t ntiles = 0;
  uint32_t max_nodes = 0;    // largest node count of a tile
  DBuf<uint32_t> ptr;        // [ntiles + 1] offsets of the tiles' node lists
  DBuf<uint32_t> nodes;      // [ptr[ntiles]]
  DBuf<uint16_t> nend;       // [ntiles * 8 te]: tile t, node k -> end of its run in inc
  DBuf<uint16_t> inc;        // [ntiles * 8 te]: tile t -> references ordered by node
  DBuf<uint4> eloc;          // [E] per element the node positions of its 8 vertices (multi-RHS set only)
  // warp tiles (at most 256 nodes per tile), all in the child-number frame
  // (frame vertex j = vertex j ^ c of the element):
  DBuf<uint8_t> eloc8;       // [8 E] per element byte j = node rank of frame vertex j
  DBuf<uint32_t> wmeta;      // [E] level | frame hanging mask << 8
  DBuf<uint8_t> ref8;        // [ntiles * kWarpRefBytes] per tile: the references sorted by node as frame
                             // positions j * te + element [8 te], their node ranks [8 te], then per lane
                             // one flag word [32 x u32] (bit q valid, 8 + q start, 16 + q leave, 24 + q store)
  DBuf<uint32_t> shared;     // ascending ids of the nodes several tiles reference
  int64_t nshared = 0;
};
// Elements grouped by parent octant for the octet operator kernel (octet.cuh):
// one entry per parent with at least one leaf child, in Morton order of the
// parents.  Arrays are lattice-point / child major so that consecutive
// octets are consecutive words.
struct OctetSet {
  int64_t n = 0;
  DBuf<uint32_t> meta;  // [n] level of the children (embedded) | child mask << 8
  DBuf<uint32_t> id;    // [27][n] node id of each lattice point, kNoNode when it hangs or no present child has it
  DBuf<uint32_t> elem;  // [8][n] element id of each present child (kNoNode when absent)
  // chunks of kOctChunk consecutive octets, staged through shared memory by
  // the chunked kernel: per chunk the ascending ids of the nodes its octets
  // touch (bit 31: another chunk touches the node too) and the range of
  // element ids of its children; per octet the chunk-local index of each
  // lattice node (0xffff: none) and of each present child's element.
  int64_t nchunk = 0;
  uint32_t max_nodes = 0, max_erange = 0;
  DBuf<uint32_t> cptr;    // [nchunk + 1]
  DBuf<uint32_t> cnodes;  // [cptr[nchunk]]
  DBuf<uint32_t> cel;     // [2 nchunk]: first element id, element range length
  DBuf<uint16_t> lidx;    // [27][n]
  DBuf<uint16_t> lelem;   // [8][n]
  DBuf<uint16_t> lnl;     // [8][E]: per element, the chunk-local index of each vertex's node (the DA's nl)
  // [n + 1][kOctRec] per octet (and a padding octet without children): the
  // 27 lattice node ids, the mask of lattice points without a node, the meta
  // word, 3 words of padding -- one 128-byte record read by the lane-per-child
  // operator and the tensor-memory multi-RHS kernel
  DBuf<uint32_t> rec;
};
// Compressed element-to-node map (cmap.cuh), built on request.
struct CompressedMap {
  int64_t ntiles = 0;    // tiles of 32 consecutive elements
  int qbits = 0;         // narrow quotient width (bits), 0 when not built
  int64_t wide_tiles = 0;
  DBuf<uint2> rem;       // [E] remainder bytes, vertex order
  DBuf<uint8_t> qmask;   // [E] vertices with a quotient
  DBuf<uint32_t> base;   // [ntiles] smallest node id of the tile
  DBuf<uint32_t> qoff;   // [ntiles] first quotient word | kCmapWide
  DBuf<uint16_t> quot;   // quotient words
  int64_t bytes() const { return 8 * rem.n + qmask.n + 4 * base.n + 4 * qoff.n + 2 * quot.n; }
};
constexpr int kOctChunk = 128;  // octets per chunk (one per thread of the chunked kernel)
constexpr int kOctRec = 32;     // words per octet record
}  // namespace dg

struct dg_octree {
  uint32_t max_depth = 0;
  int64_t n = 0;
  dg::DBuf<uint64_t> keys;  // octant keys (Morton anchor << 5 | level), sorted
};

struct dg_da {
  uint32_t D = 0;        // embedded depth = maxDepth + 1
  int64_t E = 0, N = 0, P = 0;
  dg::DBuf<uint32_t> nl;     // [8][E] node ids, vertex-major
  dg::DBuf<uint32_t> meta;   // [E] packed level / child number / hanging mask / type
  dg::DBuf<uint64_t> ekey;   // [E] element octant keys (embedded space)
  dg::DBuf<uint64_t> nkey;   // [N] node anchor Morton keys (embedded space), sorted
  // element tiles of the shared-memory operator kernels: the scalar warp-tile
  // operator's (kWarpTile elements per tile, built with the mesh) and the
  // multi-right-hand-side one's (kMultiTile elements per tile, built on first use)
  dg::TileSet tiles_w, tiles_mr;
  dg::OctetSet octs;  // elements grouped by parent (octet operator kernel)
  dg::CompressedMap cmap;  // compressed element map (on request)
  // operator launch shape picked by the autotuner on first use (-1: not yet)
  int tuned_f64 = -1, tuned_f32 = -1;
};

struct dg_mlp {
  dg::DBuf<float> params, grad, m1, m2, loss;
  int step = 0;
};

namespace dg {
struct HostPipe;  // streams, events and chunk plan of the pipelined host entry point (matvec.cu)
}

struct dg_mat {
  dg_da* da = nullptr;
  int kind = 0;  // 0 lap+mass, 1 elasticity, 2 Dirichlet Laplacian, 3 Dirichlet Jacobian
  int dof = 1;
  bool has_coef = false;
  dg::DBuf<double> coef;       // [2][E] (a then b), FP64
  dg::DBuf<float> coef32;      // [2][E] FP32 copy for the inner solver
  double mu = 0, lam = 0;
  dg::DBuf<uint8_t> dirichlet; // [N]
  dg::DBuf<double> host_x, host_y;  // device staging of dg_mat_mult_host, kept between calls
  mutable dg::DBuf<float> tc_coef;  // [octets + 1][16] element scale factors of the tensor-memory multi-RHS kernel
  std::shared_ptr<dg::HostPipe> pipe;
};

namespace dg {

// elements per tile of the multi-right-hand-side kernel and of the scalar
// warp-tile kernel (one lane each)
constexpr int kMultiTile = 128;
constexpr int kWarpTile = 32;
constexpr int kWarpRefBytes = 16 * kWarpTile + 4 * 32;  // per warp tile in TileSet::ref8
// Slack after per-element arrays that the bulk-copy operator kernel reads in
// whole 32-element windows starting on 16-byte boundaries: the [2 E]
// coefficient arrays get kCoefPad extra elements, the warp tiles' node lists
// kNodePad extra entries; eloc8 and wmeta are allocated for whole tiles.
constexpr int64_t kCoefPad = 64;
constexpr int64_t kNodePad = 8;

// ---- learned smoother (mlp.cu): 6 -> 64 -> 64 -> 1, packed FP32 parameters ----
constexpr int kMlpIn = 6;
constexpr int kMlpHidden = 64;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpHidden;
constexpr int kMlpParams = kOffB3 + 1;
dg_status mlp_forward(const float* params, const float* F, int64_t n, float* out, bool exact, cudaStream_t s);
dg_status mlp_gradient(const float* params, const float* F, const float* T, int64_t n, float* grad, float* loss_acc,
                       bool exact, cudaStream_t s);
dg_status mlp_adam(float* p, const float* g, float* m1, float* m2, int step, float lr, cudaStream_t s);

// ---- primitives (prim.cu) ----

// Device-wide exclusive scan of n uint32 values into out (out may alias in);
// returns the total through *total (host) when not null.
dg_status scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, cudaStream_t s);
// Keys-only stable LSD radix sort of n uint64 keys on bits
// [start_bit, start_bit + bits).  Sorted keys end in `keys`; tmp holds n keys.
dg_status radix_sort_u64(uint64_t* keys, uint64_t* tmp, int64_t n, int bits, cudaStream_t s,
                         int start_bit = 0);
// Remove adjacent duplicates in place; returns the new length.
dg_status unique_u64(uint64_t* keys, int64_t n, int64_t* n_out, cudaStream_t s);

// ---- octree (octree.cu) ----
dg_status points_to_octree(const double* d_pts, int64_t n, uint32_t D, uint32_t m, dg_octree* out,
                           cudaStream_t s);
dg_status balance_octree(const dg_octree* in, dg_octree* out, cudaStream_t s);
dg_status coarsen_octree(const dg_octree* in, dg_octree* out, cudaStream_t s);

// ---- mesh (mesh.cu) ----
dg_status build_mesh(const dg_octree* tree, dg_da* da, cudaStream_t s);
// Bounded device waits of the operator kernels: the wait limit in clock64
// cycles (<= 0: the default) and the check that synchronises s and reports
// DG_ETIMEOUT (then clears it) when a wait has run out.
void set_wait_limit(long long cycles);
long long wait_limit();  // clock cycles a bounded device wait may take
dg_status device_wait_status(cudaStream_t s);
dg_status build_tiles(dg_da* da, cudaStream_t s);  // da->tiles_w (kWarpTile)
dg_status build_octets(dg_da* da, cudaStream_t s);  // da->octs (octet.cu)
// da->cmap with narrow quotients of qbits (1..16) bits (cmap.cu); nl_out
// [8][E] receives the map decoded from it
dg_status build_cmap(dg_da* da, int qbits, cudaStream_t s);
dg_status cmap_decode(const dg_da* da, uint32_t* nl_out, cudaStream_t s);
// b = the load vector of a force sampled at the element centres (matvec.cu)
dg_status load_vector(const dg_da* da, const double* force, double* b, cudaStream_t s);
dg_status build_tile_set(const dg_da* da, int te, TileSet& ts, cudaStream_t s);
// Hanging mask of element type t (0..17) for child number c
// (include/oda/cnumEtypes.h:19-229).
uint32_t etype_mask(int c, int t);

// ---- operators (matvec.cu) ----
// Coarse elements of a level whose operator, with the coarse operator taken
// from the next finer level's coefficients (Jacobian3, examples/src/backend/
// omgJac.C:2139-2233), is the sum over their 8 children with the children's
// own coefficients (type-1 tables) because those differ.
struct Type1Set {
  int64_t n = 0;
  DBuf<uint32_t> elem;  // [n] element ids
  DBuf<double> coef;    // [n][16]: a of children 0..7 (child-number order), then b
  DBuf<float> coef32;
};
// The J operator of a level: coef (a then b, [2][E]) with the elements of t1
// zeroed, plus t1's children sums; coef == nullptr / t1 == nullptr: the
// operator's own coefficients / no type-1 elements.
dg_status lapmass_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s);
dg_status lapmass_apply_add_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s);
dg_status lapmass_apply_add_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s);
// y = A x for host x and y (staged in A->host_x / host_y) with the copies
// pipelined against the operator; DG_ENOTIMPL when the mesh does not qualify
dg_status lapmass_apply_host_pipelined_f64(dg_mat* A, const double* hx, double* hy);
dg_status lapmass_apply_j_f64(const dg_mat* A, const double* coef, const Type1Set* t1, const double* x, double* y,
                              cudaStream_t s);
dg_status lapmass_apply_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s);
dg_status lapmass_diag(const dg_mat* A, double* d, cudaStream_t s);
// One damped-Jacobi sweep x <- x + omega dinv (b - A x) in place, and the
// residual r = b - A x: the warp-tile operator into acc (an N-vector that must
// be zero on entry and is zero again on return), then one elementwise pass.
dg_status lapmass_smooth_f64(const dg_mat* A, double* x, const double* b, const double* dinv, double omega,
                             double* acc, cudaStream_t s, const double* coef = nullptr,
                             const Type1Set* t1 = nullptr);
dg_status lapmass_smooth_f32(const dg_mat* A, float* x, const float* b, const float* dinv, float omega, float* acc,
                             cudaStream_t s, const float* coef = nullptr,
                             const Type1Set* t1 = nullptr);
dg_status lapmass_residual_f64(const dg_mat* A, const double* x, const double* b, double* r, double* acc,
                               cudaStream_t s, const double* coef = nullptr,
                               const Type1Set* t1 = nullptr);
dg_status lapmass_residual_f32(const dg_mat* A, const float* x, const float* b, float* r, float* acc,
                               cudaStream_t s, const float* coef = nullptr,
                               const Type1Set* t1 = nullptr);
const char* matvec_variant_name(int v);
int matvec_variant_count();
// Y = A X for nrhs vectors (node-major [N][nrhs], FP32) on the tensor cores;
// split 1: TF32 products, 3: high/low TF32 split (FP32-level accuracy).
dg_status mrhs_apply(const dg_mat* A, const float* X, float* Y, int nrhs, int split, cudaStream_t s);
// Y = A X in the octet form (CUDA cores) in FP32 or FP64, node-major [N][R],
// R a multiple of 32; coef = the operator's coefficients in that precision
// ([2][E], a then b; ignored when the operator has none).
template <class T>
dg_status mrhs_octet_apply(const dg_mat* A, const T* coef, const T* X, T* Y, int R, cudaStream_t s);
// Multi-RHS operator on tcgen05 (mrhs_tc.cu): nrhs a multiple of 64, passes 1
// (TF32 products) or 3 (hi/lo split, FP32-level).
dg_status mrhs_tc_apply(const dg_mat* A, const float* X, float* Y, int R, int passes, cudaStream_t s);
// DG_ETIMEOUT (then cleared) when a bounded wait of that kernel ran out.
dg_status mrhs_tc_take_status();
dg_status elasticity_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s);
dg_status elasticity_diag(const dg_mat* A, double* d, cudaStream_t s);
// Dense row-major (3 N) x (3 N) matrix of the elasticity operator, Dirichlet
// rows the identity (the coarsest level of the dof-3 multigrid).
dg_status elasticity_assemble_dense(const dg_mat* A, double* dense, cudaStream_t s);
// Dirichlet Laplacian (kind 2) / Jacobian (kind 3) on A->dirichlet node flags.
dg_status dirichlet_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s);
dg_status dirichlet_diag(const dg_mat* A, double* d, cudaStream_t s);
// Dense assembled operator of a small level as row-major blocks, one per
// independent mesh: node r belongs to block row_blk[r] with node offset
// boff[b], size bn[b] and storage offset baoff[b].
dg_status lapmass_assemble_dense(const dg_mat* A, double* dense, int64_t dense_size, const uint32_t* row_blk,
                                 const int64_t* boff, const int64_t* bn, const int64_t* baoff, cudaStream_t s,
                                 const double* coef = nullptr, const Type1Set* t1 = nullptr);

}  // namespace dg
