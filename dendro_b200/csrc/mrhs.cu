// Multi-right-hand-side operator Y = A X on the tensor cores: the scalar
// Laplacian + mass operator (JAC_TYPE2_ELEM_MULT_BLOCK,
// examples/src/backend/omgNeumann.C:468-488) applied to nrhs vectors at once,
// X and Y node-major [N][nrhs] in FP32.  The reference applies MatMult to one
// vector at a time; the batching has no reference counterpart.
//
// Per element the contraction D (16 rhs x 8 vertices) = X_e (16 x 8) A_e^T is
// one mma.sync.m16n8k8 with TF32 inputs and FP32 accumulation (or three, with
// each input split into a TF32 high part and a TF32 remainder, which keeps
// FP32-level accuracy).  A_e = f1 L[c][t] + f2 M[c][t], where L and M are the
// per (child number, element type) tables T^T K T and T^T M T
// (Stencils/LapType2Stencils.inp, MassType2Stencils.inp; here computed from T
// and the reference-cube matrices), stored per MMA lane so that each lane
// loads its B-fragment entries with one 16-byte load.
//
// A CTA owns a tile of kMultiTile elements (its distinct nodes and, per
// element, the positions of its vertices' nodes in that list) and walks the
// right-hand sides in chunks of 16: the chunk's rows of x at the tile's nodes
// are staged in shared memory with coalesced float4 loads, each warp reads its
// elements' MMA fragments from those rows and adds the results into shared
// rows of y with shared-memory atomics, and each node's row leaves with float4
// stores (node used by this tile only) or float4 global atomics (node shared
// with other tiles).
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dg_internal.h"
#include "octet.cuh"

namespace dg {

namespace {

constexpr int kMT = kMultiTile;     // elements per tile, one thread each
constexpr int kRC = 16;             // right-hand sides per chunk (the MMA's M)

__device__ __forceinline__ float elem_hf(uint32_t lev) { return __int_as_float(int(127 + 1 - int(lev)) << 23); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// d += A (16 x 8, row) * B (8 x 8, col), TF32 inputs, FP32 accumulation.
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

constexpr int kMThreads = 256;  // 8 warps per tile
constexpr int kRW = kRC + 4;     // shared row of one node: 16 floats + pad, float4-aligned

// NS = 1: TF32 products.  NS = 3: x = hi + lo for both inputs and
// D = A_lo B_hi + A_hi B_lo + A_hi B_hi.
template <int NS>
__global__ void __launch_bounds__(kMThreads) mrhs_kernel(const uint32_t* __restrict__ meta,
                                                         const float* __restrict__ ca, const float* __restrict__ cb,
                                                         int64_t E, const uint32_t* __restrict__ tile_ptr,
                                                         const uint32_t* __restrict__ tile_nodes,
                                                         const uint4* __restrict__ eloc,
                                                         const float4* __restrict__ tbl, int R, uint32_t cap,
                                                         const float* __restrict__ X, float* __restrict__ Y) {
  extern __shared__ __align__(16) float mr_smem[];
  float* Xs = mr_smem;           // [cap][kRW] x rows of the chunk
  float* Ys = Xs + cap * kRW;    // [cap][kRW] y rows of the chunk
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int64_t tile = blockIdx.x;
  const uint32_t p0 = __ldg(tile_ptr + tile), nt = __ldg(tile_ptr + tile + 1) - p0;
  for (int r0 = 0; r0 < R; r0 += kRC) {
    for (uint32_t i = tid; i < 4 * nt; i += kMThreads) {
      const uint32_t k = i >> 2, q = i & 3;
      const uint32_t n = __ldg(tile_nodes + p0 + k) & 0x7fffffffu;
      reinterpret_cast<float4*>(Xs + k * kRW)[q] =
          __ldg(reinterpret_cast<const float4*>(X + int64_t(n) * R + r0) + q);
      reinterpret_cast<float4*>(Ys + k * kRW)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    for (int el = warp; el < kMT; el += kMThreads / 32) {
      const int64_t e = tile * kMT + el;
      if (e >= E) break;
      const uint32_t m = __ldg(meta + e);
      const uint4 L = __ldg(eloc + e);
      const float h = elem_hf(meta_lev(m));
      const float a = ca ? __ldg(ca + e) : 1.f, b = cb ? __ldg(cb + e) : 1.f;
      const float f1 = a * h * 0.5f, f2 = b * h * h * h * 0.125f;
      const float4 t = __ldg(tbl + (meta_cnum(m) * 18 + meta_type(m)) * 32 + lane);
      const float bf0 = f1 * t.x + f2 * t.z, bf1 = f1 * t.y + f2 * t.w;
      // node positions of vertices tq, tq + 4 (A columns) and 2 tq, 2 tq + 1 (D columns)
      const uint32_t lo = tq < 2 ? L.x : L.y, hi = tq < 2 ? L.z : L.w;
      const uint32_t sh = (tq & 1) * 16;
      const uint32_t s_a = (lo >> sh) & 0xffffu, s_b = (hi >> sh) & 0xffffu;
      const uint32_t dw = tq == 0 ? L.x : tq == 1 ? L.y : tq == 2 ? L.z : L.w;
      const uint32_t s_c = dw & 0xffffu, s_d = dw >> 16;
      const float* xa = Xs + s_a * kRW;
      const float* xb = Xs + s_b * kRW;
      const float x0 = xa[g], x1 = xa[g + 8], x2 = xb[g], x3 = xb[g + 8];
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      if (NS == 1) {
        mma_tf32(d, to_tf32(x0), to_tf32(x1), to_tf32(x2), to_tf32(x3), to_tf32(bf0), to_tf32(bf1));
      } else {
        const uint32_t ah0 = to_tf32(x0), ah1 = to_tf32(x1), ah2 = to_tf32(x2), ah3 = to_tf32(x3);
        const uint32_t bh0 = to_tf32(bf0), bh1 = to_tf32(bf1);
        const uint32_t al0 = to_tf32(x0 - __uint_as_float(ah0)), al1 = to_tf32(x1 - __uint_as_float(ah1));
        const uint32_t al2 = to_tf32(x2 - __uint_as_float(ah2)), al3 = to_tf32(x3 - __uint_as_float(ah3));
        const uint32_t bl0 = to_tf32(bf0 - __uint_as_float(bh0)), bl1 = to_tf32(bf1 - __uint_as_float(bh1));
        mma_tf32(d, al0, al1, al2, al3, bh0, bh1);
        mma_tf32(d, ah0, ah1, ah2, ah3, bl0, bl1);
        mma_tf32(d, ah0, ah1, ah2, ah3, bh0, bh1);
      }
      // D: rhs g / g + 8 at vertices 2 tq (node s_c) and 2 tq + 1 (node s_d)
      float* yc = Ys + s_c * kRW;
      float* yd = Ys + s_d * kRW;
      atomicAdd(yc + g, d[0]);
      atomicAdd(yd + g, d[1]);
      atomicAdd(yc + g + 8, d[2]);
      atomicAdd(yd + g + 8, d[3]);
    }
    __syncthreads();
    for (uint32_t i = tid; i < 4 * nt; i += kMThreads) {
      const uint32_t k = i >> 2, q = i & 3;
      const uint32_t id = __ldg(tile_nodes + p0 + k);
      const float4 v = reinterpret_cast<const float4*>(Ys + k * kRW)[q];
      float4* dst = reinterpret_cast<float4*>(Y + int64_t(id & 0x7fffffffu) * R + r0) + q;
      if (id & 0x80000000u) atomicAdd(dst, v);
      else *dst = v;
    }
    __syncthreads();
  }
}

// Warp-tile form: each warp owns tiles of kWarpTile elements (the scalar
// operator's tiles) and a private shared accumulator of the tile's node rows
// for one 16-RHS chunk, so the elements of a tile add their D fragments with
// plain read-modify-writes, one element after the other (no atomics, no
// other warp touching the rows).  A fragments come straight from the
// node-major X rows (8 lanes read 32 contiguous bytes of a row; rows shared by
// neighbouring elements hit L1).  Each lane keeps its own element's scaling,
// table index and node ranks; the warp walks the tile's elements taking them
// by shuffle.  Rows leave with float4 stores (node whole in this tile) or
// float4 global atomics.
constexpr int kMWarps = 4;       // warps per CTA
constexpr int kYW = kRC + 4;     // accumulator row: 16 floats + pad, float4-aligned
// Floats of shared memory per warp: the rows, then the node ids padded to a
// multiple of 4, so that every warp's rows start on a 16-byte boundary.
// STAGE adds a second block of rows for the chunk's x values.
__host__ __device__ constexpr size_t mrhs_warp_stride(uint32_t cap, bool stage) {
  return size_t(cap) * kYW * (stage ? 2 : 1) + ((size_t(cap) + 3) & ~size_t(3));
}
__device__ __forceinline__ uint32_t rank_of(uint2 r, uint32_t v) { return __byte_perm(v < 4 ? r.x : r.y, 0u, 0x4440u | (v & 3u)); }

// STAGE: the chunk's x rows of the tile are first copied into shared memory
// with every lane's float4 loads in flight together, so the element walk
// reads shared memory only; otherwise each element loads its A fragment from X.
template <int NS, bool STAGE>
__global__ void __launch_bounds__(32 * kMWarps) mrhs_warp_kernel(
    const uint32_t* __restrict__ meta, const float* __restrict__ ca, const float* __restrict__ cb, int64_t E,
    int64_t ntiles, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_nodes,
    const uint2* __restrict__ eloc8, const float4* __restrict__ tbl, int R, uint32_t cap,
    const float* __restrict__ X, float* __restrict__ Y) {
  extern __shared__ __align__(16) float mw_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, tq = lane & 3;
  // [cap][kYW] y rows, ([cap][kYW] x rows,) then the node ids
  float* Ys = mw_smem + size_t(w) * mrhs_warp_stride(cap, STAGE);
  float* Xs = Ys + size_t(cap) * kYW;
  uint32_t* sn = reinterpret_cast<uint32_t*>(Ys + size_t(cap) * kYW * (STAGE ? 2 : 1));
  const int64_t nw = int64_t(gridDim.x) * kMWarps;
  for (int64_t t = blockIdx.x * int64_t(kMWarps) + w; t < ntiles; t += nw) {
    const uint32_t p0 = __ldg(tile_ptr + t), nt = __ldg(tile_ptr + t + 1) - p0;
    for (uint32_t k = lane; k < nt; k += 32) sn[k] = __ldg(tile_nodes + p0 + k);
    // this lane's element: scaling, table row and node ranks
    const int64_t e_own = t * kWarpTile + lane;
    const int nel = int(E - t * kWarpTile < kWarpTile ? E - t * kWarpTile : kWarpTile);
    float f1o = 0.f, f2o = 0.f;
    uint32_t combo_o = 0;
    uint2 Lo = make_uint2(0, 0);
    if (e_own < E) {
      const uint32_t m = __ldg(meta + e_own);
      const float h = elem_hf(meta_lev(m));
      const float a = ca ? __ldg(ca + e_own) : 1.f, b = cb ? __ldg(cb + e_own) : 1.f;
      f1o = a * h * 0.5f;
      f2o = b * h * h * h * 0.125f;
      combo_o = ((meta_cnum(m) * 18 + meta_type(m)) * 32) | (meta_cnum(m) << 16);
      Lo = __ldg(eloc8 + e_own);
    }
    __syncwarp();
    for (int r0 = 0; r0 < R; r0 += kRC) {
      for (uint32_t i = lane; i < 4 * nt; i += 32) {
        reinterpret_cast<float4*>(Ys + (i >> 2) * kYW)[i & 3] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (STAGE)
          reinterpret_cast<float4*>(Xs + (i >> 2) * kYW)[i & 3] =
              __ldg(reinterpret_cast<const float4*>(X + int64_t(sn[i >> 2] & 0x7fffffffu) * R + r0) + (i & 3));
      }
      __syncwarp();
      for (int el = 0; el < nel; ++el) {
        const float f1 = __shfl_sync(0xffffffffu, f1o, el), f2 = __shfl_sync(0xffffffffu, f2o, el);
        const uint32_t cw = __shfl_sync(0xffffffffu, combo_o, el);
        const uint32_t combo = cw & 0xffffu, c = cw >> 16;  // table row; child number (ranks are in its frame)
        uint2 L;
        L.x = __shfl_sync(0xffffffffu, Lo.x, el);
        L.y = __shfl_sync(0xffffffffu, Lo.y, el);
        const float4 tb = __ldg(tbl + combo + lane);
        const float bf0 = f1 * tb.x + f2 * tb.z, bf1 = f1 * tb.y + f2 * tb.w;
        float x0, x1, x2, x3;
        if (STAGE) {
          const float* xa = Xs + rank_of(L, tq ^ c) * kYW;
          const float* xb = Xs + rank_of(L, (tq + 4) ^ c) * kYW;
          x0 = xa[g], x1 = xa[g + 8], x2 = xb[g], x3 = xb[g + 8];
        } else {
          const float* xa = X + int64_t(sn[rank_of(L, tq ^ c)] & 0x7fffffffu) * R + r0;
          const float* xb = X + int64_t(sn[rank_of(L, (tq + 4) ^ c)] & 0x7fffffffu) * R + r0;
          x0 = __ldg(xa + g), x1 = __ldg(xa + g + 8), x2 = __ldg(xb + g), x3 = __ldg(xb + g + 8);
        }
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        if (NS == 1) {
          mma_tf32(d, to_tf32(x0), to_tf32(x1), to_tf32(x2), to_tf32(x3), to_tf32(bf0), to_tf32(bf1));
        } else {
          const uint32_t ah0 = to_tf32(x0), ah1 = to_tf32(x1), ah2 = to_tf32(x2), ah3 = to_tf32(x3);
          const uint32_t bh0 = to_tf32(bf0), bh1 = to_tf32(bf1);
          const uint32_t al0 = to_tf32(x0 - __uint_as_float(ah0)), al1 = to_tf32(x1 - __uint_as_float(ah1));
          const uint32_t al2 = to_tf32(x2 - __uint_as_float(ah2)), al3 = to_tf32(x3 - __uint_as_float(ah3));
          const uint32_t bl0 = to_tf32(bf0 - __uint_as_float(bh0)), bl1 = to_tf32(bf1 - __uint_as_float(bh1));
          mma_tf32(d, al0, al1, al2, al3, bh0, bh1);
          mma_tf32(d, ah0, ah1, ah2, ah3, bl0, bl1);
          mma_tf32(d, ah0, ah1, ah2, ah3, bh0, bh1);
        }
        // D: rhs g / g + 8 at vertices 2 tq and 2 tq + 1 (distinct nodes of one element)
        float* yc = Ys + rank_of(L, (2 * tq) ^ c) * kYW;
        float* yd = Ys + rank_of(L, (2 * tq + 1) ^ c) * kYW;
        yc[g] += d[0];
        yd[g] += d[1];
        yc[g + 8] += d[2];
        yd[g + 8] += d[3];
        __syncwarp();  // the next element may add into the same rows
      }
      for (uint32_t i = lane; i < 4 * nt; i += 32) {
        const uint32_t k = i >> 2, q = i & 3;
        const uint32_t id = sn[k];
        const float4 v = reinterpret_cast<const float4*>(Ys + k * kYW)[q];
        float4* dst = reinterpret_cast<float4*>(Y + int64_t(id & 0x7fffffffu) * R + r0) + q;
        if (id & 0x80000000u) atomicAdd(dst, v);
        else *dst = v;
      }
      __syncwarp();
    }
  }
}

// Block form: per element the whole block of W right-hand sides of a pass
// (W = 32 or 64, W / 16 MMAs sharing one B fragment), all in the
// child-number frame: an element's node ranks come frame-ordered from the
// warp tiles and its stencil fragment from the 18-entry frame table (9 KB,
// read through L1).  The rows of the MMA map to right-hand sides
// so that a lane's A values at a vertex are the F = W / 8 consecutive floats
// F g .. F g + F - 1 of the node's row (chunk c, row g: rhs F g + 2c; row g + 8:
// F g + 2c + 1): 16-byte loads straight from X; its D values at a vertex land
// on the same F consecutive floats of the accumulator row as 16-byte
// read-modify-writes.  The next PD elements' X values travel in a ring of
// registers, walked PD elements at a time so that every slot is a
// compile-time register.
constexpr int kBWarps = 4;
__host__ __device__ constexpr size_t mrhs_block_stride(uint32_t cap, int W) {
  return size_t(cap) * (W + 4) + ((size_t(cap) + 3) & ~size_t(3));
}

template <int NS, int W, int PD>
__global__ void __launch_bounds__(32 * kBWarps) mrhs_block_kernel(
    const uint32_t* __restrict__ wmeta, const float* __restrict__ ca, const float* __restrict__ cb, int64_t E,
    int64_t ntiles, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_nodes,
    const uint2* __restrict__ eloc8, const float4* __restrict__ ftbl, int R, uint32_t cap,
    const float* __restrict__ X, float* __restrict__ Y) {
  constexpr int F = W / 8, NV = F / 4, NC = W / 16, RW = W + 4;
  extern __shared__ __align__(16) float mb_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, tq = lane & 3;
  float* Ys = mb_smem + size_t(w) * mrhs_block_stride(cap, W);  // [cap][RW] rows, then the node ids
  uint32_t* sn = reinterpret_cast<uint32_t*>(Ys + size_t(cap) * RW);
  const int64_t nw = int64_t(gridDim.x) * kBWarps;
  for (int64_t t = blockIdx.x * int64_t(kBWarps) + w; t < ntiles; t += nw) {
    const uint32_t p0 = __ldg(tile_ptr + t), nt = __ldg(tile_ptr + t + 1) - p0;
    for (uint32_t k = lane; k < nt; k += 32) sn[k] = __ldg(tile_nodes + p0 + k);
    const int64_t e_own = t * kWarpTile + lane;
    const int nel = int(E - t * kWarpTile < kWarpTile ? E - t * kWarpTile : kWarpTile);
    float f1o = 0.f, f2o = 0.f;
    uint32_t ft_o = 0;
    uint2 Lo = make_uint2(0, 0);
    if (e_own < E) {
      const uint32_t m = __ldg(wmeta + e_own);
      const float h = elem_hf(meta_lev(m));
      const float a = ca ? __ldg(ca + e_own) : 1.f, b = cb ? __ldg(cb + e_own) : 1.f;
      f1o = a * h * 0.5f;
      f2o = b * h * h * h * 0.125f;
      ft_o = wmeta_ftype(m) * 32;
      Lo = __ldg(eloc8 + e_own);  // byte j: rank of frame vertex j
    }
    __syncwarp();
    for (int r0 = 0; r0 < R; r0 += W) {
      for (uint32_t i = lane; i < (W / 4) * nt; i += 32)
        reinterpret_cast<float4*>(Ys + (i / (W / 4)) * RW)[i % (W / 4)] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncwarp();
      float4 ra[PD][NV], rb[PD][NV];
      uint2 rL[PD];
      uint32_t rf[PD];
      auto fetch = [&](int slot, int el) {  // el < 32; beyond the tile's elements nothing is loaded
        uint2 Ln;
        Ln.x = __shfl_sync(0xffffffffu, Lo.x, el);
        Ln.y = __shfl_sync(0xffffffffu, Lo.y, el);
        rf[slot] = __shfl_sync(0xffffffffu, ft_o, el);
        rL[slot] = Ln;
        if (el < nel) {
          const float4* a4 =
              reinterpret_cast<const float4*>(X + int64_t(sn[byte_of(Ln, tq)] & 0x7fffffffu) * R + r0 + F * g);
          const float4* b4 =
              reinterpret_cast<const float4*>(X + int64_t(sn[byte_of(Ln, tq + 4)] & 0x7fffffffu) * R + r0 + F * g);
#pragma unroll
          for (int k = 0; k < NV; ++k) {
            ra[slot][k] = __ldg(a4 + k);
            rb[slot][k] = __ldg(b4 + k);
          }
        }
      };
#pragma unroll
      for (int q = 0; q < PD; ++q) fetch(q, q);
      for (int el0 = 0; el0 < nel; el0 += PD) {
#pragma unroll
        for (int q = 0; q < PD; ++q) {
          const int el = el0 + q;
          if (el >= nel) break;
          float4 xa[NV], xb[NV];
#pragma unroll
          for (int k = 0; k < NV; ++k) {
            xa[k] = ra[q][k];
            xb[k] = rb[q][k];
          }
          const uint2 L = rL[q];
          const float4 tb = __ldg(ftbl + rf[q] + lane);
          const float f1 = __shfl_sync(0xffffffffu, f1o, el), f2 = __shfl_sync(0xffffffffu, f2o, el);
          fetch(q, el + PD < 32 ? el + PD : 31);  // this slot now carries element el + PD
          const float bf0 = f1 * tb.x + f2 * tb.z, bf1 = f1 * tb.y + f2 * tb.w;
          const uint32_t bh0 = to_tf32(bf0), bh1 = to_tf32(bf1);
          const uint32_t bl0 = to_tf32(bf0 - __uint_as_float(bh0)), bl1 = to_tf32(bf1 - __uint_as_float(bh1));
          float d[NC][4];
#pragma unroll
          for (int cc = 0; cc < NC; ++cc) {
            const float4& qa = xa[cc / 2];
            const float4& qb = xb[cc / 2];
            const float x0 = (cc & 1) ? qa.z : qa.x, x1 = (cc & 1) ? qa.w : qa.y;
            const float x2 = (cc & 1) ? qb.z : qb.x, x3 = (cc & 1) ? qb.w : qb.y;
            d[cc][0] = d[cc][1] = d[cc][2] = d[cc][3] = 0.f;
            const uint32_t ah0 = to_tf32(x0), ah1 = to_tf32(x1), ah2 = to_tf32(x2), ah3 = to_tf32(x3);
            if (NS == 1) {
              mma_tf32(d[cc], ah0, ah1, ah2, ah3, bh0, bh1);
            } else {
              const uint32_t al0 = to_tf32(x0 - __uint_as_float(ah0)), al1 = to_tf32(x1 - __uint_as_float(ah1));
              const uint32_t al2 = to_tf32(x2 - __uint_as_float(ah2)), al3 = to_tf32(x3 - __uint_as_float(ah3));
              float e[4] = {0.f, 0.f, 0.f, 0.f};  // the two correction products, a chain of their own
              mma_tf32(e, al0, al1, al2, al3, bh0, bh1);
              mma_tf32(d[cc], ah0, ah1, ah2, ah3, bh0, bh1);
              mma_tf32(e, ah0, ah1, ah2, ah3, bl0, bl1);
#pragma unroll
              for (int r = 0; r < 4; ++r) d[cc][r] += e[r];
            }
          }
          // D: rows g / g + 8 of chunk cc are right-hand sides F g + 2 cc / F g + 2 cc + 1,
          // at frame vertices 2 tq and 2 tq + 1
          float4* yc = reinterpret_cast<float4*>(Ys + byte_of(L, 2 * tq) * RW + F * g);
          float4* yd = reinterpret_cast<float4*>(Ys + byte_of(L, 2 * tq + 1) * RW + F * g);
#pragma unroll
          for (int k = 0; k < NV; ++k) {
            float4 u = yc[k], v = yd[k];
            u.x += d[2 * k][0];
            u.y += d[2 * k][2];
            u.z += d[2 * k + 1][0];
            u.w += d[2 * k + 1][2];
            v.x += d[2 * k][1];
            v.y += d[2 * k][3];
            v.z += d[2 * k + 1][1];
            v.w += d[2 * k + 1][3];
            yc[k] = u;
            yd[k] = v;
          }
          __syncwarp();  // the next element may add into the same rows
        }
      }
      for (uint32_t i = lane; i < (W / 4) * nt; i += 32) {
        const uint32_t k = i / (W / 4), q = i % (W / 4);
        const uint32_t id = sn[k];
        const float4 v = reinterpret_cast<const float4*>(Ys + k * RW)[q];
        float4* dst = reinterpret_cast<float4*>(Y + int64_t(id & 0x7fffffffu) * R + r0) + q;
        if (id & 0x80000000u) atomicAdd(dst, v);
        else *dst = v;
      }
      __syncwarp();
    }
  }
}

// Zero the rows of the nodes that several tiles share (their sums arrive by atomics).
__global__ void zero_shared_rows(const uint32_t* __restrict__ shared, int64_t ns, int R4, float4* __restrict__ Y) {
  const int64_t n = ns * R4;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    Y[int64_t(shared[i / R4]) * R4 + i % R4] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Element matrices T^T K T and T^T M T per (child number, element type), in
// the per-lane layout of the B fragment: lane (g = lane / 4, tq = lane % 4)
// holds {L[g][tq], L[g][tq + 4], M[g][tq], M[g][tq + 4]}.
std::vector<float> stencil_tables() {
  const double M1[2][2] = {{2.0 / 3.0, 1.0 / 3.0}, {1.0 / 3.0, 2.0 / 3.0}};
  const double K1[2][2] = {{0.5, -0.5}, {-0.5, 0.5}};
  double K[8][8], Mm[8][8];
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      const int ix = i & 1, iy = (i >> 1) & 1, iz = i >> 2, jx = j & 1, jy = (j >> 1) & 1, jz = j >> 2;
      Mm[i][j] = M1[ix][jx] * M1[iy][jy] * M1[iz][jz];
      K[i][j] = K1[ix][jx] * M1[iy][jy] * M1[iz][jz] + M1[ix][jx] * K1[iy][jy] * M1[iz][jz] +
                M1[ix][jx] * M1[iy][jy] * K1[iz][jz];
    }
  std::vector<float> out(size_t(8) * 18 * 32 * 4);
  for (int c = 0; c < 8; ++c)
    for (int t = 0; t < 18; ++t) {
      const uint32_t mask = etype_mask(c, t);
      double T[8][8] = {};
      for (int i = 0; i < 8; ++i) {
        if (!((mask >> i) & 1u)) {
          T[i][i] = 1.0;
          continue;
        }
        const uint32_t keep = ~(uint32_t(i) ^ uint32_t(c)) & 7u;
        const double w = __builtin_popcount(keep) == 2 ? 0.5 : 0.25;
        for (int j = 0; j < 8; ++j)
          if (((uint32_t(j ^ i)) & keep) == 0u) T[i][j] = w;
      }
      double L[8][8], MM[8][8];
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
          double sl = 0, sm = 0;
          for (int p = 0; p < 8; ++p)
            for (int q = 0; q < 8; ++q) {
              sl += T[p][i] * K[p][q] * T[q][j];
              sm += T[p][i] * Mm[p][q] * T[q][j];
            }
          L[i][j] = sl;
          MM[i][j] = sm;
        }
      for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, tq = lane & 3;
        float* o = out.data() + ((size_t(c) * 18 + t) * 32 + lane) * 4;
        o[0] = float(L[g][tq]);
        o[1] = float(L[g][tq + 4]);
        o[2] = float(MM[g][tq]);
        o[3] = float(MM[g][tq + 4]);
      }
    }
  return out;
}

// The 18 frame stencils (child number 0 frame, kFrameMasks order) in the
// same per-lane fragment layout: T for a frame mask has vertex 0's frame
// parent corner and hanging vertex i averages the nodes j with j a bit subset
// of i (2 on an edge, 4 on a face).
std::vector<float> frame_stencil_tables() {
  const double M1[2][2] = {{2.0 / 3.0, 1.0 / 3.0}, {1.0 / 3.0, 2.0 / 3.0}};
  const double K1[2][2] = {{0.5, -0.5}, {-0.5, 0.5}};
  double K[8][8], Mm[8][8];
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      const int ix = i & 1, iy = (i >> 1) & 1, iz = i >> 2, jx = j & 1, jy = (j >> 1) & 1, jz = j >> 2;
      Mm[i][j] = M1[ix][jx] * M1[iy][jy] * M1[iz][jz];
      K[i][j] = K1[ix][jx] * M1[iy][jy] * M1[iz][jz] + M1[ix][jx] * K1[iy][jy] * M1[iz][jz] +
                M1[ix][jx] * M1[iy][jy] * K1[iz][jz];
    }
  std::vector<float> out(size_t(18) * 32 * 4);
  for (int t = 0; t < 18; ++t) {
    const uint32_t mask = kFrameMasks[t];
    double T[8][8] = {};
    for (int i = 0; i < 8; ++i) {
      if (!((mask >> i) & 1u)) {
        T[i][i] = 1.0;
        continue;
      }
      const double w = __builtin_popcount(uint32_t(i)) == 1 ? 0.5 : 0.25;
      for (int j = 0; j < 8; ++j)
        if ((uint32_t(j) & ~uint32_t(i)) == 0u) T[i][j] = w;
    }
    for (int lane = 0; lane < 32; ++lane) {
      const int g = lane >> 2, tq = lane & 3;
      const int rows[2] = {tq, tq + 4};
      float* o = out.data() + (size_t(t) * 32 + lane) * 4;
      for (int h = 0; h < 2; ++h) {
        double sl = 0, sm = 0;
        for (int p = 0; p < 8; ++p)
          for (int q = 0; q < 8; ++q) {
            sl += T[p][g] * K[p][q] * T[q][rows[h]];
            sm += T[p][g] * Mm[p][q] * T[q][rows[h]];
          }
        o[h] = float(sl);
        o[2 + h] = float(sm);
      }
    }
  }
  return out;
}

// Octet form on the CUDA cores: a warp per (octet, 32 right-hand sides), one
// lane per right-hand side.  Each lane holds its column's 27 lattice values
// of the octet in registers and runs the octet arithmetic of the scalar
// kernel (octet_apply: hanging points, the children's Walsh-form element
// operators, T^T) in FP32; the octet's node ids, meta word and element ids
// are the same for the whole warp, and the X rows read and the Y rows added
// are 32 consecutive floats per node (one 128-byte access per node and
// warp).  Each warp copies those 36 words of the task one grid stride ahead
// into its own shared-memory slot (4-byte cp.async, one word per lane) while
// it works the current task, so the X row loads of a task issue without the
// round trip for its ids.  Y must be zero on entry (the sums leave with global
// reductions; the centre of a full octet with a store).  Exact FP32 products:
// no TF32 rounding, so `split` does not apply.
constexpr int kMoWords = 36;  // 27 node ids, meta, 8 element ids
template <class T>
__global__ void __launch_bounds__(128) mrhs_octet_pf_kernel(int64_t n, const uint32_t* __restrict__ ometa,
                                                            const uint32_t* __restrict__ oid,
                                                            const uint32_t* __restrict__ oelem,
                                                            const T* __restrict__ ca, const T* __restrict__ cb,
                                                            int R, const T* __restrict__ X, T* __restrict__ Y) {
  __shared__ uint32_t slot[4][2][kMoWords];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nb = R / 32;
  const int64_t tasks = n * nb;
  const int64_t wstride = (int64_t(gridDim.x) * blockDim.x) >> 5;
  auto fetch = [&](int64_t t, int sl) {
    if (t < tasks) {
      const int64_t o = t / nb;
      for (int k = lane; k < kMoWords; k += 32) {
        const uint32_t* src = k < 27 ? oid + int64_t(k) * n + o : k == 27 ? ometa + o : oelem + int64_t(k - 28) * n + o;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         static_cast<uint32_t>(__cvta_generic_to_shared(&slot[w][sl][k]))),
                     "l"(src)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  fetch(t, 0);
  for (int it = 0; t < tasks; t += wstride, ++it) {
    const int sl = it & 1;
    __syncwarp();  // every lane is done with the slot the next fetch overwrites
    fetch(t + wstride, sl ^ 1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncwarp();  // the whole slot of this task has landed
    const uint32_t* W = slot[w][sl];
    const int64_t o = t / nb;
    const int col = int(t - o * nb) * 32 + lane;
    const uint32_t m = W[27];
    uint32_t none = 0;
    T xv[27], yv[27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = W[p];
      none |= id == kNoNode ? (1u << p) : 0u;
      xv[p] = id != kNoNode ? __ldg(X + int64_t(id) * R + col) : T(0);
    }
    octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
      if (ca) {
        const uint32_t e = W[28 + c];
        f1 *= __ldg(ca + e);
        f2 *= __ldg(cb + e);
      }
    });
    const uint32_t cm = ometa_cmask(m);
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = W[p];
      if (id == kNoNode) continue;
      T* dst = Y + int64_t(id) * R + col;
      if (p == 13 && cm == 255u) *dst = yv[p];
      else if (yv[p] != T(0)) atomicAdd(dst, yv[p]);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Two FP32 values in one 64-bit register, worked by the packed FP32
// instructions of sm_100 (add / sub / mul .f32x2): the octet arithmetic runs
// on two right-hand sides per instruction.
struct F2 {
  uint64_t v;
  __device__ __forceinline__ F2() {}
  __device__ __forceinline__ F2(double s) {
    const uint64_t u = __float_as_uint(float(s));
    v = (u << 32) | u;
  }
  __device__ __forceinline__ F2& operator+=(F2 b) {
    asm("add.rn.f32x2 %0, %0, %1;" : "+l"(v) : "l"(b.v));
    return *this;
  }
  __device__ __forceinline__ F2& operator*=(F2 b) {
    asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(v) : "l"(b.v));
    return *this;
  }
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return a += b; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return a *= b; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ bool nonzero(F2 a) { return (a.v & 0x7fffffff7fffffffull) != 0ull; }

// The octet form with two right-hand sides per lane (64 per warp): X rows
// read as 8-byte pairs, Y rows added with 8-byte vector reductions, the
// element arithmetic on packed pairs.  nrhs a multiple of 64.
__global__ void __launch_bounds__(128) mrhs_octet_pair_kernel(int64_t n, const uint32_t* __restrict__ ometa,
                                                              const uint32_t* __restrict__ oid,
                                                              const uint32_t* __restrict__ oelem,
                                                              const float* __restrict__ ca,
                                                              const float* __restrict__ cb, int R,
                                                              const float* __restrict__ X, float* __restrict__ Y) {
  __shared__ uint32_t slot[4][2][kMoWords];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nb = R / 64;
  const int64_t tasks = n * nb;
  const int64_t wstride = (int64_t(gridDim.x) * blockDim.x) >> 5;
  auto fetch = [&](int64_t t, int sl) {
    if (t < tasks) {
      const int64_t o = t / nb;
      for (int k = lane; k < kMoWords; k += 32) {
        const uint32_t* src = k < 27 ? oid + int64_t(k) * n + o : k == 27 ? ometa + o : oelem + int64_t(k - 28) * n + o;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         static_cast<uint32_t>(__cvta_generic_to_shared(&slot[w][sl][k]))),
                     "l"(src)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int64_t t = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  fetch(t, 0);
  for (int it = 0; t < tasks; t += wstride, ++it) {
    const int sl = it & 1;
    __syncwarp();
    fetch(t + wstride, sl ^ 1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncwarp();
    const uint32_t* W = slot[w][sl];
    const int64_t o = t / nb;
    const int col = int(t - o * nb) * 64 + 2 * lane;
    const uint32_t m = W[27];
    uint32_t none = 0;
    F2 xv[27], yv[27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = W[p];
      none |= id == kNoNode ? (1u << p) : 0u;
      xv[p].v = id != kNoNode ? __ldg(reinterpret_cast<const unsigned long long*>(X + int64_t(id) * R + col))
                              : 0ull;
    }
    octet_apply<F2>(xv, yv, none, m, [&](int c, F2& f1, F2& f2) {
      if (ca) {
        const uint32_t e = W[28 + c];
        f1 *= F2(__ldg(ca + e));
        f2 *= F2(__ldg(cb + e));
      }
    });
    const uint32_t cm = ometa_cmask(m);
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = W[p];
      if (id == kNoNode) continue;
      float* dst = Y + int64_t(id) * R + col;
      const float a = __uint_as_float(uint32_t(yv[p].v)), b = __uint_as_float(uint32_t(yv[p].v >> 32));
      if (p == 13 && cm == 255u)
        asm volatile("st.global.v2.f32 [%0], {%1, %2};" ::"l"(dst), "f"(a), "f"(b) : "memory");
      else if (nonzero(yv[p]))
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(dst), "f"(a), "f"(b) : "memory");
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Octet chunks with the chunk's sums in shared memory: a CTA per (chunk of
// kOctChunk octets, 32 right-hand sides).  Its warps work the chunk's octets
// as the octet kernel above does (a lane per right-hand side, the next
// octet's words in flight), but add each octet's lattice sums into the
// chunk's rows in shared memory (shared atomics: lanes hit 32 distinct
// words of one row); then each node's row leaves once -- a store for a node
// no other chunk touches, a global reduction for the others.  The global
// reductions per node fall from one per octet touching it to one per chunk.
template <class T, int WARPS>
__global__ void __launch_bounds__(32 * WARPS, 1) mrhs_chunk_kernel(
    int64_t n, int64_t nchunk, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
    const uint16_t* __restrict__ lidx, const uint32_t* __restrict__ oelem, const uint32_t* __restrict__ cptr,
    const uint32_t* __restrict__ cnodes, const T* __restrict__ ca, const T* __restrict__ cb, int R,
    const T* __restrict__ X, T* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char mc_smem[];
  uint32_t(*slot)[2][kMoWords] = reinterpret_cast<uint32_t(*)[2][kMoWords]>(mc_smem);
  T* sy = reinterpret_cast<T*>(mc_smem + sizeof(uint32_t) * WARPS * 2 * kMoWords);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ng = R / 32;
  const int64_t items = nchunk * ng;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int64_t q = it / ng;
    const int col = int(it - q * ng) * 32 + lane;
    const uint32_t p0 = __ldg(cptr + q), nn = __ldg(cptr + q + 1) - p0;
    for (uint32_t i = threadIdx.x; i < nn * 32; i += 32 * WARPS) sy[i] = T(0);
    __syncthreads();
    const int64_t o0 = q * kOctChunk;
    const int cnt = int(n - o0 < kOctChunk ? n - o0 : kOctChunk);
    auto fetch = [&](int j, int sl) {
      if (j < cnt) {
        const int64_t o = o0 + j;
        for (int k = lane; k < kMoWords; k += 32) {
          const uint32_t* src = k < 27 ? oid + int64_t(k) * n + o : k == 27 ? ometa + o : oelem + int64_t(k - 28) * n + o;
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                           static_cast<uint32_t>(__cvta_generic_to_shared(&slot[w][sl][k]))),
                       "l"(src)
                       : "memory");
        }
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    fetch(w, 0);
    for (int j = w, i = 0; j < cnt; j += WARPS, ++i) {
      const int sl = i & 1;
      __syncwarp();
      fetch(j + WARPS, sl ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
      __syncwarp();
      const uint32_t* W = slot[w][sl];
      const int64_t o = o0 + j;
      const uint32_t m = W[27];
      uint32_t none = 0;
      T xv[27], yv[27];
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        const uint32_t id = W[p];
        none |= id == kNoNode ? (1u << p) : 0u;
        xv[p] = id != kNoNode ? __ldg(X + int64_t(id) * R + col) : T(0);
      }
      octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
        if (ca) {
          const uint32_t e = W[28 + c];
          f1 *= __ldg(ca + e);
          f2 *= __ldg(cb + e);
        }
      });
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        if ((none >> p) & 1u) continue;
        const uint32_t li = __ldg(lidx + int64_t(p) * n + o);
        if (yv[p] != T(0)) atomicAdd(sy + size_t(li) * 32 + lane, yv[p]);
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    for (uint32_t k = w; k < nn; k += WARPS) {
      const uint32_t id = __ldg(cnodes + p0 + k);
      const T v = sy[size_t(k) * 32 + lane];
      T* dst = Y + int64_t(id & 0x7fffffffu) * R + col;
      if (!(id >> 31)) *dst = v;
      else if (v != T(0)) atomicAdd(dst, v);
    }
    __syncthreads();
  }
}
constexpr int kMcWarps = 16;
template <class T>
constexpr size_t mrhs_chunk_smem(uint32_t max_nodes) {
  return sizeof(uint32_t) * kMcWarps * 2 * kMoWords + sizeof(T) * 32 * size_t(max_nodes);
}

}  // namespace

template <class T>
dg_status mrhs_octet_apply(const dg_mat* A, const T* coef, const T* X, T* Y, int R, cudaStream_t s) {
  const dg_da* da = A->da;
  const OctetSet& O = da->octs;
  DG_CHECK(A->kind == 0 && R % 32 == 0 && O.n > 0, DG_EINVAL, "multi-RHS octet operator: bad arguments");
  DG_CUDA(cudaMemsetAsync(Y, 0, sizeof(T) * size_t(da->N) * R, s));
  const T* ca = A->has_coef ? coef : nullptr;
  const T* cb = A->has_coef ? coef + da->E : nullptr;
  // chunks whose rows fit in shared memory: the chunked form (one CTA per SM)
  const size_t csmem = mrhs_chunk_smem<T>(O.max_nodes);
  // DG_MRHS_OCTET=chunk: the chunked form (measured slower than the direct
  // one on the 64-RHS benchmark mesh: one CTA per SM and a barrier per chunk)
  static int chunked = -1;
  if (chunked < 0) {
    const char* e = getenv("DG_MRHS_OCTET");
    chunked = (e && !strcmp(e, "chunk")) ? 1 : 0;
  }
  if (chunked && O.nchunk > 0 && csmem <= size_t(220) << 10) {
    static bool attr[2] = {false, false};
    auto kern = mrhs_chunk_kernel<T, kMcWarps>;
    if (!attr[sizeof(T) == 8]) {
      DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(size_t(220) << 10)));
      attr[sizeof(T) == 8] = true;
    }
    const unsigned grid = unsigned(std::min<int64_t>(O.nchunk * (R / 32), int64_t(sm_count())));
    kern<<<grid, 32 * kMcWarps, csmem, s>>>(O.n, O.nchunk, O.meta.p, O.id.p, O.lidx.p, O.elem.p, O.cptr.p,
                                            O.cnodes.p, ca, cb, R, X, Y);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  static int pairs = -1;  // DG_MRHS_OCTET=single: one right-hand side per lane
  if (pairs < 0) {
    const char* e = getenv("DG_MRHS_OCTET");
    pairs = (e && !strcmp(e, "single")) ? 0 : 1;
  }
  if (sizeof(T) == 4 && pairs && R % 64 == 0) {
    const int64_t warps = O.n * (R / 64);
    const unsigned grid = unsigned(std::min<int64_t>((warps + 3) / 4, int64_t(sm_count()) * 16));
    mrhs_octet_pair_kernel<<<grid, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p,
                                                reinterpret_cast<const float*>(ca),
                                                reinterpret_cast<const float*>(cb), R,
                                                reinterpret_cast<const float*>(X), reinterpret_cast<float*>(Y));
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  const int64_t warps = O.n * (R / 32);
  const unsigned grid = unsigned(std::min<int64_t>((warps + 3) / 4, int64_t(sm_count()) * 16));
  mrhs_octet_pf_kernel<T><<<grid, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, R, X, Y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
template dg_status mrhs_octet_apply<float>(const dg_mat*, const float*, const float*, float*, int, cudaStream_t);
template dg_status mrhs_octet_apply<double>(const dg_mat*, const double*, const double*, double*, int,
                                            cudaStream_t);

dg_status mrhs_apply(const dg_mat* A, const float* X, float* Y, int R, int split, cudaStream_t s) {
  dg_da* da = A->da;
  DG_CHECK(A->kind == 0, DG_EINVAL, "mat_mult_multi: scalar operator expected");
  DG_CHECK(R > 0 && R % kRC == 0, DG_EINVAL, "mat_mult_multi: nrhs must be a positive multiple of 16");
  DG_CHECK(split == 0 || split == 1 || split == 3 || split == 4 || split == 5, DG_EINVAL,
           "mat_mult_multi: split must be 0, 1, 3, 4 or 5");
  DG_CHECK((reinterpret_cast<uintptr_t>(X) & 15) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0, DG_EINVAL,
           "mat_mult_multi: X and Y must be 16-byte aligned");
  if (split >= 4) return mrhs_tc_apply(A, X, Y, R, split == 4 ? 1 : 3, s);
  static float4* tbls[64] = {};  // one table per device, kept for the process
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CHECK(dev >= 0 && dev < 64, DG_EINVAL, "device index");
  if (!tbls[dev]) {
    std::vector<float> h = stencil_tables();
    float4* p = nullptr;
    DG_CUDA(cudaMalloc(&p, h.size() * sizeof(float)));
    DG_CUDA(cudaMemcpy(p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
    tbls[dev] = p;
  }
  const float4* tbl = tbls[dev];
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  static int form = -1;
  if (form < 0) {  // DG_MRHS_KERNEL: block (default, 32 per pass) | block64 | direct | stage | cta | octet
    const char* e = getenv("DG_MRHS_KERNEL");
    form = (e && !strcmp(e, "cta"))       ? 2
           : (e && !strcmp(e, "stage"))   ? 1
           : (e && !strcmp(e, "direct"))  ? 0
           : (e && !strcmp(e, "block64")) ? 4
           : (e && !strcmp(e, "octet"))   ? 5
                                          : 3;
  }
  if (split == 0 || form == 5) {
    DG_CHECK(R % 32 == 0 && da->octs.n > 0, DG_EINVAL, "mat_mult_multi: the octet form takes nrhs a multiple of 32");
    return mrhs_octet_apply<float>(A, A->has_coef ? A->coef32.p : nullptr, X, Y, R, s);
  }
  if (form >= 3 && R % 32 == 0) {
    static float4* ftbls[64] = {};  // frame tables, one per device, kept for the process
    if (!ftbls[dev]) {
      std::vector<float> h = frame_stencil_tables();
      float4* p = nullptr;
      DG_CUDA(cudaMalloc(&p, h.size() * sizeof(float)));
      DG_CUDA(cudaMemcpy(p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
      ftbls[dev] = p;
    }
    const TileSet& ts = da->tiles_w;
    if (ts.nshared)
      zero_shared_rows<<<grid_for(ts.nshared * (R / 4), 256, 8), 256, 0, s>>>(ts.shared.p, ts.nshared, R / 4,
                                                                             reinterpret_cast<float4*>(Y));
    const uint32_t cap = ts.max_nodes;
    const int W = (R % 64 == 0 && form == 4) ? 64 : 32;
    const int smem = int(kBWarps * mrhs_block_stride(cap, W) * sizeof(float));
    DG_CHECK(smem <= 220 * 1024, DG_EINVAL, "mat_mult_multi: tile node count too large");
    auto kern = W == 64 ? (split == 1 ? mrhs_block_kernel<1, 64, 2> : mrhs_block_kernel<3, 64, 2>)
                        : (split == 1 ? mrhs_block_kernel<1, 32, 3> : mrhs_block_kernel<3, 32, 3>);
    static int granted_b[4] = {48 * 1024, 48 * 1024, 48 * 1024, 48 * 1024};
    int& gr = granted_b[(W == 64 ? 2 : 0) + (split == 1 ? 0 : 1)];
    if (smem > gr) {
      DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      gr = smem;
    }
    const unsigned grid = grid_for(ts.ntiles * 32, 32 * kBWarps, 16);
    kern<<<grid, 32 * kBWarps, smem, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p, ts.nodes.p,
                                          reinterpret_cast<const uint2*>(ts.eloc8.p), ftbls[dev], R, cap, X, Y);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  if (form != 2) {  // warp tiles, 16 right-hand sides per pass
    const TileSet& ts = da->tiles_w;
    if (ts.nshared)
      zero_shared_rows<<<grid_for(ts.nshared * (R / 4), 256, 8), 256, 0, s>>>(ts.shared.p, ts.nshared, R / 4,
                                                                             reinterpret_cast<float4*>(Y));
    const uint32_t cap = ts.max_nodes;
    const bool stage = form == 1;
    const int smem = int(kMWarps * mrhs_warp_stride(cap, stage) * sizeof(float));
    DG_CHECK(smem <= 220 * 1024, DG_EINVAL, "mat_mult_multi: tile node count too large");
    auto kern = stage ? (split == 1 ? mrhs_warp_kernel<1, true> : mrhs_warp_kernel<3, true>)
                      : (split == 1 ? mrhs_warp_kernel<1, false> : mrhs_warp_kernel<3, false>);
    static int granted_w[4] = {48 * 1024, 48 * 1024, 48 * 1024, 48 * 1024};
    int& gr = granted_w[(stage ? 2 : 0) + (split == 1 ? 0 : 1)];
    if (smem > gr) {
      DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      gr = smem;
    }
    const unsigned grid = grid_for(ts.ntiles * 32, 32 * kMWarps, 16);
    kern<<<grid, 32 * kMWarps, smem, s>>>(da->meta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p, ts.nodes.p,
                                          reinterpret_cast<const uint2*>(ts.eloc8.p), tbl, R, cap, X, Y);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  if (!da->tiles_mr.ntiles) DG_TRY(build_tile_set(da, kMultiTile, da->tiles_mr, s));
  const TileSet& ts = da->tiles_mr;
  if (ts.nshared)
    zero_shared_rows<<<grid_for(ts.nshared * (R / 4), 256, 8), 256, 0, s>>>(ts.shared.p, ts.nshared, R / 4,
                                                                           reinterpret_cast<float4*>(Y));
  const uint32_t cap = ts.max_nodes;
  const int smem = int(2 * size_t(cap) * kRW * sizeof(float));
  DG_CHECK(smem <= 220 * 1024, DG_EINVAL, "mat_mult_multi: tile node count too large");
  static int granted = 48 * 1024;
  if (smem > granted) {
    DG_CUDA(cudaFuncSetAttribute(mrhs_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    DG_CUDA(cudaFuncSetAttribute(mrhs_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    granted = smem;
  }
  if (split == 1)
    mrhs_kernel<1><<<unsigned(ts.ntiles), kMThreads, smem, s>>>(da->meta.p, ca, cb, da->E, ts.ptr.p, ts.nodes.p,
                                                               ts.eloc.p, tbl, R, cap, X, Y);
  else
    mrhs_kernel<3><<<unsigned(ts.ntiles), kMThreads, smem, s>>>(da->meta.p, ca, cb, da->E, ts.ptr.p, ts.nodes.p,
                                                               ts.eloc.p, tbl, R, cap, X, Y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg
