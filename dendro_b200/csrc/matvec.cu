// Matrix-free elemental operators on the GPU (the PETSc MatShell callbacks):
//  * Laplacian + mass, JAC_TYPE2_ELEM_MULT_BLOCK / Jacobian2MatMult
//    (examples/src/backend/omgNeumann.C:468-557),
//  * its diagonal, JAC_TYPE2_ELEM_DIAG_BLOCK (omgNeumann.C:396-465),
//  * 3-dof linear elasticity, ELASTICITY_ELEM_MULT_BLOCK
//    (examples/src/backend/elasticityJac.C:130-230).
//
// The reference multiplies by precomputed tables L[c][t], M[c][t] (8x8) and
// GD[c][t] (24x24) per (child number, element type).  Each table equals
// T^T A T, where A is the reference-cube Q1 matrix and T interpolates the
// element's vertex values from its node values (a hanging vertex takes the
// mean of the parent vertices on its edge or face).  The kernels apply T,
// A on [-1,1]^3, then T^T, which needs no tables.  A itself is applied in the
// basis where it is diagonal: along each axis the 1D mass and stiffness
// matrices M1 = [[2,1],[1,2]]/3 and K1 = [[1,-1],[-1,1]]/2 share the
// eigenvectors (1,1) and (1,-1), so A = f1 K + f2 M = W diag(l) W / 8 with W
// the 8-point Walsh-Hadamard transform and l depending only on the number of
// (1,-1) factors; 56 flops per scalar element instead of 256.
#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

#include "cmap.cuh"
#include "dg_internal.h"
#include "octet.cuh"

namespace dg {

namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

// Hanging interpolation u_vertex = T u_node, in place.  A hanging vertex i
// takes the mean of the nodes j that differ from i only on the axes where i
// and the child number c differ (2 nodes on an edge, 4 on a face).  All array
// indices are compile-time constants so the values stay in registers.
template <class T>
__device__ __forceinline__ void interp_hanging(T (&u)[8], uint32_t c, uint32_t mask) {
  T un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) un[v] = u[v];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if ((mask >> i) & 1u) {
      const uint32_t keep = ~((uint32_t(i) ^ c)) & 7u;  // axes on which j must equal i
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc += (((uint32_t(j ^ i)) & keep) == 0u) ? un[j] : T(0);
      u[i] = acc * ((__popc(keep) == 2) ? T(0.5) : T(0.25));
    }
  }
}
// r_node = T^T r_vertex, in place.
template <class T>
__device__ __forceinline__ void scatter_hanging(T (&r)[8], uint32_t c, uint32_t mask) {
  T rn[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) rn[v] = ((mask >> v) & 1u) ? T(0) : r[v];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if ((mask >> i) & 1u) {
      const uint32_t keep = ~((uint32_t(i) ^ c)) & 7u;
      const T w = r[i] * ((__popc(keep) == 2) ? T(0.5) : T(0.25));
#pragma unroll
      for (int j = 0; j < 8; ++j) rn[j] += (((uint32_t(j ^ i)) & keep) == 0u) ? w : T(0);
    }
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] = rn[v];
}

// XOR relabelling of a vertex-indexed array by the child number: a[j] <- a[j ^ c]
// (an involution).  In this frame the element's own corner of its parent is
// vertex 0 and the hanging-vertex structure no longer depends on c.
template <class T>
__device__ __forceinline__ void xor_perm(T (&a)[8], uint32_t c) {
#pragma unroll
  for (int B = 1; B < 8; B <<= 1) {
    const bool f = (c & B) != 0;
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (!(v & B)) {
        const T p = a[v], q = a[v | B];
        a[v] = f ? q : p;
        a[v | B] = f ? p : q;
      }
  }
}
// T and T^T in the child-number frame.  A hanging vertex j lies on the
// parent's edge (j = 1, 2, 4) or face (j = 3, 5, 6) through the shared corner
// 0 and takes the mean of the node values of the vertices j' with j' a bit
// subset of j; vertices 0 and 7 are never hanging.
template <class T>
__device__ __forceinline__ void interp_frame(T (&w)[8], uint32_t mp) {
  const T w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3], w4 = w[4], w5 = w[5], w6 = w[6];
  if (mp & 0x02u) w[1] = (w0 + w1) * T(0.5);
  if (mp & 0x04u) w[2] = (w0 + w2) * T(0.5);
  if (mp & 0x10u) w[4] = (w0 + w4) * T(0.5);
  if (mp & 0x08u) w[3] = ((w0 + w1) + (w2 + w3)) * T(0.25);
  if (mp & 0x20u) w[5] = ((w0 + w1) + (w4 + w5)) * T(0.25);
  if (mp & 0x40u) w[6] = ((w0 + w2) + (w4 + w6)) * T(0.25);
}
template <class T>
__device__ __forceinline__ void scatter_frame(T (&r)[8], uint32_t mp) {
  const T h1 = (mp & 0x02u) ? r[1] * T(0.5) : T(0), h2 = (mp & 0x04u) ? r[2] * T(0.5) : T(0);
  const T h4 = (mp & 0x10u) ? r[4] * T(0.5) : T(0);
  const T q3 = (mp & 0x08u) ? r[3] * T(0.25) : T(0), q5 = (mp & 0x20u) ? r[5] * T(0.25) : T(0);
  const T q6 = (mp & 0x40u) ? r[6] * T(0.25) : T(0);
  r[0] += (h1 + h2) + (h4 + q3) + (q5 + q6);
  r[1] = ((mp & 0x02u) ? h1 : r[1]) + (q3 + q5);
  r[2] = ((mp & 0x04u) ? h2 : r[2]) + (q3 + q6);
  r[4] = ((mp & 0x10u) ? h4 : r[4]) + (q5 + q6);
  if (mp & 0x08u) r[3] = q3;
  if (mp & 0x20u) r[5] = q5;
  if (mp & 0x40u) r[6] = q6;
}

// One thread per element: gather, apply, scatter with atomics.  BLOCK and
// MINB set the launch bounds (registers per thread) of each tuned variant.
template <class T, class CT, int BLOCK = 256, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_kernel(const uint32_t* __restrict__ nl,
                                                              const uint32_t* __restrict__ meta,
                                                              const CT* __restrict__ ca, const CT* __restrict__ cb,
                                                              int64_t E, const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const T h = elem_h<T>(lev);
    const T a = ca ? T(ca[e]) : T(1), b = cb ? T(cb[e]) : T(1);
    const T f1 = a * h / T(2), f2 = b * h * h * h / T(8);
    uint32_t id[8];
    T u[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) id[v] = __ldg(nl + int64_t(v) * E + e);
    xor_perm(id, c);  // child-number frame: id[j] is the node of vertex j ^ c
#pragma unroll
    for (int j = 0; j < 8; ++j) u[j] = __ldg(x + id[j]);
    const uint32_t mp = xor_perm_mask(mask, c);
    if (mp) interp_frame(u, mp);
    lapmass_ref(u, f1, f2);
    if (mp) scatter_frame(u, mp);
#pragma unroll
    for (int j = 0; j < 8; ++j) atomicAdd(y + id[j], u[j]);
  }
}

// Load vector (ComputeRHS_omgNeumann, examples/src/backend/omgNeumann.C:
// 749-785): b += f_e h^3 / 8 T^T 1 per element, the force sampled at the
// element's centre times the integrals of its vertices' shape functions
// (RHSType2Stencil), the hanging vertices' shares moved to their nodes by the
// frame fold.
__global__ void load_vector_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                   const double* __restrict__ force, int64_t E, double* __restrict__ b) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t c = meta_cnum(m);
    const double h = elem_h<double>(meta_lev(m));
    const double w = force[e] * h * h * h * 0.125;
    uint32_t id[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) id[v] = __ldg(nl + int64_t(v) * E + e);
    xor_perm(id, c);
    double u[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) u[j] = w;
    const uint32_t mp = xor_perm_mask(meta_mask(m), c);
    if (mp) scatter_frame(u, mp);
#pragma unroll
    for (int j = 0; j < 8; ++j) atomicAdd(b + id[j], u[j]);
  }
}

// The element kernel on the compressed element map: a warp per tile of 32
// consecutive elements decodes its lanes' node ids (cmap.cuh), then each lane
// gathers, applies and scatters its element as lapmass_kernel does.  The map
// moves about 12 bytes per element instead of 32.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_cmap_kernel(CMapView M, int64_t ntiles,
                                                                   const uint32_t* __restrict__ meta,
                                                                   const CT* __restrict__ ca,
                                                                   const CT* __restrict__ cb, const T* __restrict__ x,
                                                                   T* __restrict__ y) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t nw = int64_t(gridDim.x) * (BLOCK / 32);
  for (int64_t t = (int64_t(blockIdx.x) * BLOCK + threadIdx.x) >> 5; t < ntiles; t += nw) {
    uint32_t id[8];
    cmap_ids(M, t, lane, id);
    const int64_t e = t * 32 + lane;
    if (e >= M.E) continue;
    const uint32_t m = __ldg(meta + e);
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const T h = elem_h<T>(lev);
    const T a = ca ? T(ca[e]) : T(1), b = cb ? T(cb[e]) : T(1);
    const T f1 = a * h / T(2), f2 = b * h * h * h / T(8);
    T u[8];
    xor_perm(id, c);
#pragma unroll
    for (int j = 0; j < 8; ++j) u[j] = __ldg(x + id[j]);
    const uint32_t mp = xor_perm_mask(mask, c);
    if (mp) interp_frame(u, mp);
    lapmass_ref(u, f1, f2);
    if (mp) scatter_frame(u, mp);
#pragma unroll
    for (int j = 0; j < 8; ++j) atomicAdd(y + id[j], u[j]);
  }
}

// Jacobi update and residual from an operator application t = A x, which
// they read and zero again (t stays zero between uses, as the warp-tile
// kernel's atomics need).
template <class T>
__global__ void jacobi_from(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv,
                            T* __restrict__ t, T omega, int64_t n) {
  #pragma unroll 4
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const T ti = t[i];
    t[i] = T(0);
    x[i] += omega * dinv[i] * (b[i] - ti);
  }
}
template <class T>
__global__ void residual_from(const T* __restrict__ b, T* __restrict__ t, T* __restrict__ r, int64_t n) {
  #pragma unroll 4
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const T ti = t[i];
    t[i] = T(0);
    r[i] = b[i] - ti;
  }
}

// 16-byte forms (4 floats or 2 doubles per step) for vectors that are whole
// allocations (16-byte aligned); the callers check the alignment.
template <class T>
using Vec16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
// Each thread takes kVecU 16-byte steps a grid stride apart and issues all
// their loads before any store: with one step per iteration these passes ran
// at a third of the HBM bandwidth (the next step's loads waited behind the
// stores), with four they stream at 0.9 of it.
constexpr int kVecU = 4;
template <class T>
__global__ void jacobi_from_v(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv,
                              T* __restrict__ t, T omega, int64_t nv, int64_t n) {
  using V = Vec16<T>;
  constexpr int W = 16 / sizeof(T);
  const int64_t S = gstride();
  // the last n - nv * W (< W) entries, by the first threads
  if (nv * W + gtid() < n) {
    const int64_t j = nv * W + gtid();
    const T tj = t[j];
    t[j] = T(0);
    x[j] += omega * dinv[j] * (b[j] - tj);
  }
  for (int64_t i0 = gtid(); i0 < nv; i0 += S * kVecU) {
    V tv[kVecU], xv[kVecU], bv[kVecU], dv[kVecU];
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * S;
      if (i < nv) {
        tv[u] = reinterpret_cast<const V*>(t)[i];
        xv[u] = reinterpret_cast<const V*>(x)[i];
        bv[u] = reinterpret_cast<const V*>(b)[i];
        dv[u] = reinterpret_cast<const V*>(dinv)[i];
      }
    }
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * S;
      if (i >= nv) continue;
      T* tp = reinterpret_cast<T*>(&tv[u]);
      T* xp = reinterpret_cast<T*>(&xv[u]);
      const T* bp = reinterpret_cast<const T*>(&bv[u]);
      const T* dp = reinterpret_cast<const T*>(&dv[u]);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        xp[k] += omega * dp[k] * (bp[k] - tp[k]);
        tp[k] = T(0);
      }
      reinterpret_cast<V*>(t)[i] = tv[u];
      reinterpret_cast<V*>(x)[i] = xv[u];
    }
  }
}
template <class T>
__global__ void residual_from_v(const T* __restrict__ b, T* __restrict__ t, T* __restrict__ r, int64_t nv,
                                int64_t n) {
  using V = Vec16<T>;
  constexpr int W = 16 / sizeof(T);
  const int64_t S = gstride();
  if (nv * W + gtid() < n) {
    const int64_t j = nv * W + gtid();
    const T tj = t[j];
    t[j] = T(0);
    r[j] = b[j] - tj;
  }
  for (int64_t i0 = gtid(); i0 < nv; i0 += S * kVecU) {
    V tv[kVecU], bv[kVecU];
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * S;
      if (i < nv) {
        tv[u] = reinterpret_cast<const V*>(t)[i];
        bv[u] = reinterpret_cast<const V*>(b)[i];
      }
    }
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * S;
      if (i >= nv) continue;
      V rv;
      T* tp = reinterpret_cast<T*>(&tv[u]);
      T* rp = reinterpret_cast<T*>(&rv);
      const T* bp = reinterpret_cast<const T*>(&bv[u]);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        rp[k] = bp[k] - tp[k];
        tp[k] = T(0);
      }
      reinterpret_cast<V*>(t)[i] = tv[u];
      reinterpret_cast<V*>(r)[i] = rv;
    }
  }
}

// Warp-tile variant: each warp owns tiles of kWarpTile consecutive elements
// (one per lane) with warp-private shared buffers, so the phases of a tile
// synchronise with __syncwarp only and the warps of an SM progress
// independently.  Per tile: x at the tile's nodes is staged once; each lane
// applies its element operator, reading x through its 8 node ranks (one
// 8-byte load), and writes its 8 results by (vertex, element) position; the
// tile's 256 references, sorted by node, are then summed 8 consecutive ones
// per lane, following per-reference flags built with the mesh (start a sum,
// let it leave, as a store or an atomic).  Node ranks, hanging masks and
// result positions are stored in the child-number frame, so an element needs
// no relabelling at run time.  A sum leaves with a store when the
// node's whole run lies in one lane and no other tile uses the node, else
// with an FP64 global atomic (y is zeroed first).
constexpr int kWarpCta = 8;  // warps per CTA


// Predicated global store / reduction-add (no branch; c == 0 skips the access).
__device__ __forceinline__ void st_if(double* p, double v, uint32_t c) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.f64 [%0], %1;\n}" ::"l"(p), "d"(v),
               "r"(c)
               : "memory");
}
__device__ __forceinline__ void st_if(float* p, float v, uint32_t c) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.f32 [%0], %1;\n}" ::"l"(p), "f"(v),
               "r"(c)
               : "memory");
}
__device__ __forceinline__ void red_add_if(double* p, double v, uint32_t c) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q red.global.add.f64 [%0], %1;\n}" ::"l"(p),
               "d"(v), "r"(c)
               : "memory");
}
__device__ __forceinline__ void red_add_if(float* p, float v, uint32_t c) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q red.global.add.f32 [%0], %1;\n}" ::"l"(p),
               "f"(v), "r"(c)
               : "memory");
}

// The segmented sum of a lane's 8 sorted references, without branches:
// sx holds the element results by frame position, sn the tile's node ids by
// rank.  A reference that starts a sum replaces it; one whose flag says the
// sum leaves stores it (node whole in this lane and tile) or adds it with a
// global reduction.  Padding references (after a lane's last real one) point
// at position 0 and rank 0 and carry no flags, so they read valid slots and
// never leave.
template <class T>
__device__ __forceinline__ void warp_seg_sum(const T* sx, const uint32_t* sn, uint2 pp, uint2 rr, uint32_t ff,
                                             T* __restrict__ y) {
  T sum = T(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const T v = sx[byte_of(pp, q)];
    sum = (ff & (0x100u << q)) ? v : sum + v;
    const uint32_t leave = ff & (0x10000u << q), store = ff & (0x1000000u << q);
    const uint32_t id = leave ? sn[byte_of(rr, q)] : 0u;  // shared load only where the sum leaves
    T* dst = y + (id & 0x7fffffffu);
    st_if(dst, sum, store);
    red_add_if(dst, sum, leave && !store);
  }
}

// Per-lane record of one tile: the lane's element and its 8 sorted references.
template <class T>
struct WarpTileLoad {
  uint32_t m, p0, nt;
  uint2 L, pp, rr;
  uint32_t ff;  // bit q: reference q valid; 8 + q: starts a sum; 16 + q: sum leaves; 24 + q: as a store
  T a, b;
};
template <class T, class CT>
__device__ __forceinline__ void load_warp_tile(WarpTileLoad<T>& d, int64_t t, int lane, int64_t E,
                                               const uint32_t* __restrict__ wmeta, const CT* __restrict__ ca,
                                               const CT* __restrict__ cb, const uint32_t* __restrict__ tile_ptr,
                                               const uint2* __restrict__ eloc8, const uint8_t* __restrict__ ref8) {
  constexpr int S = 8 * kWarpTile;
  const int64_t e = t * kWarpTile + lane;
  d.m = 0;
  d.L = make_uint2(0, 0);
  d.a = T(1);
  d.b = T(1);
  if (e < E) {
    d.m = __ldg(wmeta + e);
    d.L = __ldg(eloc8 + e);
    if (ca) {
      d.a = T(__ldg(ca + e));
      d.b = T(__ldg(cb + e));
    }
  }
  const uint8_t* tr = ref8 + t * kWarpRefBytes;
  d.pp = __ldg(reinterpret_cast<const uint2*>(tr) + lane);
  d.rr = __ldg(reinterpret_cast<const uint2*>(tr + S) + lane);
  d.ff = __ldg(reinterpret_cast<const uint32_t*>(tr + 2 * S) + lane);
  d.p0 = __ldg(tile_ptr + t);
  d.nt = __ldg(tile_ptr + t + 1) - d.p0;
}

// MINB: CTAs per SM the register budget is set for.  PF: load the next
// tile's records before working on the current one (more registers, the
// loads' latency hidden behind the current tile).
template <class T, class CT, int MINB, bool PF>
__global__ void __launch_bounds__(32 * kWarpCta, MINB) lapmass_warp_kernel(
    const uint32_t* __restrict__ wmeta, const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
    int64_t ntiles, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_nodes,
    const uint2* __restrict__ eloc8, const uint8_t* __restrict__ ref8, const T* __restrict__ x,
    T* __restrict__ y) {
  constexpr int S = 8 * kWarpTile;
  __shared__ T s_x[kWarpCta][S];  // x at the tile's nodes by rank, then element results by position
  __shared__ uint32_t s_nodes[kWarpCta][S];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T* sx = s_x[w];
  uint32_t* sn = s_nodes[w];
  const int64_t nw = int64_t(gridDim.x) * kWarpCta;
  int64_t t = blockIdx.x * int64_t(kWarpCta) + w;
  WarpTileLoad<T> cur, nxt;
  if (PF && t < ntiles) load_warp_tile<T, CT>(cur, t, lane, E, wmeta, ca, cb, tile_ptr, eloc8, ref8);
  for (; t < ntiles; t += nw) {
    if (PF) {
      if (t + nw < ntiles) load_warp_tile<T, CT>(nxt, t + nw, lane, E, wmeta, ca, cb, tile_ptr, eloc8, ref8);
    } else {
      load_warp_tile<T, CT>(cur, t, lane, E, wmeta, ca, cb, tile_ptr, eloc8, ref8);
    }
    const bool live = t * kWarpTile + lane < E;
    for (uint32_t k = lane; k < cur.nt; k += 32) {
      const uint32_t id = __ldg(tile_nodes + cur.p0 + k);
      sn[k] = id;
      sx[k] = __ldg(x + (id & 0x7fffffffu));
    }
    __syncwarp();
    T wv[8];
    if (live) {
      const T h = elem_h<T>(meta_lev(cur.m));
      const T f1 = cur.a * h * T(0.5), f2 = cur.b * h * h * h * T(0.125);
#pragma unroll
      for (int j = 0; j < 8; ++j) wv[j] = sx[byte_of(cur.L, j)];  // byte j: rank of frame vertex j
      const uint32_t mp = wmeta_mask(cur.m);
      if (mp) interp_frame(wv, mp);
      lapmass_ref(wv, f1, f2);
      if (mp) scatter_frame(wv, mp);
    }
    __syncwarp();  // every lane has read x: its buffer now takes the results
    if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) sx[j * kWarpTile + lane] = wv[j];
    }
    __syncwarp();
    warp_seg_sum(sx, sn, cur.pp, cur.rr, cur.ff, y);
    __syncwarp();
    if (PF) cur = nxt;
  }
}


// Deeper software pipeline over a warp's tiles: while tile t is worked on,
// the records of tile t + 1 (loaded at the top), then its node ids (issued
// after the element phase of t) and then x at those nodes (issued after the
// segmented sum of t) travel in registers, so that of the three dependent
// global round trips of a tile (list offsets, node ids, x) only the last is
// exposed.  Up to kPipeIds node ids per lane ride along (tiles of up to
// 32 kPipeIds nodes); larger tiles load the rest in place.
constexpr int kPipeIds = 3;
template <class T, class CT, int MINB>
__global__ void __launch_bounds__(32 * kWarpCta, MINB) lapmass_warp_pipe_kernel(
    const uint32_t* __restrict__ wmeta, const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
    int64_t ntiles, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_nodes,
    const uint2* __restrict__ eloc8, const uint8_t* __restrict__ ref8, const T* __restrict__ x,
    T* __restrict__ y) {
  constexpr int S = 8 * kWarpTile;
  __shared__ T s_x[kWarpCta][S];
  __shared__ uint32_t s_nodes[kWarpCta][S];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T* sx = s_x[w];
  uint32_t* sn = s_nodes[w];
  const int64_t nw = int64_t(gridDim.x) * kWarpCta;
  int64_t t = blockIdx.x * int64_t(kWarpCta) + w;
  WarpTileLoad<T> cur, nxt;
  uint32_t idc[kPipeIds];
  T xc[kPipeIds];
  if (t < ntiles) {
    load_warp_tile<T, CT>(cur, t, lane, E, wmeta, ca, cb, tile_ptr, eloc8, ref8);
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      idc[j] = k < cur.nt ? __ldg(tile_nodes + cur.p0 + k) : 0u;
    }
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      xc[j] = k < cur.nt ? __ldg(x + (idc[j] & 0x7fffffffu)) : T(0);
    }
  }
  for (; t < ntiles; t += nw) {
    const bool has_next = t + nw < ntiles;
    if (has_next) load_warp_tile<T, CT>(nxt, t + nw, lane, E, wmeta, ca, cb, tile_ptr, eloc8, ref8);
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      if (k < cur.nt) {
        sn[k] = idc[j];
        sx[k] = xc[j];
      }
    }
    for (uint32_t k = lane + 32 * kPipeIds; k < cur.nt; k += 32) {
      const uint32_t id = __ldg(tile_nodes + cur.p0 + k);
      sn[k] = id;
      sx[k] = __ldg(x + (id & 0x7fffffffu));
    }
    __syncwarp();
    const bool live = t * kWarpTile + lane < E;
    T wv[8];
    if (live) {
      const T h = elem_h<T>(meta_lev(cur.m));
      const T f1 = cur.a * h * T(0.5), f2 = cur.b * h * h * h * T(0.125);
#pragma unroll
      for (int j = 0; j < 8; ++j) wv[j] = sx[byte_of(cur.L, j)];  // byte j: rank of frame vertex j
      const uint32_t mp = wmeta_mask(cur.m);
      if (mp) interp_frame(wv, mp);
      lapmass_ref(wv, f1, f2);
      if (mp) scatter_frame(wv, mp);
    }
    // the next tile's node ids: its record has had the element phase to arrive
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      idc[j] = (has_next && k < nxt.nt) ? __ldg(tile_nodes + nxt.p0 + k) : 0u;
    }
    __syncwarp();
    if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) sx[j * kWarpTile + lane] = wv[j];
    }
    __syncwarp();
    warp_seg_sum(sx, sn, cur.pp, cur.rr, cur.ff, y);
    // x at the next tile's nodes: the ids have had the segmented sum to arrive
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      xc[j] = (has_next && k < nxt.nt) ? __ldg(x + (idc[j] & 0x7fffffffu)) : T(0);
    }
    __syncwarp();
    if (has_next) cur = nxt;
  }
}

// ------------------------------------------------------------ octet form --
// One thread per octet, x and y in global memory: the octet's nodes gathered
// from x, each node's sum added into y (which must be zero or hold the
// values to add to) with one global reduction; the centre of an octet with
// all 8 children present belongs to no other element and leaves with a store.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octet_kernel(
    int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
    const uint32_t* __restrict__ oelem, const CT* __restrict__ ca, const CT* __restrict__ cb,
    const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t o = gtid(); o < n; o += gstride()) {
    const uint32_t m = __ldg(ometa + o);
    uint32_t id[27], none = 0;
    T xv[27], yv[27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      id[p] = __ldg(oid + int64_t(p) * n + o);
      none |= id[p] == kNoNode ? (1u << p) : 0u;
    }
    T fa[8], fb[8];
    if (ca) {
      const uint32_t cm0 = ometa_cmask(m);
      uint32_t el[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) el[c] = ((cm0 >> c) & 1u) ? __ldg(oelem + int64_t(c) * n + o) : 0u;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        fa[c] = ((cm0 >> c) & 1u) ? T(__ldg(ca + el[c])) : T(0);
        fb[c] = ((cm0 >> c) & 1u) ? T(__ldg(cb + el[c])) : T(0);
      }
    }
#pragma unroll
    for (int p = 0; p < 27; ++p) xv[p] = id[p] != kNoNode ? __ldg(x + id[p]) : T(0);
    octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
      if (ca) {
        f1 *= fa[c];
        f2 *= fb[c];
      }
    });
    const uint32_t cm = ometa_cmask(m);
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const bool node = id[p] != kNoNode;
      T* dst = y + (node ? id[p] : 0u);
      if (p == 13) {
        st_if(dst, yv[p], node && cm == 255u);
        red_add_if(dst, yv[p], node && cm != 255u);
      } else {
        red_add_if(dst, yv[p], node && yv[p] != T(0));
      }
    }
  }
}

// The one-thread-per-octet form with the next octet's words in flight: each
// thread copies the 27 node ids, 8 element ids and the meta word of the
// octet it works next (grid stride ahead) into its own shared-memory slot with
// 4-byte cp.async while it works the current one, so an octet's x gathers
// and coefficient loads issue at once, without the round trip for the ids,
// and the ids are read from shared memory (not held in registers) when the
// sums leave.  Slots are private to a thread: its own cp.async.wait_group is
// the only synchronisation.
constexpr int kOctPfWords = 36;  // 27 node ids, 8 element ids, meta
template <class T, class CT, int BLOCK, int MINB, bool HOIST = true, bool FAST = false>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octet_pf_kernel(
    int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
    const uint32_t* __restrict__ oelem, const CT* __restrict__ ca, const CT* __restrict__ cb,
    const T* __restrict__ x, T* __restrict__ y) {
  __shared__ uint32_t sw[2][kOctPfWords][BLOCK];  // [slot][word][thread]: a warp's accesses are consecutive words
  const int tid = threadIdx.x;
  const int64_t stride = gstride();
  auto fetch = [&](int64_t oo, int slot) {
    if (oo < n) {
#pragma unroll
      for (int p = 0; p < 27; ++p)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][p][tid]))),
                     "l"(oid + int64_t(p) * n + oo)
                     : "memory");
      if (ca) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                           static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][27 + c][tid]))),
                       "l"(oelem + int64_t(c) * n + oo)
                       : "memory");
      }
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                       static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][35][tid]))),
                   "l"(ometa + oo)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int64_t o = gtid();
  fetch(o, 0);
  for (int it = 0; o < n; o += stride, ++it) {
    const int sl = it & 1;
    fetch(o + stride, sl ^ 1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    const uint32_t m = sw[sl][35][tid];
    const uint32_t cm0 = ometa_cmask(m);
    // HOIST: all 16 coefficients loaded with the x gathers (more loads in
    // flight); otherwise each child's pair is loaded when its operator runs
    // (fewer registers)
    T fa[HOIST ? 8 : 1], fb[HOIST ? 8 : 1];
    if (HOIST && ca) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint32_t e = sw[sl][27 + c][tid];
        fa[c] = ((cm0 >> c) & 1u) ? T(__ldg(ca + e)) : T(0);
        fb[c] = ((cm0 >> c) & 1u) ? T(__ldg(cb + e)) : T(0);
      }
    }
    uint32_t none = 0;
    T xv[27], yv[27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = sw[sl][p][tid];
      none |= id == kNoNode ? (1u << p) : 0u;
      xv[p] = id != kNoNode ? __ldg(x + id) : T(0);
    }
    auto scale = [&](int c, T& f1, T& f2) {
      if (ca) {
        if (HOIST) {
          f1 *= fa[c];
          f2 *= fb[c];
        } else {
          const uint32_t e = sw[sl][27 + c][tid];
          f1 *= T(__ldg(ca + e));
          f2 *= T(__ldg(cb + e));
        }
      }
    };
    // FAST: a warp whose octets all have 8 children and no point to fill
    // takes the compile-time form of the arithmetic
    if (FAST && __all_sync(__activemask(), cm0 == 255u && (none & oct_hangable()) == 0u))
      octet_apply<T, true>(xv, yv, none, m, scale);
    else
      octet_apply<T>(xv, yv, none, m, scale);
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = sw[sl][p][tid];
      const bool node = id != kNoNode;
      T* dst = y + (node ? id : 0u);
      if (p == 13) {
        st_if(dst, yv[p], node && cm0 == 255u);
        red_add_if(dst, yv[p], node && cm0 != 255u);
      } else {
        red_add_if(dst, yv[p], node && yv[p] != T(0));
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// The next-ids-in-flight octet kernel worked in two halves to keep fewer
// lattice values live: the lower children (z bit 0) on lattice planes z = 0
// and 1, then the upper ones on planes 1 and 2.  Plane 0's sums are complete
// after the lower half (only those children touch it) and leave then, except
// its four corners, which still receive the folds of hanging points of plane
// 1 (vertical edges and faces); plane 1 interpolates its hanging points from
// the plane-2 corners, read with the lower half.  Peak: 22 x values and 18
// sums (instead of 27 + 27), so more warps fit.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octet_pf2_kernel(
    int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
    const uint32_t* __restrict__ oelem, const CT* __restrict__ ca, const CT* __restrict__ cb,
    const T* __restrict__ x, T* __restrict__ y) {
  __shared__ uint32_t sw[2][kOctPfWords][BLOCK];
  const int tid = threadIdx.x;
  const int64_t stride = gstride();
  auto fetch = [&](int64_t oo, int slot) {
    if (oo < n) {
#pragma unroll
      for (int p = 0; p < 27; ++p)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][p][tid]))),
                     "l"(oid + int64_t(p) * n + oo)
                     : "memory");
      if (ca) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                           static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][27 + c][tid]))),
                       "l"(oelem + int64_t(c) * n + oo)
                       : "memory");
      }
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                       static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][35][tid]))),
                   "l"(ometa + oo)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // plane-2 corners, lattice 18, 20, 24, 26, in c2[0..3]
  constexpr int kC2[4] = {18, 20, 24, 26};
  int64_t o = gtid();
  fetch(o, 0);
  for (int it = 0; o < n; o += stride, ++it) {
    const int sl = it & 1;
    fetch(o + stride, sl ^ 1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    const uint32_t m = sw[sl][35][tid];
    const uint32_t cm = ometa_cmask(m);
    uint32_t none = 0;
#pragma unroll
    for (int p = 0; p < 27; ++p) none |= sw[sl][p][tid] == kNoNode ? (1u << p) : 0u;
    auto xat = [&](int p) {
      const uint32_t id = sw[sl][p][tid];
      return id != kNoNode ? T(__ldg(x + id)) : T(0);
    };
    const T hh = elem_h<T>(ometa_lev(m));
    const T g1 = hh * T(0.5), g2 = hh * hh * hh * T(0.125);
    auto child = [&](int c, T (&u)[8]) {
      T f1 = g1, f2 = g2;
      if (ca) {
        const uint32_t e = sw[sl][27 + c][tid];
        f1 *= T(__ldg(ca + e));
        f2 *= T(__ldg(cb + e));
      }
      lapmass_ref(u, f1, f2);
    };
    // ---- lower half: planes 0, 1 (lattice 0..17) and the plane-2 corners
    T xa[18], c2[4];
#pragma unroll
    for (int p = 0; p < 18; ++p) xa[p] = xat(p);
#pragma unroll
    for (int k = 0; k < 4; ++k) c2[k] = xat(kC2[k]);
    auto xlow = [&](int q) -> T { return q < 18 ? xa[q] : c2[q == 18 ? 0 : q == 20 ? 1 : q == 24 ? 2 : 3]; };
#pragma unroll
    for (int p = 0; p < 18; ++p) {
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        if ((none >> p) & 1u) xa[p] = (xlow(p - s0) + xlow(p + s0)) * T(0.5);
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        if ((none >> p) & 1u)
          xa[p] = ((xlow(p - s0 - s1) + xlow(p + s0 - s1)) + (xlow(p - s0 + s1) + xlow(p + s0 + s1))) * T(0.25);
      }
    }
    T ya[18];
#pragma unroll
    for (int p = 0; p < 18; ++p) ya[p] = T(0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if ((cm >> c) & 1u) {
        T u[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) u[v] = xa[oct_lat(c, v)];
        child(c, u);
#pragma unroll
        for (int v = 0; v < 8; ++v) ya[oct_lat(c, v)] += u[v];
      }
    }
    // plane 0's hanging points fold onto plane-0 corners; its other node
    // sums leave now, its corners are kept for the folds of plane 1
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        const T w = ((none >> p) & 1u) ? ya[p] * T(0.5) : T(0);
        ya[p - s0] += w;
        ya[p + s0] += w;
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        const T w = ((none >> p) & 1u) ? ya[p] * T(0.25) : T(0);
        ya[p - s0 - s1] += w;
        ya[p + s0 - s1] += w;
        ya[p - s0 + s1] += w;
        ya[p + s0 + s1] += w;
      }
    }
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      if (oct_free(p) == 0) continue;  // corners: later
      const uint32_t id = sw[sl][p][tid];
      const bool node = id != kNoNode;
      red_add_if(y + (node ? id : 0u), ya[p], node && ya[p] != T(0));
    }
    T yc0[4] = {ya[0], ya[2], ya[6], ya[8]};
    // ---- upper half: planes 1, 2 (lattice 9..26)
    T xb[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int p = 18 + q;
      xb[q] = p == 18 ? c2[0] : p == 20 ? c2[1] : p == 24 ? c2[2] : p == 26 ? c2[3] : xat(p);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int p = 18 + q;
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        if ((none >> p) & 1u) xb[q] = (xb[q - s0] + xb[q + s0]) * T(0.5);
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        if ((none >> p) & 1u)
          xb[q] = ((xb[q - s0 - s1] + xb[q + s0 - s1]) + (xb[q - s0 + s1] + xb[q + s0 + s1])) * T(0.25);
      }
    }
    T yb[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) yb[q] = T(0);
#pragma unroll
    for (int c = 4; c < 8; ++c) {
      if ((cm >> c) & 1u) {
        T u[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int p = oct_lat(c, v);
          u[v] = p < 18 ? xa[p] : xb[p - 18];
        }
        child(c, u);
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int p = oct_lat(c, v);
          if (p < 18) ya[p] += u[v];
          else yb[p - 18] += u[v];
        }
      }
    }
    // folds of planes 1 and 2: a corner q is plane 0 (yc0), plane 2 (yb)
    auto addc = [&](int q, T w) {
      if (q < 9) yc0[q == 0 ? 0 : q == 2 ? 1 : q == 6 ? 2 : 3] += w;
      else if (q >= 18) yb[q - 18] += w;
      else ya[q] += w;
    };
#pragma unroll
    for (int p = 9; p < 27; ++p) {
      const T yp = p < 18 ? ya[p] : yb[p - 18];
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        const T w = ((none >> p) & 1u) ? yp * T(0.5) : T(0);
        addc(p - s0, w);
        addc(p + s0, w);
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        const T w = ((none >> p) & 1u) ? yp * T(0.25) : T(0);
        addc(p - s0 - s1, w);
        addc(p + s0 - s1, w);
        addc(p - s0 + s1, w);
        addc(p + s0 + s1, w);
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = k == 0 ? 0 : k == 1 ? 2 : k == 2 ? 6 : 8;
      const uint32_t id = sw[sl][p][tid];
      const bool node = id != kNoNode;
      red_add_if(y + (node ? id : 0u), yc0[k], node && yc0[k] != T(0));
    }
#pragma unroll
    for (int p = 9; p < 27; ++p) {
      const T yp = p < 18 ? ya[p] : yb[p - 18];
      const uint32_t id = sw[sl][p][tid];
      const bool node = id != kNoNode;
      T* dst = y + (node ? id : 0u);
      if (p == 13) {
        st_if(dst, yp, node && cm == 255u);
        red_add_if(dst, yp, node && cm != 255u);
      } else {
        red_add_if(dst, yp, node && yp != T(0));
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// The same with x in flight too: per thread the words of the octet two grid
// strides ahead and the x values (8- or 4-byte cp.async gathers) of the
// next one are copied while it works the current one, whose x is read from
// its shared slot; only the coefficients are read straight from global
// memory.  Shared memory per thread: 3 word slots + 2 value slots.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octet_pfx_kernel(
    int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
    const uint32_t* __restrict__ oelem, const CT* __restrict__ ca, const CT* __restrict__ cb,
    const T* __restrict__ x, T* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char pfx_smem[];
  uint32_t(*sw)[kOctPfWords][BLOCK] = reinterpret_cast<uint32_t(*)[kOctPfWords][BLOCK]>(pfx_smem);
  T(*sx)[27][BLOCK] = reinterpret_cast<T(*)[27][BLOCK]>(pfx_smem + sizeof(uint32_t) * 3 * kOctPfWords * BLOCK);
  const int tid = threadIdx.x;
  const int64_t stride = gstride();
  auto fetch_words = [&](int64_t oo, int slot) {
    if (oo < n) {
#pragma unroll
      for (int p = 0; p < 27; ++p)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                         static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][p][tid]))),
                     "l"(oid + int64_t(p) * n + oo)
                     : "memory");
      if (ca) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                           static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][27 + c][tid]))),
                       "l"(oelem + int64_t(c) * n + oo)
                       : "memory");
      }
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                       static_cast<uint32_t>(__cvta_generic_to_shared(&sw[slot][35][tid]))),
                   "l"(ometa + oo)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto fetch_x = [&](int64_t oo, int wslot, int xslot) {
    if (oo < n) {
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        const uint32_t id = sw[wslot][p][tid];
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(&sx[xslot][p][tid]));
        if (id != kNoNode) {
          if (sizeof(T) == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(x + id) : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(x + id) : "memory");
        } else {
          sx[xslot][p][tid] = T(0);
        }
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  int64_t o = gtid();
  fetch_words(o, 0);
  fetch_words(o + stride, 1);
  asm volatile("cp.async.wait_group 1;" ::: "memory");
  fetch_x(o, 0, 0);
  for (int it = 0; o < n; o += stride, ++it) {
    const int ws = it % 3, xs = it & 1;
    fetch_words(o + 2 * stride, (it + 2) % 3);
    asm volatile("cp.async.wait_group 2;" ::: "memory");  // words of the next octet
    fetch_x(o + stride, (it + 1) % 3, xs ^ 1);
    asm volatile("cp.async.wait_group 2;" ::: "memory");  // x of this octet
    const uint32_t m = sw[ws][35][tid];
    const uint32_t cm0 = ometa_cmask(m);
    T fa[8], fb[8];
    if (ca) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint32_t e = sw[ws][27 + c][tid];
        fa[c] = ((cm0 >> c) & 1u) ? T(__ldg(ca + e)) : T(0);
        fb[c] = ((cm0 >> c) & 1u) ? T(__ldg(cb + e)) : T(0);
      }
    }
    uint32_t none = 0;
    T xv[27], yv[27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      none |= sw[ws][p][tid] == kNoNode ? (1u << p) : 0u;
      xv[p] = sx[xs][p][tid];
    }
    octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
      if (ca) {
        f1 *= fa[c];
        f2 *= fb[c];
      }
    });
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = sw[ws][p][tid];
      const bool node = id != kNoNode;
      T* dst = y + (node ? id : 0u);
      if (p == 13) {
        st_if(dst, yv[p], node && cm0 == 255u);
        red_add_if(dst, yv[p], node && cm0 != 255u);
      } else {
        red_add_if(dst, yv[p], node && yv[p] != T(0));
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}
template <class T, int BLOCK>
constexpr size_t octet_pfx_smem() {
  return sizeof(uint32_t) * 3 * kOctPfWords * BLOCK + sizeof(T) * 2 * 27 * BLOCK;
}

// Octet form with a child per lane: the 8 lanes 8g .. 8g + 7 of a warp work
// the 8 children of one parent octant (4 octets per warp), lane c child c.
// A lane holds its child's 8 vertex values in the child's mirrored frame
// f = v ^ c, in which f_a = 0 is the parent's outer face on axis a and
// f_a = 1 the middle plane that child c shares with child c ^ (1 << a); the
// element operator is unchanged by the relabelling (its entries depend on
// popcount(v ^ w) only).  In that frame:
//  * vertex f is lattice point sum_a (c_a ? 2 - f_a : f_a) 3^a; a hanging
//    vertex reads x at its far corner, the parent corner f ^ c (the DA's
//    node for a hanging vertex), and takes the mean of the values at the
//    frame vertices j that are bit subsets of f (2 on an edge, 4 on a face:
//    the interpolation of the hanging-node stencils, handleType2Stencils.C);
//  * the lattice sums over the children sharing a point are a butterfly: on
//    axis a the 4 values with f_a = 1 are exchanged with lane c ^ (1 << a)
//    at the same frame index (one shuffle each), so after the three axes
//    every sharer holds the point's full sum;
//  * the transpose of the interpolation is local: a hanging point's sum
//    goes, times 1/2 (edge) or 1/4 (face), to frame vertex 0 (the parent
//    corner c) of every child at one of its corners, each of which holds the
//    point (a lane whose child is not an element of the mesh still holds it
//    after the butterfly, and adds its corner's sum);
//  * each node's sum leaves once, from the lowest-numbered present child
//    that shares it.
// The octet's record (octet.cuh, 128 bytes) gives the node ids, the mask of
// points without a node and the level; a lane keeps 8 values, 8 ids and its
// two scale factors, so many warps fit on an SM.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octlane_kernel(
    int64_t n, const uint32_t* __restrict__ orec, const uint32_t* __restrict__ oelem, const CT* __restrict__ ca,
    const CT* __restrict__ cb, const T* __restrict__ x, T* __restrict__ y) {
  const int lane = threadIdx.x & 31, c = lane & 7;
  const int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
  const int64_t nw = gstride() >> 5;
  for (int64_t ob = (gtid() >> 5) * 4; ob < n; ob += nw * 4) {
    const int64_t o = ob + (lane >> 3);
    const uint32_t* r = orec + (o < n ? o : n) * kOctRec;
    const uint32_t none = __ldg(r + 27), m = __ldg(r + 28);
    const uint32_t cm = ometa_cmask(m);
    const bool present = (cm >> c) & 1u;
    // lattice index of frame vertex f, and of the parent corner f ^ c
    const int base = 2 * (cx + 3 * cy + 9 * cz);
    const int dx = cx ? -1 : 1, dy = cy ? -3 : 3, dz = cz ? -9 : 9;
    uint32_t hang = 0;
    T u[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      const int L = base + (f & 1) * dx + ((f >> 1) & 1) * dy + (f >> 2) * dz;
      const int F = 2 * (((f ^ c) & 1) + 3 * (((f ^ c) >> 1) & 1) + 9 * ((f ^ c) >> 2));
      const bool h = (f != 0 && f != 7) && ((none >> L) & 1u);
      hang |= h ? (1u << f) : 0u;
      const uint32_t id = present ? __ldg(r + (h ? F : L)) : kNoNode;
      u[f] = id != kNoNode ? __ldg(x + id) : T(0);
    }
    T f1 = T(0), f2 = T(0);
    if (present) {
      const T hh = elem_h<T>(ometa_lev(m));
      f1 = hh * T(0.5);
      f2 = hh * hh * hh * T(0.125);
      if (ca) {
        const uint32_t e = __ldg(oelem + int64_t(c) * n + o);
        f1 *= T(__ldg(ca + e));
        f2 *= T(__ldg(cb + e));
      }
    }
    // hanging vertices from the raw values: faces first (they read the raw
    // edge values), then edges
#pragma unroll
    for (int f = 3; f < 7; ++f) {
      if (f == 4) continue;
      const int b0 = f & -f, b1 = f ^ b0;
      if ((hang >> f) & 1u) u[f] = ((u[0] + u[f]) + (u[b0] + u[b1])) * T(0.25);
    }
#pragma unroll
    for (int f = 1; f <= 4; f <<= 1)
      if ((hang >> f) & 1u) u[f] = (u[0] + u[f]) * T(0.5);
    lapmass_ref(u, f1, f2);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int f = 0; f < 8; ++f)
        if ((f >> a) & 1) u[f] += __shfl_xor_sync(0xffffffffu, u[f], 1 << a);
    T fold = T(0);
#pragma unroll
    for (int f = 1; f < 7; ++f) {
      const T w = (f == 1 || f == 2 || f == 4) ? T(0.5) : T(0.25);
      fold += ((hang >> f) & 1u) ? u[f] * w : T(0);
    }
    u[0] += fold;
    // sharers of frame vertex f: c with the bits of f replaced by any
    // subset; the node ids are read again from the record (L1) so that they
    // do not occupy registers during the arithmetic
#pragma unroll
    for (int f = 0; f < 8; ++f) {
      uint32_t subsets = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if ((q & ~f) == 0) subsets |= 1u << q;
      const uint32_t ps = (subsets << (c & ~f)) & cm;
      // f = 0 (the parent corner c) belongs to this lane alone; it may hold
      // folded sums even when child c is not an element of this mesh (an
      // element subset of a partitioned mesh leaves children out)
      const bool mine = (present || (f == 0 && u[0] != T(0))) && !((hang >> f) & 1u) &&
                        (ps & ((1u << c) - 1u)) == 0u;
      const int L = base + (f & 1) * dx + ((f >> 1) & 1) * dy + (f >> 2) * dz;
      const uint32_t id = mine ? __ldg(r + L) : kNoNode;
      const bool owner = id != kNoNode;
      T* dst = y + (owner ? id : 0u);
      if (f == 7) {
        st_if(dst, u[f], owner && cm == 255u);
        red_add_if(dst, u[f], owner && cm != 255u);
      } else {
        red_add_if(dst, u[f], owner);
      }
    }
  }
}

// Octet form with a column of two children per lane: the 4 lanes 4g .. 4g + 3
// of a warp work one parent octant (8 octets per warp); lane q = (qx, qy)
// holds the two children c = q (lower half, z bit 0) and c = q + 4 (upper),
// i.e. the 12 lattice points with x in {qx, qx + 1}, y in {qy, qy + 1} and
// z in {0, 1, 2}.  Lane point i = fx + 2 fy + 4 z, mirrored on x and y
// (lattice coordinate qx ? 2 - fx : fx, the same for y), so that fx = 1 /
// fy = 1 are the planes shared with lane q ^ 1 / q ^ 2 and z = 1 the plane the
// lane's two children share.  Per octet a lane
//  * reads x at its 12 points, a hanging point (no node in the record) as the
//    mean of its 2 or 4 parent corners (the interpolation T of the
//    hanging-node stencils, handleType2Stencils.C);
//  * applies the two children's element operators (points 0..7 and 4..11;
//    the operator is unchanged by the mirroring) and adds their results;
//  * sums the shared planes with the neighbour lanes (one shuffle per value
//    on x, one on y): every sharer then holds the full lattice sum;
//  * folds each hanging point's sum, times 1/2 (edge) or 1/4 (face), onto
//    its corners in the lane's own range (every lane holding one of the
//    corners also holds the point);
//  * adds each node's sum into y once, from the sharer with qx = 0 / qy = 0 on
//    the shared axes.
// A lane keeps 12 values, so the kernel runs at twice the warps per SM of
// the one-thread-per-octet form with about the same instructions per element.
template <class T, class CT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_octquad_kernel(
    int64_t n, const uint32_t* __restrict__ orec, const uint32_t* __restrict__ oelem, const CT* __restrict__ ca,
    const CT* __restrict__ cb, const T* __restrict__ x, T* __restrict__ y) {
  const int lane = threadIdx.x & 31, q = lane & 3, qx = q & 1, qy = q >> 1;
  const int base = (qx ? 2 : 0) + (qy ? 6 : 0), sx = qx ? -1 : 1, sy = qy ? -3 : 3;
  const int64_t nw = gstride() >> 5;
  for (int64_t ob = (gtid() >> 5) * 8; ob < n; ob += nw * 8) {
    const int64_t o = ob + (lane >> 2);
    const uint32_t* r = orec + (o < n ? o : n) * kOctRec;
    const uint32_t none = __ldg(r + 27), m = __ldg(r + 28);
    const uint32_t cm = ometa_cmask(m);
    uint32_t hang = 0;
    T u[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const int L = base + sx * (i & 1) + sy * ((i >> 1) & 1) + 9 * (i >> 2);
      const bool h = (none >> L) & 1u;
      hang |= h ? (1u << i) : 0u;
      const uint32_t id = h ? kNoNode : __ldg(r + L);
      u[i] = id != kNoNode ? __ldg(x + id) : T(0);
    }
    if (hang) {
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int fx = i & 1, fy = (i >> 1) & 1, z = i >> 2;
        const int nf = fx + fy + (z == 1);
        if (nf == 0 || nf == 3 || !((hang >> i) & 1u)) continue;
        const int L = base + sx * fx + sy * fy + 9 * z;
        // corners: L -/+ the lattice stride of each free axis (1, 3, 9); a
        // point that no present child has may have corners without nodes
        const int s0 = fx ? 1 : fy ? 3 : 9;
        const int s1 = nf == 2 ? ((fx && fy) ? 3 : 9) : 0;
        auto xat = [&](int Lc) {
          const uint32_t id = __ldg(r + Lc);
          return id != kNoNode ? __ldg(x + id) : T(0);
        };
        if (nf == 1) u[i] = (xat(L - s0) + xat(L + s0)) * T(0.5);
        else u[i] = ((xat(L - s0 - s1) + xat(L + s0 - s1)) + (xat(L - s0 + s1) + xat(L + s0 + s1))) * T(0.25);
      }
    }
    T f1[2] = {T(0), T(0)}, f2[2] = {T(0), T(0)};
    const T hh = elem_h<T>(ometa_lev(m));
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = q + 4 * k;
      if ((cm >> c) & 1u) {
        f1[k] = hh * T(0.5);
        f2[k] = hh * hh * hh * T(0.125);
        if (ca) {
          const uint32_t e = __ldg(oelem + int64_t(c) * n + o);
          f1[k] *= T(__ldg(ca + e));
          f2[k] *= T(__ldg(cb + e));
        }
      }
    }
    T lo[8], up[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      lo[v] = u[v];
      up[v] = u[v + 4];
    }
    lapmass_ref(lo, f1[0], f2[0]);
    lapmass_ref(up, f1[1], f2[1]);
#pragma unroll
    for (int i = 0; i < 12; ++i) u[i] = (i < 8 ? lo[i] : T(0)) + (i >= 4 ? up[i - 4] : T(0));
#pragma unroll
    for (int i = 0; i < 12; ++i)
      if (i & 1) u[i] += __shfl_xor_sync(0xffffffffu, u[i], 1);
#pragma unroll
    for (int i = 0; i < 12; ++i)
      if (i & 2) u[i] += __shfl_xor_sync(0xffffffffu, u[i], 2);
    if (hang) {
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int fx = i & 1, fy = (i >> 1) & 1, z = i >> 2;
        const int nf = fx + fy + (z == 1);
        if (nf == 0 || nf == 3) continue;
        const T w = ((hang >> i) & 1u) ? u[i] * (nf == 1 ? T(0.5) : T(0.25)) : T(0);
        // its corners in this lane's range are the parent corners of the
        // lane's column, points 0 (z = 0) and 8 (z = 2)
        if (z != 2) u[0] += w;
        if (z != 0) u[8] += w;
      }
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const bool mine = (!(i & 1) || !qx) && (!(i & 2) || !qy) && !((hang >> i) & 1u);
      const int L = base + sx * (i & 1) + sy * ((i >> 1) & 1) + 9 * (i >> 2);
      const uint32_t id = mine ? __ldg(r + L) : kNoNode;
      const bool go = id != kNoNode && u[i] != T(0);
      T* dst = y + (go ? id : 0u);
      if (i == 7) {  // the parent's centre: only this octet's children touch it when all 8 are leaves
        st_if(dst, u[i], go && cm == 255u);
        red_add_if(dst, u[i], go && cm != 255u);
      } else {
        red_add_if(dst, u[i], go);
      }
    }
  }
}

constexpr int kStageBatch = 8;  // node values each thread has in flight while staging a chunk

// Chunked octet kernel: a CTA of kOctChunk threads per chunk of kOctChunk
// consecutive octets (OctetSet chunks).  x at the chunk's nodes (ascending
// ids: mostly contiguous runs) and the coefficients of the chunk's element
// range are staged in shared memory with coalesced loads; every thread works
// its octet from shared memory and adds its 27 lattice sums into the chunk's
// shared accumulator (shared-memory atomics: octets of one chunk share
// nodes); then the chunk's sums leave with coalesced stores (nodes no other
// chunk touches) or global reductions.  Chunks whose element range exceeds
// the staged coefficient window read their coefficients from global memory.
template <class T, class CT, int MINB>
__global__ void __launch_bounds__(kOctChunk, MINB) lapmass_octchunk_kernel(
    int64_t n, int64_t nchunk, uint32_t node_cap, uint32_t coef_cap, const uint32_t* __restrict__ ometa,
    const uint16_t* __restrict__ lidx, const uint16_t* __restrict__ lelem, const uint32_t* __restrict__ cptr,
    const uint32_t* __restrict__ cnodes, const uint32_t* __restrict__ cel, const CT* __restrict__ ca,
    const CT* __restrict__ cb, const T* __restrict__ x, T* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char oc_smem[];
  T* sx = reinterpret_cast<T*>(oc_smem);
  T* sy = sx + node_cap;
  T* sa = sy + node_cap;
  T* sb = sa + coef_cap;
  for (int64_t q = blockIdx.x; q < nchunk; q += gridDim.x) {
    const uint32_t p0 = __ldg(cptr + q), nn = __ldg(cptr + q + 1) - p0;
    const uint32_t e0 = __ldg(cel + 2 * q), ne = __ldg(cel + 2 * q + 1);
    const bool staged = ca && ne <= coef_cap;
    // staging in batches of kStageBatch per thread: the node ids of a batch,
    // then their x values, each batch's loads independent of one another
    for (uint32_t k0 = threadIdx.x; k0 < nn; k0 += kStageBatch * kOctChunk) {
      uint32_t id[kStageBatch];
      T v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        id[u] = k < nn ? (__ldg(cnodes + p0 + k) & 0x7fffffffu) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        v[u] = k < nn ? __ldg(x + id[u]) : T(0);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        if (k < nn) {
          sx[k] = v[u];
          sy[k] = T(0);
        }
      }
    }
    if (staged)
      for (uint32_t k0 = threadIdx.x; k0 < ne; k0 += kStageBatch * kOctChunk) {
        T a[kStageBatch], b[kStageBatch];
#pragma unroll
        for (int u = 0; u < kStageBatch; ++u) {
          const uint32_t k = k0 + u * kOctChunk;
          a[u] = k < ne ? T(__ldg(ca + e0 + k)) : T(0);
          b[u] = k < ne ? T(__ldg(cb + e0 + k)) : T(0);
        }
#pragma unroll
        for (int u = 0; u < kStageBatch; ++u) {
          const uint32_t k = k0 + u * kOctChunk;
          if (k < ne) {
            sa[k] = a[u];
            sb[k] = b[u];
          }
        }
      }
    __syncthreads();
    const int64_t o = q * kOctChunk + threadIdx.x;
    if (o < n) {
      const uint32_t m = __ldg(ometa + o);
      uint32_t none = 0;
      uint16_t li[27];
      T xv[27], yv[27];
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        li[p] = __ldg(lidx + int64_t(p) * n + o);
        none |= li[p] == 0xffffu ? (1u << p) : 0u;
      }
      uint32_t le[8];
      if (ca) {
        const uint32_t cm = ometa_cmask(m);
#pragma unroll
        for (int c = 0; c < 8; ++c) le[c] = ((cm >> c) & 1u) ? __ldg(lelem + int64_t(c) * n + o) : 0u;
      }
#pragma unroll
      for (int p = 0; p < 27; ++p) xv[p] = li[p] != 0xffffu ? sx[li[p]] : T(0);
      octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
        if (ca) {
          if (staged) {
            f1 *= sa[le[c]];
            f2 *= sb[le[c]];
          } else {
            f1 *= T(__ldg(ca + e0 + le[c]));
            f2 *= T(__ldg(cb + e0 + le[c]));
          }
        }
      });
#pragma unroll
      for (int p = 0; p < 27; ++p)
        if (li[p] != 0xffffu && yv[p] != T(0)) atomicAdd(sy + li[p], yv[p]);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nn; k += kOctChunk) {
      const uint32_t id = __ldg(cnodes + p0 + k);
      T* dst = y + (id & 0x7fffffffu);
      const T v = sy[k];
      st_if(dst, v, !(id >> 31));
      red_add_if(dst, v, (id >> 31) && v != T(0));
    }
    __syncthreads();  // the buffers are reused by the next chunk
  }
}

// Lean chunked octet kernel: the same staging and flush as
// lapmass_octchunk_kernel, but no 27-value register arrays -- each child's 8
// vertex values are read from the staged x on demand (a hanging point as the
// mean of its corners), and the child's 8 results go straight into the
// chunk's shared accumulator (a hanging point's share onto its corners), so
// a thread holds only the 27 local indices and one element: far fewer
// registers and more resident chunks per SM, for 64 shared-memory atomics per
// complete octet instead of 27.
template <class T>
__device__ __forceinline__ T lean_value(const T* sx, const uint16_t (&li)[27], int p) {
  if (oct_free(p) == 1) {
    const int s0 = oct_s0(p);
    if (li[p] == 0xffffu) return (sx[li[p - s0]] + sx[li[p + s0]]) * T(0.5);
  } else if (oct_free(p) == 2) {
    const int s0 = oct_s0(p), s1 = oct_s1(p);
    if (li[p] == 0xffffu)
      return ((sx[li[p - s0 - s1]] + sx[li[p + s0 - s1]]) + (sx[li[p - s0 + s1]] + sx[li[p + s0 + s1]])) * T(0.25);
  }
  return sx[li[p]];
}
template <class T>
__device__ __forceinline__ void lean_add(T* sy, const uint16_t (&li)[27], int p, T v) {
  if (oct_free(p) == 1) {
    const int s0 = oct_s0(p);
    if (li[p] == 0xffffu) {
      const T w = v * T(0.5);
      atomicAdd(sy + li[p - s0], w);
      atomicAdd(sy + li[p + s0], w);
      return;
    }
  } else if (oct_free(p) == 2) {
    const int s0 = oct_s0(p), s1 = oct_s1(p);
    if (li[p] == 0xffffu) {
      const T w = v * T(0.25);
      atomicAdd(sy + li[p - s0 - s1], w);
      atomicAdd(sy + li[p + s0 - s1], w);
      atomicAdd(sy + li[p - s0 + s1], w);
      atomicAdd(sy + li[p + s0 + s1], w);
      return;
    }
  }
  atomicAdd(sy + li[p], v);
}

template <class T, class CT, int MINB>
__global__ void __launch_bounds__(kOctChunk, MINB) lapmass_octchunk_lean_kernel(
    int64_t n, int64_t nchunk, uint32_t node_cap, const uint32_t* __restrict__ ometa,
    const uint16_t* __restrict__ lidx, const uint16_t* __restrict__ lelem, const uint32_t* __restrict__ cptr,
    const uint32_t* __restrict__ cnodes, const uint32_t* __restrict__ cel, const CT* __restrict__ ca,
    const CT* __restrict__ cb, const T* __restrict__ x, T* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char oc_smem[];
  T* sx = reinterpret_cast<T*>(oc_smem);
  T* sy = sx + node_cap;
  for (int64_t q = blockIdx.x; q < nchunk; q += gridDim.x) {
    const uint32_t p0 = __ldg(cptr + q), nn = __ldg(cptr + q + 1) - p0;
    const uint32_t e0 = __ldg(cel + 2 * q);
    const int64_t o = q * kOctChunk + threadIdx.x;
    // this thread's octet records, issued before the staging so that their
    // latency overlaps it
    uint32_t m = 0;
    uint16_t li[27];
    if (o < n) {
      m = __ldg(ometa + o);
#pragma unroll
      for (int p = 0; p < 27; ++p) li[p] = __ldg(lidx + int64_t(p) * n + o);
    }
    for (uint32_t k0 = threadIdx.x; k0 < nn; k0 += kStageBatch * kOctChunk) {
      uint32_t id[kStageBatch];
      T v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        id[u] = k < nn ? (__ldg(cnodes + p0 + k) & 0x7fffffffu) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        v[u] = k < nn ? __ldg(x + id[u]) : T(0);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const uint32_t k = k0 + u * kOctChunk;
        if (k < nn) {
          sx[k] = v[u];
          sy[k] = T(0);
        }
      }
    }
    __syncthreads();
    if (o < n) {
      const uint32_t cm = ometa_cmask(m);
      const T h = elem_h<T>(ometa_lev(m));
      const T g1 = h * T(0.5), g2 = h * h * h * T(0.125);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if ((cm >> c) & 1u) {
          T f1 = g1, f2 = g2;
          if (ca) {  // used once per element: read through L1, not staged
            const uint32_t le = __ldg(lelem + int64_t(c) * n + o);
            f1 *= T(__ldg(ca + e0 + le));
            f2 *= T(__ldg(cb + e0 + le));
          }
          T u[8];
#pragma unroll
          for (int v = 0; v < 8; ++v) u[v] = lean_value<T>(sx, li, oct_lat(c, v));
          lapmass_ref(u, f1, f2);
#pragma unroll
          for (int v = 0; v < 8; ++v) lean_add<T>(sy, li, oct_lat(c, v), u[v]);
        }
      }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nn; k += kOctChunk) {
      const uint32_t id = __ldg(cnodes + p0 + k);
      T* dst = y + (id & 0x7fffffffu);
      const T v = sy[k];
      st_if(dst, v, !(id >> 31));
      red_add_if(dst, v, (id >> 31) && v != T(0));
    }
    __syncthreads();
  }
}

// Pipelined chunked octet kernel: the chunked kernel with its staging moved
// off the critical path.  A CTA walks its chunks i = 0, 1, 2, ... (chunk
// blockIdx.x + i gridDim.x); while it works chunk i, the x gathers of chunk
// i + 1 (cp.async, 4 or 8 bytes each, from the node ids already in shared
// memory) and the node ids of chunk i + 2 (cp.async) are in flight.  Shared
// memory: node ids in three slots (i: flush, i + 1: gathering, i + 2:
// arriving), x in two, the accumulator in one.  Coefficients are read
// through L1 (each is used once).
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <class T>
__device__ __forceinline__ void octchunk_issue_ids(uint32_t* ib, const uint32_t* __restrict__ cnodes, uint32_t p0,
                                                   uint32_t nn) {
  for (uint32_t k = threadIdx.x; k < nn; k += kOctChunk) cp_async4(ib + k, cnodes + p0 + k);
}
template <class T>
__device__ __forceinline__ void octchunk_issue_x(T* xb, const uint32_t* ib, const T* __restrict__ x, uint32_t nn) {
  for (uint32_t k = threadIdx.x; k < nn; k += kOctChunk) {
    const T* src = x + (ib[k] & 0x7fffffffu);
    if constexpr (sizeof(T) == 8) cp_async8(xb + k, src);
    else cp_async4(xb + k, src);
  }
}

template <class T, class CT, int MINB>
__global__ void __launch_bounds__(kOctChunk, MINB) lapmass_octchunk_pipe_kernel(
    int64_t n, int64_t nchunk, uint32_t node_cap, const uint32_t* __restrict__ ometa,
    const uint16_t* __restrict__ lidx, const uint16_t* __restrict__ lelem, const uint32_t* __restrict__ cptr,
    const uint32_t* __restrict__ cnodes, const uint32_t* __restrict__ cel, const CT* __restrict__ ca,
    const CT* __restrict__ cb, const T* __restrict__ x, T* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char oc_smem[];
  T* xb0 = reinterpret_cast<T*>(oc_smem);
  T* xb1 = xb0 + node_cap;
  T* sy = xb1 + node_cap;
  uint32_t* ib0 = reinterpret_cast<uint32_t*>(sy + node_cap);
  uint32_t* ib1 = ib0 + node_cap;
  uint32_t* ib2 = ib1 + node_cap;
  const int64_t G = gridDim.x;
  int64_t q = blockIdx.x;
  if (q >= nchunk) return;
  // prologue: ids of chunks 0 and 1, then x of chunk 0
  {
    const uint32_t a0 = __ldg(cptr + q), a1 = __ldg(cptr + q + 1);
    octchunk_issue_ids<T>(ib0, cnodes, a0, a1 - a0);
    if (q + G < nchunk) {
      const uint32_t b0 = __ldg(cptr + q + G), b1 = __ldg(cptr + q + G + 1);
      octchunk_issue_ids<T>(ib1, cnodes, b0, b1 - b0);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    octchunk_issue_x<T>(xb0, ib0, x, a1 - a0);
    cp_async_commit();
    for (uint32_t k = threadIdx.x; k < node_cap; k += kOctChunk) sy[k] = T(0);
    cp_async_wait_all();
    __syncthreads();
  }
  for (int i = 0; q < nchunk; ++i, q += G) {
    T* xc = (i & 1) ? xb1 : xb0;
    T* xn = (i & 1) ? xb0 : xb1;
    uint32_t* ic = (i % 3 == 0) ? ib0 : (i % 3 == 1) ? ib1 : ib2;  // chunk i
    uint32_t* in1 = (i % 3 == 0) ? ib1 : (i % 3 == 1) ? ib2 : ib0;  // chunk i + 1
    uint32_t* in2 = (i % 3 == 0) ? ib2 : (i % 3 == 1) ? ib0 : ib1;  // chunk i + 2
    const uint32_t p0 = __ldg(cptr + q), nn = __ldg(cptr + q + 1) - p0;
    const uint32_t e0 = __ldg(cel + 2 * q);
    // 1. in flight during this chunk: x of chunk i + 1, ids of chunk i + 2
    if (q + G < nchunk) {
      const uint32_t c0 = __ldg(cptr + q + G), c1 = __ldg(cptr + q + G + 1);
      octchunk_issue_x<T>(xn, in1, x, c1 - c0);
    }
    if (q + 2 * G < nchunk) {
      const uint32_t d0 = __ldg(cptr + q + 2 * G), d1 = __ldg(cptr + q + 2 * G + 1);
      octchunk_issue_ids<T>(in2, cnodes, d0, d1 - d0);
    }
    cp_async_commit();
    // 2. this chunk's octets
    const int64_t o = q * kOctChunk + threadIdx.x;
    if (o < n) {
      const uint32_t m = __ldg(ometa + o);
      uint32_t none = 0;
      uint16_t li[27];
      T xv[27], yv[27];
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        li[p] = __ldg(lidx + int64_t(p) * n + o);
        none |= li[p] == 0xffffu ? (1u << p) : 0u;
      }
      // the children's coefficients, all issued before the arithmetic (a
      // load inside the predicated child loop would expose its round trip
      // once per child)
      T fa[8], fb[8];
      if (ca) {
        const uint32_t cm = ometa_cmask(m);
        uint32_t le[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) le[c] = ((cm >> c) & 1u) ? __ldg(lelem + int64_t(c) * n + o) : 0u;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          fa[c] = ((cm >> c) & 1u) ? T(__ldg(ca + e0 + le[c])) : T(0);
          fb[c] = ((cm >> c) & 1u) ? T(__ldg(cb + e0 + le[c])) : T(0);
        }
      }
#pragma unroll
      for (int p = 0; p < 27; ++p) xv[p] = li[p] != 0xffffu ? xc[li[p]] : T(0);
      octet_apply<T>(xv, yv, none, m, [&](int c, T& f1, T& f2) {
        if (ca) {
          f1 *= fa[c];
          f2 *= fb[c];
        }
      });
#pragma unroll
      for (int p = 0; p < 27; ++p)
        if (li[p] != 0xffffu && yv[p] != T(0)) atomicAdd(sy + li[p], yv[p]);
    }
    __syncthreads();
    // 3. this chunk's sums leave; the accumulator is zeroed for the next
    for (uint32_t k = threadIdx.x; k < nn; k += kOctChunk) {
      const uint32_t id = ic[k];
      T* dst = y + (id & 0x7fffffffu);
      const T v = sy[k];
      sy[k] = T(0);
      st_if(dst, v, !(id >> 31));
      red_add_if(dst, v, (id >> 31) && v != T(0));
    }
    // 4. the next chunk's x and the ids after it have landed
    cp_async_wait_all();
    __syncthreads();
  }
}

// ---------------------------------------------------- bulk-copy staging --
// The warp-tile operator with its tile records staged by the copy engine:
// one lane per warp issues cp.async.bulk copies of a tile's contiguous
// records (sorted references, frame ranks, element words, coefficients and
// the window of its node ids) into the warp's shared memory, completing on an
// mbarrier; two stages per warp, tile t + 2 issued as soon as tile t has been
// summed, x at the next tile's nodes gathered into registers as soon as its
// stage has landed.  The records never occupy registers in flight and the
// lanes issue no global loads for them.
//
// Every copy starts on a 16-byte boundary: per-tile offsets of the reference
// lists (kWarpRefBytes), ranks (256 B), element words (128 B) and first
// coefficients (32 per tile) are multiples of 16; the second coefficient
// array and the node list are copied from the 16-byte boundary at or below
// their start (lead-in skipped when read), and the arrays carry slack so
// that whole-tile windows stay inside their allocations.
//
// Waits are bounded: lane 0 polls the stage's mbarrier until a clock64
// deadline; past it the warp records DG_ETIMEOUT in a device status word,
// waits (bounded again) for its copies still in flight, and returns.
constexpr int kTmaWarps = 4;  // warps per CTA
constexpr long long kDefaultWaitLimit = 1ll << 31;  // clock64 cycles, about a second
static long long g_wait_limit = kDefaultWaitLimit;

__device__ int g_wait_status;  // DG_ETIMEOUT once a bounded wait has run out
// Set when, after such a timeout, the bounded wait for the warp's copies
// still in flight ran out as well: the warp returned with copies pending, so
// they may have landed in shared memory that a later block already owned.
__device__ int g_drain_gave_up;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

template <class CT>
struct alignas(16) TmaStage {
  uint8_t ref[kWarpRefBytes];                 // sorted frame positions, their node ranks, flag words
  uint2 eloc[kWarpTile];                      // per element the ranks of its frame vertices
  uint32_t wm[kWarpTile];                     // per element level | frame hanging mask << 8
  CT ca[kWarpTile];                           // first coefficient
  CT cb[kWarpTile + 16 / sizeof(CT)];         // second coefficient, from the 16-byte boundary below
  uint32_t nodes[8 * kWarpTile + kNodePad];   // node ids, from the 16-byte boundary below
};
template <class T, class CT>
struct alignas(16) TmaWarp {
  TmaStage<CT> st[2];
  T sx[8 * kWarpTile];  // x at the tile's nodes by rank, then element results by frame position
  uint64_t bar[2];
  uint32_t info[2][4];  // per stage: node count, node lead-in, second-coefficient lead-in
};
static_assert(sizeof(TmaStage<double>) % 16 == 0 && sizeof(TmaStage<float>) % 16 == 0, "stage alignment");
static_assert(offsetof(TmaStage<double>, cb) % 16 == 0 && offsetof(TmaStage<double>, nodes) % 16 == 0, "fields");
static_assert(offsetof(TmaStage<float>, cb) % 16 == 0 && offsetof(TmaStage<float>, nodes) % 16 == 0, "fields");

// Lane 0: copy tile tt's records into stage st (p0, p1: its node list offsets).
template <class T, class CT>
__device__ __forceinline__ void tma_issue(TmaWarp<T, CT>& W, int st, int64_t tt, uint32_t p0, uint32_t p1,
                                          const CT* ca, const CT* cb, const uint32_t* tile_nodes,
                                          const uint2* eloc8, const uint32_t* wmeta, const uint8_t* ref8) {
  TmaStage<CT>& S = W.st[st];
  const uint32_t n0 = p0 & ~3u;
  const uint32_t nbytes = ((p1 - n0 + 3u) & ~3u) * 4u;
  uint32_t total = kWarpRefBytes + 8 * kWarpTile + 4 * kWarpTile + nbytes;
  uintptr_t cb0 = 0;
  uint32_t cbbytes = 0, cblead = 0;
  if (ca) {
    const uintptr_t cbs = reinterpret_cast<uintptr_t>(cb + tt * kWarpTile);
    cb0 = cbs & ~uintptr_t(15);
    cblead = uint32_t(cbs - cb0) / sizeof(CT);
    cbbytes = (uint32_t(cbs - cb0) + kWarpTile * sizeof(CT) + 15u) & ~15u;
    total += kWarpTile * sizeof(CT) + cbbytes;
  }
  W.info[st][0] = p1 - p0;
  W.info[st][1] = p0 - n0;
  W.info[st][2] = cblead;
  mbar_expect_tx(&W.bar[st], total);
  bulk_g2s(S.ref, ref8 + tt * kWarpRefBytes, kWarpRefBytes, &W.bar[st]);
  bulk_g2s(S.eloc, eloc8 + tt * kWarpTile, 8 * kWarpTile, &W.bar[st]);
  bulk_g2s(S.wm, wmeta + tt * kWarpTile, 4 * kWarpTile, &W.bar[st]);
  if (ca) {
    bulk_g2s(S.ca, ca + tt * kWarpTile, kWarpTile * sizeof(CT), &W.bar[st]);
    bulk_g2s(S.cb, reinterpret_cast<const void*>(cb0), cbbytes, &W.bar[st]);
  }
  bulk_g2s(S.nodes, tile_nodes + n0, nbytes, &W.bar[st]);
}

// Warp-uniform bounded wait for the phase `parity` of bar.  try_wait
// suspends the warp in hardware until the phase completes or a short
// hardware limit passes; every lane sees the completed phase itself (its own
// acquire of the staged data) before the warp goes on, and the warp gives up
// together once lane clocks pass `limit` cycles.
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool tma_wait(uint64_t* bar, uint32_t parity, int /*lane*/, long long limit) {
  const long long t0 = clock64();
  while (true) {
    if (__any_sync(0xffffffffu, clock64() - t0 > limit)) return false;
    const bool done = mbar_try(bar, parity);
    if (__all_sync(0xffffffffu, done)) return true;
  }
}

template <class T, class CT, int MINB>
__global__ void __launch_bounds__(32 * kTmaWarps, MINB) lapmass_warp_tma_kernel(
    const uint32_t* __restrict__ wmeta, const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
    int64_t ntiles, const uint32_t* __restrict__ tile_ptr, const uint32_t* __restrict__ tile_nodes,
    const uint2* __restrict__ eloc8, const uint8_t* __restrict__ ref8, const T* __restrict__ x, T* __restrict__ y,
    long long wait_limit) {
  extern __shared__ __align__(16) unsigned char tma_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  TmaWarp<T, CT>& W = reinterpret_cast<TmaWarp<T, CT>*>(tma_smem)[w];
  const int64_t nw = int64_t(gridDim.x) * kTmaWarps;
  int64_t t = blockIdx.x * int64_t(kTmaWarps) + w;
  if (t >= ntiles) return;
  if (lane == 0) {
    mbar_init(&W.bar[0], 1);
    mbar_init(&W.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncwarp();
  // lane 0 keeps the node-list offsets of the tile after next (read early)
  uint32_t q0 = 0, q1 = 0;
  bool pend0 = false, pend1 = false;  // stage has copies not yet waited for
  if (lane == 0) {
    tma_issue(W, 0, t, __ldg(tile_ptr + t), __ldg(tile_ptr + t + 1), ca, cb, tile_nodes, eloc8, wmeta, ref8);
    pend0 = true;
    if (t + nw < ntiles) {
      tma_issue(W, 1, t + nw, __ldg(tile_ptr + t + nw), __ldg(tile_ptr + t + nw + 1), ca, cb, tile_nodes, eloc8,
                wmeta, ref8);
      pend1 = true;
    }
    if (t + 2 * nw < ntiles) {
      q0 = __ldg(tile_ptr + t + 2 * nw);
      q1 = __ldg(tile_ptr + t + 2 * nw + 1);
    }
  }
  __syncwarp();  // lane 0's stage info words are visible to the warp
  uint32_t par0 = 0, par1 = 0;
  bool failed = !tma_wait(&W.bar[0], par0, lane, wait_limit);
  if (!failed) {
    pend0 = false;
    par0 ^= 1u;
  }
  T xc[kPipeIds];
  if (!failed) {
    const uint32_t nt = W.info[0][0], nl = W.info[0][1];
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      xc[j] = k < nt ? __ldg(x + (W.st[0].nodes[nl + k] & 0x7fffffffu)) : T(0);
    }
  }
  int st = 0;
  for (; !failed && t < ntiles; t += nw, st ^= 1) {
    TmaStage<CT>& S = W.st[st];
    T* sx = W.sx;
    const uint32_t nt = W.info[st][0], nl = W.info[st][1], cbl = W.info[st][2];
    const uint32_t* sn = S.nodes + nl;
#pragma unroll
    for (int j = 0; j < kPipeIds; ++j) {
      const uint32_t k = lane + 32 * j;
      if (k < nt) sx[k] = xc[j];
    }
    for (uint32_t k = lane + 32 * kPipeIds; k < nt; k += 32) sx[k] = __ldg(x + (sn[k] & 0x7fffffffu));
    __syncwarp();
    const bool live = t * kWarpTile + lane < E;
    T wv[8];
    if (live) {
      const uint32_t m = S.wm[lane];
      const uint2 L = S.eloc[lane];
      const T a = ca ? T(S.ca[lane]) : T(1), b = ca ? T(S.cb[cbl + lane]) : T(1);
      const T h = elem_h<T>(meta_lev(m));
      const T f1 = a * h * T(0.5), f2 = b * h * h * h * T(0.125);
#pragma unroll
      for (int j = 0; j < 8; ++j) wv[j] = sx[byte_of(L, j)];
      const uint32_t mp = wmeta_mask(m);
      if (mp) interp_frame(wv, mp);
      lapmass_ref(wv, f1, f2);
      if (mp) scatter_frame(wv, mp);
    }
    // x at the next tile's nodes, once its stage has landed
    const bool has_next = t + nw < ntiles;
    if (has_next) {
      uint64_t* nb = &W.bar[st ^ 1];
      if (!tma_wait(nb, st ? par0 : par1, lane, wait_limit)) {
        failed = true;
      } else {
        if (st) {
          pend0 = false;
          par0 ^= 1u;
        } else {
          pend1 = false;
          par1 ^= 1u;
        }
        const uint32_t nt2 = W.info[st ^ 1][0], nl2 = W.info[st ^ 1][1];
        const uint32_t* sn2 = W.st[st ^ 1].nodes + nl2;
#pragma unroll
        for (int j = 0; j < kPipeIds; ++j) {
          const uint32_t k = lane + 32 * j;
          xc[j] = k < nt2 ? __ldg(x + (sn2[k] & 0x7fffffffu)) : T(0);
        }
      }
    }
    __syncwarp();  // every lane has read x: the buffer now takes the results
    if (live) {
#pragma unroll
      for (int j = 0; j < 8; ++j) sx[j * kWarpTile + lane] = wv[j];
    }
    __syncwarp();
    const uint2 pp = reinterpret_cast<const uint2*>(S.ref)[lane];
    const uint2 rr = reinterpret_cast<const uint2*>(S.ref + 8 * kWarpTile)[lane];
    const uint32_t ff = reinterpret_cast<const uint32_t*>(S.ref + 16 * kWarpTile)[lane];
    warp_seg_sum(sx, sn, pp, rr, ff, y);
    __syncwarp();  // stage st and the result buffer are free
    if (failed) break;
    if (lane == 0 && t + 2 * nw < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tma_issue(W, st, t + 2 * nw, q0, q1, ca, cb, tile_nodes, eloc8, wmeta, ref8);
      if (st) pend1 = true;
      else pend0 = true;
      if (t + 3 * nw < ntiles) {
        q0 = __ldg(tile_ptr + t + 3 * nw);
        q1 = __ldg(tile_ptr + t + 3 * nw + 1);
      }
    }
  }
  if (failed) {
    // record the timeout and let the copies still in flight land before the
    // warp's shared memory can be reused
    if (lane == 0) {
      atomicExch(&g_wait_status, int(DG_ETIMEOUT));
      const long long drain = wait_limit > (1ll << 31) ? wait_limit : (1ll << 31);
      const long long t0 = clock64();
      while ((pend0 && !mbar_test(&W.bar[0], par0)) || (pend1 && !mbar_test(&W.bar[1], par1)))
        if (clock64() - t0 > drain) {
          atomicExch(&g_drain_gave_up, 1);
          break;
        }
    }
    __syncwarp();
  }
}

template <class CT>
__global__ void lapmass_diag_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                    const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
                                    double* __restrict__ d) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(lev);
    const double a = ca ? double(ca[e]) : 1.0, b = cb ? double(cb[e]) : 1.0;
    const double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    for (int j = 0; j < 8; ++j) {
      double u[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) u[v] = v == j ? 1.0 : 0.0;
      if (mask) interp_hanging(u, c, mask);
      lapmass_ref(u, f1, f2);
      if (mask) scatter_hanging(u, c, mask);
      atomicAdd(d + nl[int64_t(j) * E + e], u[j]);
    }
  }
}

// Dense assembly of a small level into per-mesh row-major blocks: node r of
// block b = row_blk[r] lands at dense[aoff[b] + (r - off[b]) * n[b] + ...].
template <class CT>
__global__ void lapmass_dense_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                     const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
                                     const uint32_t* __restrict__ row_blk, const int64_t* __restrict__ boff,
                                     const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                                     double* __restrict__ A) {
  for (int64_t t = gtid(); t < E * 8; t += gstride()) {
    int64_t e = t >> 3;
    int j = int(t & 7);
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(lev);
    const double a = ca ? double(ca[e]) : 1.0, b = cb ? double(cb[e]) : 1.0;
    const double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    double u[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) u[v] = v == j ? 1.0 : 0.0;
    if (mask) interp_hanging(u, c, mask);
    lapmass_ref(u, f1, f2);
    if (mask) scatter_hanging(u, c, mask);
    const uint32_t col = nl[int64_t(j) * E + e];
    const uint32_t blk = row_blk[col];
    const int64_t o = boff[blk], n = bn[blk];
    double* Ab = A + baoff[blk];
    for (int k = 0; k < 8; ++k)
      atomicAdd(Ab + (int64_t(nl[int64_t(k) * E + e]) - o) * n + (int64_t(col) - o), u[k]);
  }
}

// Type-1 element operator (JAC_TYPE3_MULT_BLOCK's children sum,
// examples/src/backend/omgJac.C:2206-2230): u (natural vertex order) <- the
// sum over the element's 8 children of their operators with their own
// coefficients (cf: a of children 0..7, then b), in the coarse element's
// vertex basis, with the hanging interpolation T on both sides.  Worked in the
// child-number frame: T applied, the frame corner values interpolated
// trilinearly to the 3x3x3 points of the children, each child's Walsh-form
// operator at half the size (f1 = a h/4, f2 = b h^3/64), the children's results
// summed at the points and restricted back to the corners (the transpose of
// the interpolation), then T^T.  Equal to the type-1 tables
// T^T P_f^T (a_f K h/4 + b_f M h^3/64) P_f T (LapType1Stencils.inp /
// MassType1Stencils.inp).
template <int P, int W>
__host__ __device__ constexpr double t1_weight() {  // trilinear weight of corner W at sub-grid point P
  return ((W & 1) ? 0.5 * (P % 3) : 1.0 - 0.5 * (P % 3)) * ((W & 2) ? 0.5 * ((P / 3) % 3) : 1.0 - 0.5 * ((P / 3) % 3)) *
         ((W & 4) ? 0.5 * (P / 9) : 1.0 - 0.5 * (P / 9));
}
template <int F, int V>
__host__ __device__ constexpr int t1_point() {  // sub-grid point of vertex V of frame child F
  return ((F & 1) + (V & 1)) + 3 * (((F >> 1) & 1) + ((V >> 1) & 1)) + 9 * (((F >> 2) & 1) + ((V >> 2) & 1));
}
template <class T, int P>
__device__ __forceinline__ T t1_interp(const T (&w)[8]) {
  T s = T(0);
  if (t1_weight<P, 0>() != 0.0) s += T(t1_weight<P, 0>()) * w[0];
  if (t1_weight<P, 1>() != 0.0) s += T(t1_weight<P, 1>()) * w[1];
  if (t1_weight<P, 2>() != 0.0) s += T(t1_weight<P, 2>()) * w[2];
  if (t1_weight<P, 3>() != 0.0) s += T(t1_weight<P, 3>()) * w[3];
  if (t1_weight<P, 4>() != 0.0) s += T(t1_weight<P, 4>()) * w[4];
  if (t1_weight<P, 5>() != 0.0) s += T(t1_weight<P, 5>()) * w[5];
  if (t1_weight<P, 6>() != 0.0) s += T(t1_weight<P, 6>()) * w[6];
  if (t1_weight<P, 7>() != 0.0) s += T(t1_weight<P, 7>()) * w[7];
  return s;
}
template <class T, int P>
__device__ __forceinline__ void t1_restrict(const T (&R)[27], T (&r)[8]) {
  if constexpr (P < 27) {
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const double wt = (w == 0)   ? t1_weight<P, 0>()
                        : (w == 1) ? t1_weight<P, 1>()
                        : (w == 2) ? t1_weight<P, 2>()
                        : (w == 3) ? t1_weight<P, 3>()
                        : (w == 4) ? t1_weight<P, 4>()
                        : (w == 5) ? t1_weight<P, 5>()
                        : (w == 6) ? t1_weight<P, 6>()
                                   : t1_weight<P, 7>();
      if (wt != 0.0) r[w] += T(wt) * R[P];
    }
    t1_restrict<T, P + 1>(R, r);
  }
}
template <class T, int P>
__device__ __forceinline__ void t1_interp_all(const T (&w)[8], T (&S)[27]) {
  if constexpr (P < 27) {
    S[P] = t1_interp<T, P>(w);
    t1_interp_all<T, P + 1>(w, S);
  }
}
template <class T, int F>
__device__ __forceinline__ void t1_children(const T (&S)[27], T (&R)[27], uint32_t c, T h, const T* __restrict__ a,
                                            const T* __restrict__ b) {
  if constexpr (F < 8) {
    const uint32_t k = uint32_t(F) ^ c;  // the child's number
    const T f1 = a[k] * h * T(0.25), f2 = b[k] * h * h * h * T(1.0 / 64.0);
    T v[8];
    v[0] = S[t1_point<F, 0>()];
    v[1] = S[t1_point<F, 1>()];
    v[2] = S[t1_point<F, 2>()];
    v[3] = S[t1_point<F, 3>()];
    v[4] = S[t1_point<F, 4>()];
    v[5] = S[t1_point<F, 5>()];
    v[6] = S[t1_point<F, 6>()];
    v[7] = S[t1_point<F, 7>()];
    lapmass_ref(v, f1, f2);
    R[t1_point<F, 0>()] += v[0];
    R[t1_point<F, 1>()] += v[1];
    R[t1_point<F, 2>()] += v[2];
    R[t1_point<F, 3>()] += v[3];
    R[t1_point<F, 4>()] += v[4];
    R[t1_point<F, 5>()] += v[5];
    R[t1_point<F, 6>()] += v[6];
    R[t1_point<F, 7>()] += v[7];
    t1_children<T, F + 1>(S, R, c, h, a, b);
  }
}
template <class T>
__device__ __forceinline__ void type1_elem(T (&u)[8], uint32_t m, const T (&a)[8], const T (&b)[8]) {
  const uint32_t c = meta_cnum(m);
  const T h = elem_h<T>(meta_lev(m));
  T w[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) w[j] = u[j ^ c];  // frame
  const uint32_t mp = xor_perm_mask(meta_mask(m), c);
  if (mp) interp_frame(w, mp);
  T S[27], R[27];
  t1_interp_all<T, 0>(w, S);
#pragma unroll
  for (int p = 0; p < 27; ++p) R[p] = T(0);
  t1_children<T, 0>(S, R, c, h, a, b);
  T r[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = T(0);
  t1_restrict<T, 0>(R, r);
  if (mp) scatter_frame(r, mp);
#pragma unroll
  for (int j = 0; j < 8; ++j) u[j ^ c] = r[j];
}

// y += the type-1 operators of the listed elements applied to x (atomics).
template <class T, class CT>
__global__ void type1_add_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta, int64_t E,
                                 const uint32_t* __restrict__ elems, const CT* __restrict__ cf, int64_t n,
                                 const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t e = elems[i];
    T u[8], a[8], b[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      u[v] = x[nl[int64_t(v) * E + e]];
      a[v] = T(cf[16 * i + v]);
      b[v] = T(cf[16 * i + 8 + v]);
    }
    type1_elem(u, meta[e], a, b);
#pragma unroll
    for (int v = 0; v < 8; ++v) atomicAdd(y + nl[int64_t(v) * E + e], u[v]);
  }
}

// The listed elements' type-1 operators added into the dense blocks (one
// thread per element and column), like lapmass_dense_kernel.
__global__ void type1_dense_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta, int64_t E,
                                   const uint32_t* __restrict__ elems, const double* __restrict__ cf, int64_t n,
                                   const uint32_t* __restrict__ row_blk, const int64_t* __restrict__ boff,
                                   const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                                   double* __restrict__ A) {
  for (int64_t t = gtid(); t < n * 8; t += gstride()) {
    const int64_t i = t >> 3;
    const int j = int(t & 7);
    const uint32_t e = elems[i];
    double u[8], a[8], b[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      u[v] = v == j ? 1.0 : 0.0;
      a[v] = cf[16 * i + v];
      b[v] = cf[16 * i + 8 + v];
    }
    type1_elem(u, meta[e], a, b);
    const uint32_t col = nl[int64_t(j) * E + e];
    const uint32_t blk = row_blk[col];
    const int64_t o = boff[blk], nb = bn[blk];
    double* Ab = A + baoff[blk];
    for (int k = 0; k < 8; ++k) atomicAdd(Ab + (int64_t(nl[int64_t(k) * E + e]) - o) * nb + (int64_t(col) - o), u[k]);
  }
}

}  // namespace

// Launch shapes tried by the autotuner: one thread per element with
// different block sizes / register caps / grid sizes, and the warp-tile
// shared-memory form.  The first application on a mesh times each once
// (after one untimed launch) and keeps the fastest for that mesh and
// precision; DG_MATVEC_KERNEL=<index> forces one (testing).
struct MatvecVariant {
  int block, per_sm;  // threads per CTA, CTAs per SM in the grid (0: one thread per element)
  int kind;           // 0 atomic (BLOCK, MINB), 2 warp-tile, 3 + records prefetched, 4 + ids and x too,
                      // 5 records staged by bulk copies, 6 octet (one thread per parent octant),
                      // 7 octet chunks staged through shared memory, 8 the same, lean,
                      // 9 the same with the staging of the next chunks in flight (cp.async),
                      // 10 octet lanes (a child per lane, 8 lanes per parent octant),
                      // 11 octet quads (a column of two children per lane, 4 lanes per octant),
                      // 12 octet with the next octet's ids in flight (cp.async), 13 the same
                      // with each child's coefficients loaded when its operator runs, 14 the
                      // words two octets ahead and x one octet ahead in flight, 15 next ids
                      // in flight, the octet worked in two halves, 16 the element kernel on
                      // the compressed element map, 17 as 12 with a compile-time form for
                      // warps of complete octets without points to fill
  int minb;
  const char* name;
};
constexpr MatvecVariant kVariants[] = {
    {256, 8, 0, 1, "atomic b256 grid 8/SM"},  {256, 0, 0, 1, "atomic b256 grid E"},
    {256, 8, 0, 4, "atomic b256 minB4"},      {128, 16, 0, 8, "atomic b128 minB8"},
    {512, 4, 0, 2, "atomic b512 minB2"},
    {32 * kWarpCta, 5, 2, 5, "warp-tile 32 elems, 5 CTAs/SM"}, {32 * kWarpCta, 6, 2, 6, "warp-tile 32 elems, 6 CTAs/SM"},
    {32 * kWarpCta, 4, 3, 4, "warp-tile 32 elems, 4 CTAs/SM, next tile prefetched"},
    {32 * kWarpCta, 8, 2, 8, "warp-tile 32 elems, 8 CTAs/SM"},
    {32 * kWarpCta, 3, 4, 3, "warp-tile 32 elems, 3 CTAs/SM, ids and x of the next tile in flight"},
    {32 * kWarpCta, 4, 4, 4, "warp-tile 32 elems, 4 CTAs/SM, ids and x of the next tile in flight"},
    {32 * kTmaWarps, 5, 5, 5, "warp-tile 32 elems, records by bulk copy, 5 CTAs of 4 warps/SM"},
    {32 * kTmaWarps, 6, 5, 6, "warp-tile 32 elems, records by bulk copy, 6 CTAs of 4 warps/SM"},
    {32 * kTmaWarps, 7, 5, 7, "warp-tile 32 elems, records by bulk copy, 7 CTAs of 4 warps/SM"},
    {128, 3, 6, 3, "octet b128, 3 CTAs/SM"},
    {128, 4, 6, 4, "octet b128, 4 CTAs/SM"},
    {256, 2, 6, 2, "octet b256, 2 CTAs/SM"},
    {128, 5, 6, 5, "octet b128, 5 CTAs/SM"},
    {kOctChunk, 2, 7, 2, "octet chunks of 128, 2 CTAs/SM"},
    {kOctChunk, 3, 7, 3, "octet chunks of 128, 3 CTAs/SM"},
    {kOctChunk, 4, 7, 4, "octet chunks of 128, 4 CTAs/SM"},
    {kOctChunk, 6, 8, 6, "octet chunks of 128, lean, 6 CTAs/SM"},
    {kOctChunk, 8, 8, 8, "octet chunks of 128, lean, 8 CTAs/SM"},
    {kOctChunk, 5, 8, 5, "octet chunks of 128, lean, 5 CTAs/SM"},
    {kOctChunk, 3, 9, 3, "octet chunks of 128, pipelined staging, 3 CTAs/SM"},
    {kOctChunk, 4, 9, 4, "octet chunks of 128, pipelined staging, 4 CTAs/SM"},
    {256, 4, 10, 4, "octet lanes b256, 4 CTAs/SM"},
    {256, 4, 11, 4, "octet quads b256, 4 CTAs/SM"},
    {128, 4, 12, 4, "octet b128, next ids in flight, 4 CTAs/SM"},
    {128, 5, 12, 5, "octet b128, next ids in flight, 5 CTAs/SM"},
    {128, 4, 13, 4, "octet b128, next ids in flight, coefficients per child, 4 CTAs/SM"},
    {128, 5, 13, 5, "octet b128, next ids in flight, coefficients per child, 5 CTAs/SM"},
    {128, 6, 13, 6, "octet b128, next ids in flight, coefficients per child, 6 CTAs/SM"},
    {128, 2, 14, 2, "octet b128, next ids and x in flight, 2 CTAs/SM"},
    {128, 4, 15, 4, "octet b128, next ids in flight, two halves, 4 CTAs/SM"},
    {128, 5, 15, 5, "octet b128, next ids in flight, two halves, 5 CTAs/SM"},
    {256, 8, 16, 4, "element, compressed map, b256, 8 CTAs/SM"},
    {128, 4, 17, 4, "octet b128, next ids in flight, complete-warp fast path, 4 CTAs/SM"},
};
// Coefficients of at most this many consecutive elements are staged per chunk.
constexpr uint32_t kOctCoefCap = 2048;
// Largest shared-memory need of the chunked kernel, in values: x and sums of
// at most 27 kOctChunk nodes, and kOctCoefCap coefficient pairs.
constexpr size_t kOctChunkSmemMax = 2 * 27 * kOctChunk + 2 * kOctCoefCap;

// Raise a kernel's dynamic shared-memory limit once (the first launch of
// each kernel, normally the autotuner's, outside any stream capture).
static dg_status allow_dynamic_smem(const void* kern, size_t bytes) {
  static std::mutex mu;
  static std::vector<const void*> done;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), kern) != done.end()) return DG_OK;
  DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  done.push_back(kern);
  return DG_OK;
}
constexpr int kNumVariants = int(sizeof(kVariants) / sizeof(kVariants[0]));

// Whether the mesh has the structure a launch shape of this kind reads:
// octets, octet chunks, warp tiles or the compressed map.
static bool variant_runs(int k, const dg_da* da) {
  if (k == 16) return da->cmap.qbits != 0;
  if ((k == 6 || k >= 10) && da->octs.n == 0) return false;
  if (k >= 7 && k <= 9 && da->octs.nchunk == 0) return false;
  if (k >= 2 && k <= 5 && da->tiles_w.ntiles == 0) return false;
  return true;
}

template <class T, class CT>
static dg_status launch_variant(int v, const dg_da* da, const CT* ca, const CT* cb, const T* x, T* y,
                                cudaStream_t s) {
  // a shape fixed by the caller that this mesh cannot run (no octets, no
  // octet chunks or no warp tiles, e.g. a batch of meshes) falls back to
  // the element kernel rather than leaving y unwritten
  {
    if (!variant_runs(kVariants[v].kind, da)) v = 0;
  }
  const MatvecVariant& V = kVariants[v];
  const unsigned g = V.per_sm ? grid_for(da->E, V.block, V.per_sm)
                              : unsigned((da->E + V.block - 1) / V.block > 0 ? (da->E + V.block - 1) / V.block : 1);
  if (V.kind == 16) {
    const CompressedMap& C = da->cmap;
    const CMapView M{C.rem.p, C.qmask.p, C.base.p, C.qoff.p, C.quot.p, da->E};
    lapmass_cmap_kernel<T, CT, 256, 4><<<grid_for(C.ntiles * 32, 256, V.per_sm), 256, 0, s>>>(
        M, C.ntiles, da->meta.p, ca, cb, x, y);
  } else if (V.kind == 9) {
    const OctetSet& O = da->octs;
    const size_t smem = (3 * sizeof(T) + 3 * sizeof(uint32_t)) * size_t(O.max_nodes);
    const unsigned gq = unsigned(std::min<int64_t>(O.nchunk, int64_t(sm_count()) * V.per_sm));
    auto go = [&](auto kern) -> dg_status {
      DG_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(kern),
                                (3 * sizeof(T) + 3 * sizeof(uint32_t)) * 27 * kOctChunk));
      kern<<<gq, kOctChunk, smem, s>>>(O.n, O.nchunk, O.max_nodes, O.meta.p, O.lidx.p, O.lelem.p, O.cptr.p,
                                       O.cnodes.p, O.cel.p, ca, cb, x, y);
      return DG_OK;
    };
    if (V.minb == 3) DG_TRY(go(lapmass_octchunk_pipe_kernel<T, CT, 3>));
    else DG_TRY(go(lapmass_octchunk_pipe_kernel<T, CT, 4>));
  } else if (V.kind == 8) {
    const OctetSet& O = da->octs;
    const size_t smem = sizeof(T) * 2 * size_t(O.max_nodes);
    const unsigned gq = unsigned(std::min<int64_t>(O.nchunk, int64_t(sm_count()) * V.per_sm));
    auto go = [&](auto kern) -> dg_status {
      DG_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(kern), kOctChunkSmemMax * sizeof(T)));
      kern<<<gq, kOctChunk, smem, s>>>(O.n, O.nchunk, O.max_nodes, O.meta.p, O.lidx.p, O.lelem.p, O.cptr.p,
                                       O.cnodes.p, O.cel.p, ca, cb, x, y);
      return DG_OK;
    };
    if (V.minb == 6) DG_TRY(go(lapmass_octchunk_lean_kernel<T, CT, 6>));
    else if (V.minb == 5) DG_TRY(go(lapmass_octchunk_lean_kernel<T, CT, 5>));
    else DG_TRY(go(lapmass_octchunk_lean_kernel<T, CT, 8>));
  } else if (V.kind == 7) {
    const OctetSet& O = da->octs;
    const uint32_t coef_cap = ca ? std::min(O.max_erange, kOctCoefCap) : 0u;
    const size_t smem = sizeof(T) * (2 * size_t(O.max_nodes) + 2 * size_t(coef_cap));
    const unsigned gq = unsigned(std::min<int64_t>(O.nchunk, int64_t(sm_count()) * V.per_sm));
    auto go = [&](auto kern) -> dg_status {
      DG_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(kern), kOctChunkSmemMax * sizeof(T)));
      kern<<<gq, kOctChunk, smem, s>>>(O.n, O.nchunk, O.max_nodes, coef_cap, O.meta.p, O.lidx.p, O.lelem.p,
                                       O.cptr.p, O.cnodes.p, O.cel.p, ca, cb, x, y);
      return DG_OK;
    };
    if (V.minb == 2) DG_TRY(go(lapmass_octchunk_kernel<T, CT, 2>));
    else if (V.minb == 3) DG_TRY(go(lapmass_octchunk_kernel<T, CT, 3>));
    else DG_TRY(go(lapmass_octchunk_kernel<T, CT, 4>));
  } else if (V.kind == 17) {
    const OctetSet& O = da->octs;
    const unsigned gp = grid_for(O.n, 128, V.per_sm);
    lapmass_octet_pf_kernel<T, CT, 128, 4, true, true><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 15) {
    const OctetSet& O = da->octs;
    const unsigned gp = grid_for(O.n, 128, V.per_sm);
    if (V.minb == 5)
      lapmass_octet_pf2_kernel<T, CT, 128, 5><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else
      lapmass_octet_pf2_kernel<T, CT, 128, 4><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 14) {
    const OctetSet& O = da->octs;
    const unsigned gp = grid_for(O.n, 128, V.per_sm);
    auto kern = lapmass_octet_pfx_kernel<T, CT, 128, 2>;
    DG_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(kern), octet_pfx_smem<T, 128>()));
    kern<<<gp, 128, octet_pfx_smem<T, 128>(), s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 13) {
    const OctetSet& O = da->octs;
    const unsigned gp = grid_for(O.n, 128, V.per_sm);
    if (V.minb == 6)
      lapmass_octet_pf_kernel<T, CT, 128, 6, false><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else if (V.minb == 5)
      lapmass_octet_pf_kernel<T, CT, 128, 5, false><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else
      lapmass_octet_pf_kernel<T, CT, 128, 4, false><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 12) {
    const OctetSet& O = da->octs;
    const unsigned gp = grid_for(O.n, 128, V.per_sm);
    if (V.minb == 5)
      lapmass_octet_pf_kernel<T, CT, 128, 5><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else
      lapmass_octet_pf_kernel<T, CT, 128, 4><<<gp, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 11) {
    const OctetSet& O = da->octs;
    lapmass_octquad_kernel<T, CT, 256, 4><<<grid_for(4 * O.n, 256, V.per_sm), 256, 0, s>>>(O.n, O.rec.p, O.elem.p,
                                                                                          ca, cb, x, y);
  } else if (V.kind == 10) {
    const OctetSet& O = da->octs;
    lapmass_octlane_kernel<T, CT, 256, 4><<<grid_for(8 * O.n, 256, V.per_sm), 256, 0, s>>>(O.n, O.rec.p, O.elem.p,
                                                                                          ca, cb, x, y);
  } else if (V.kind == 6) {
    const OctetSet& O = da->octs;
    const unsigned go = grid_for(O.n, V.block, V.per_sm);
    if (V.block == 128 && V.minb == 3)
      lapmass_octet_kernel<T, CT, 128, 3><<<go, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else if (V.block == 128 && V.minb == 5)
      lapmass_octet_kernel<T, CT, 128, 5><<<go, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else if (V.block == 128)
      lapmass_octet_kernel<T, CT, 128, 4><<<go, 128, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
    else
      lapmass_octet_kernel<T, CT, 256, 2><<<go, 256, 0, s>>>(O.n, O.meta.p, O.id.p, O.elem.p, ca, cb, x, y);
  } else if (V.kind == 5) {
    const TileSet& ts = da->tiles_w;
    const unsigned gt = grid_for(ts.ntiles * 32, 32 * kTmaWarps, V.per_sm);
    const uint2* e8 = reinterpret_cast<const uint2*>(ts.eloc8.p);
    const size_t smem = kTmaWarps * sizeof(TmaWarp<T, CT>);
    const long long lim = g_wait_limit;
    if (V.minb == 5)
      lapmass_warp_tma_kernel<T, CT, 5><<<gt, 32 * kTmaWarps, smem, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                        ts.nodes.p, e8, ts.ref8.p, x, y, lim);
    else if (V.minb == 6)
      lapmass_warp_tma_kernel<T, CT, 6><<<gt, 32 * kTmaWarps, smem, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                        ts.nodes.p, e8, ts.ref8.p, x, y, lim);
    else
      lapmass_warp_tma_kernel<T, CT, 7><<<gt, 32 * kTmaWarps, smem, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                        ts.nodes.p, e8, ts.ref8.p, x, y, lim);
  } else if (V.kind >= 2) {
    const TileSet& ts = da->tiles_w;
    const unsigned gw = grid_for(ts.ntiles * 32, 32 * kWarpCta, V.per_sm);
    const uint2* e8 = reinterpret_cast<const uint2*>(ts.eloc8.p);
    if (V.kind == 4 && V.minb == 3)
      lapmass_warp_pipe_kernel<T, CT, 3><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                     ts.nodes.p, e8, ts.ref8.p, x, y);
    else if (V.kind == 4)
      lapmass_warp_pipe_kernel<T, CT, 4><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                     ts.nodes.p, e8, ts.ref8.p, x, y);
    else if (V.kind == 3)
      lapmass_warp_kernel<T, CT, 4, true><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles, ts.ptr.p,
                                                                      ts.nodes.p, e8, ts.ref8.p, x, y);
    else if (V.minb == 6)
      lapmass_warp_kernel<T, CT, 6, false><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles,
                                                                       ts.ptr.p, ts.nodes.p, e8, ts.ref8.p, x, y);
    else if (V.minb == 8)
      lapmass_warp_kernel<T, CT, 8, false><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles,
                                                                       ts.ptr.p, ts.nodes.p, e8, ts.ref8.p, x, y);
    else
      lapmass_warp_kernel<T, CT, 5, false><<<gw, 32 * kWarpCta, 0, s>>>(ts.wmeta.p, ca, cb, da->E, ts.ntiles,
                                                                       ts.ptr.p, ts.nodes.p, e8, ts.ref8.p, x, y);
  } else if (V.block == 256 && V.minb == 1) {
    lapmass_kernel<T, CT, 256, 1><<<g, 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else if (V.block == 256 && V.minb == 4) {
    lapmass_kernel<T, CT, 256, 4><<<g, 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else if (V.block == 128) {
    lapmass_kernel<T, CT, 128, 8><<<g, 128, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else {
    lapmass_kernel<T, CT, 512, 2><<<g, 512, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

static int forced_variant() {
  static int v = -2;
  if (v == -2) {
    const char* e = getenv("DG_MATVEC_KERNEL");
    v = -1;
    if (e && *e) {
      const int kind = !strcmp(e, "atomic") ? 0 : !strcmp(e, "warp") ? 2 : !strcmp(e, "octet") ? 6
                     : !strcmp(e, "chunk") ? 7 : !strcmp(e, "lanes") ? 10 : !strcmp(e, "quads") ? 11
                     : !strcmp(e, "cmap") ? 16 : -1;
      if (kind >= 0) {
        for (int i = kNumVariants - 1; i >= 0; --i)
          if (kVariants[i].kind == kind) v = i;
      } else {
        v = atoi(e) % kNumVariants;
      }
    }
  }
  return v;
}

// The launch shape for a mesh and precision: the forced one, the tuned one,
// or -- on first use outside a stream capture -- tune now: one untimed launch,
// then per variant the best of two timed launches, each after overwriting a
// buffer larger than L2 so that the mesh streams from HBM as it does for
// meshes larger than L2.  y is used as scratch and left zero.  Inside a
// capture an untuned mesh gets the default warp-tile shape.
constexpr int kDefaultVariant = 5;  // "warp-tile 32 elems, 5 CTAs/SM"
template <class T, class CT>
static dg_status pick_variant(const dg_da* da, int& choice, const CT* ca, const CT* cb, const T* x, T* y,
                              cudaStream_t s, int* v_out) {
  if (forced_variant() >= 0) {
    *v_out = forced_variant();
    return DG_OK;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  DG_CUDA(cudaStreamIsCapturing(s, &cap));
  if (choice < 0 && cap != cudaStreamCaptureStatusNone) {  // no timing inside a graph capture
    *v_out = kDefaultVariant;
    return DG_OK;
  }
  if (choice < 0) {
    cudaEvent_t e0, e1;
    DG_CUDA(cudaEventCreate(&e0));
    DG_CUDA(cudaEventCreate(&e1));
    DBuf<uint8_t> flush;
    const int64_t flush_bytes = int64_t(192) << 20;
    DG_TRY(flush.alloc(flush_bytes));
    float best = 1e30f;
    int bi = kDefaultVariant;
    DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
    DG_TRY((launch_variant<T, CT>(0, da, ca, cb, x, y, s)));
    for (int v = 0; v < kNumVariants; ++v) {
      if (!variant_runs(kVariants[v].kind, da)) continue;
      for (int trial = 0; trial < 2; ++trial) {
        DG_CUDA(cudaMemsetAsync(flush.p, trial + 1, flush_bytes, s));
        DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
        DG_CUDA(cudaEventRecord(e0, s));
        DG_TRY((launch_variant<T, CT>(v, da, ca, cb, x, y, s)));
        DG_CUDA(cudaEventRecord(e1, s));
        DG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        DG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          bi = v;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    choice = bi;
    DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
  }
  *v_out = choice;
  return DG_OK;
}

// y = A x with the mesh's launch shape.
template <class T, class CT>
static dg_status lapmass_launch(dg_da* da, int& choice, const CT* ca, const CT* cb, const T* x, T* y,
                                cudaStream_t s) {
  int v = 0;
  DG_TRY((pick_variant<T, CT>(da, choice, ca, cb, x, y, s, &v)));
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
  return launch_variant<T, CT>(v, da, ca, cb, x, y, s);
}

int matvec_variant_count() { return kNumVariants; }

void set_wait_limit(long long cycles) { g_wait_limit = cycles > 0 ? cycles : kDefaultWaitLimit; }
long long wait_limit() { return g_wait_limit; }

dg_status device_wait_status(cudaStream_t s) {
  DG_CUDA(cudaStreamSynchronize(s));
  DG_TRY(mrhs_tc_take_status());
  int v = 0, drained = 0;
  DG_CUDA(cudaMemcpyFromSymbol(&v, g_wait_status, sizeof(int)));
  DG_CUDA(cudaMemcpyFromSymbol(&drained, g_drain_gave_up, sizeof(int)));
  if (v || drained) {
    const int z = 0;
    DG_CUDA(cudaMemcpyToSymbol(g_wait_status, &z, sizeof(int)));
    DG_CUDA(cudaMemcpyToSymbol(g_drain_gave_up, &z, sizeof(int)));
    DG_CHECK(!drained, DG_ETIMEOUT,
             "a bounded device wait of an operator kernel ran out and the copies it had in flight did not land "
             "in time either: shared memory of later blocks may have been overwritten, so every result computed "
             "since the last check is void");
    DG_CHECK(false, DG_ETIMEOUT, "a bounded device wait of an operator kernel ran out");
  }
  return DG_OK;
}

const char* matvec_variant_name(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].name : "untuned"; }

dg_status lapmass_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  dg_da* da = A->da;
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  return lapmass_launch<double, double>(da, da->tuned_f64, ca, cb, x, y, s);
}

// y += A x: the one-thread-per-element shape (launch shape 0), whose FP64
// atomics add into y as it stands, so no clearing pass precedes it.
dg_status lapmass_apply_add_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  dg_da* da = A->da;
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  return launch_variant<double, double>(0, da, ca, cb, x, y, s);
}

dg_status lapmass_apply_add_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s) {
  dg_da* da = A->da;
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  return launch_variant<float, float>(0, da, ca, cb, x, y, s);
}

// ---------------------------------------------------------------------------
// Host entry point with the copies pipelined against the operator.  The warp
// tiles are split into kPipeGroups consecutive groups.  x travels to the GPU
// in node-order chunks on one stream -- the positive-boundary nodes first
// (their anchors have a coordinate equal to the domain size, so their Morton
// keys follow every other node's, yet tiles all along the curve read them) --
// and each group's launch waits (stream event) for the chunk that completes
// the nodes it reads.  After group g, the nodes below the smallest node any
// later group touches are final and go back on a third stream while the
// later groups run.  No kernel waits on a copy: the ordering is stream events.
// 16 groups measured fastest on the 4.7M-element benchmark mesh (8: 0.92-1.07,
// 32: 0.97-0.99, 64: 1.08 ms per call); replaying the sequence from a CUDA
// graph gave nothing measurable, so it is enqueued directly.
struct HostPipe {
  cudaStream_t sx = nullptr, sk = nullptr, sy = nullptr;
  std::vector<cudaEvent_t> ex, ek;
  cudaEvent_t efork = nullptr, ejx = nullptr, ejy = nullptr;
  std::vector<int64_t> tile0;   // [G + 1] tile ranges of the groups
  std::vector<int64_t> xend;    // [G] x [0, xend[g]) (and the tail) present before group g
  std::vector<int64_t> yfinal;  // [G] y [0, yfinal[g]) final after group g
  int64_t tail = 0;             // first positive-boundary node
  int variant = -1;
  ~HostPipe() {
    for (auto e : ex) cudaEventDestroy(e);
    for (auto e : ek) cudaEventDestroy(e);
    if (efork) cudaEventDestroy(efork);
    if (ejx) cudaEventDestroy(ejx);
    if (ejy) cudaEventDestroy(ejy);
    if (sx) cudaStreamDestroy(sx);
    if (sk) cudaStreamDestroy(sk);
    if (sy) cudaStreamDestroy(sy);
  }
};

constexpr int kPipeGroups = 16;
constexpr int64_t kPipeMinElements = int64_t(1) << 20;

static dg_status build_host_pipe(const dg_da* da, HostPipe& P) {
  const TileSet& ts = da->tiles_w;
  const int64_t nt = ts.ntiles, N = da->N;
  std::vector<uint32_t> tptr(nt + 1);
  DG_CUDA(cudaMemcpy(tptr.data(), ts.ptr.p, 4 * (nt + 1), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> nodes(tptr[nt]);
  DG_CUDA(cudaMemcpy(nodes.data(), ts.nodes.p, 4 * nodes.size(), cudaMemcpyDeviceToHost));
  std::vector<uint64_t> nk(N);
  DG_CUDA(cudaMemcpy(nk.data(), da->nkey.p, 8 * N, cudaMemcpyDeviceToHost));
  const uint64_t tail_key = uint64_t(1) << (3 * (da->D - 1));
  P.tail = std::lower_bound(nk.begin(), nk.end(), tail_key) - nk.begin();
  const int G = kPipeGroups;
  P.tile0.resize(G + 1);
  for (int g = 0; g <= G; ++g) P.tile0[g] = nt * g / G;
  std::vector<int64_t> lo(G, P.tail), hi(G, -1);
  for (int g = 0; g < G; ++g)
    for (uint32_t k = tptr[P.tile0[g]]; k < tptr[P.tile0[g + 1]]; ++k) {
      const int64_t v = nodes[k] & 0x7fffffffu;
      if (v >= P.tail) continue;
      lo[g] = std::min(lo[g], v);
      hi[g] = std::max(hi[g], v);
    }
  P.xend.resize(G);
  int64_t run = 0;
  for (int g = 0; g < G; ++g) {
    run = std::max(run, hi[g] + 1);
    P.xend[g] = g + 1 == G ? P.tail : std::min(run, P.tail);
  }
  P.yfinal.resize(G);
  int64_t suffix = P.tail;
  for (int g = G - 1; g >= 0; --g) {
    P.yfinal[g] = suffix;
    suffix = std::min(suffix, lo[g]);
  }
  for (int g = 1; g < G; ++g) P.yfinal[g] = std::max(P.yfinal[g], P.yfinal[g - 1]);
  DG_CUDA(cudaStreamCreateWithFlags(&P.sx, cudaStreamNonBlocking));
  DG_CUDA(cudaStreamCreateWithFlags(&P.sk, cudaStreamNonBlocking));
  DG_CUDA(cudaStreamCreateWithFlags(&P.sy, cudaStreamNonBlocking));
  P.ex.resize(G);
  P.ek.resize(G);
  for (int g = 0; g < G; ++g) {
    DG_CUDA(cudaEventCreateWithFlags(&P.ex[g], cudaEventDisableTiming));
    DG_CUDA(cudaEventCreateWithFlags(&P.ek[g], cudaEventDisableTiming));
  }
  DG_CUDA(cudaEventCreateWithFlags(&P.efork, cudaEventDisableTiming));
  DG_CUDA(cudaEventCreateWithFlags(&P.ejx, cudaEventDisableTiming));
  DG_CUDA(cudaEventCreateWithFlags(&P.ejy, cudaEventDisableTiming));
  return DG_OK;
}

// One warp-tile launch over tiles [t0, t1): the per-element and per-tile
// arrays are offset to the range; tile_ptr holds absolute offsets into the
// node lists, so those stay whole.
static dg_status launch_warp_range(int v, const dg_da* da, const double* ca, const double* cb, int64_t t0,
                                   int64_t t1, const double* x, double* y, cudaStream_t s) {
  const MatvecVariant& V = kVariants[v];
  const TileSet& ts = da->tiles_w;
  const int64_t e0 = t0 * kWarpTile;
  const int64_t E = std::min<int64_t>(da->E, t1 * kWarpTile) - e0;
  const int64_t nt = t1 - t0;
  if (nt <= 0) return DG_OK;
  const unsigned gw = grid_for(nt * 32, 32 * kWarpCta, V.per_sm);
  const uint32_t* wm = ts.wmeta.p + e0;
  const double* a = ca ? ca + e0 : nullptr;
  const double* b = cb ? cb + e0 : nullptr;
  const uint32_t* tp = ts.ptr.p + t0;
  const uint2* e8 = reinterpret_cast<const uint2*>(ts.eloc8.p) + e0;
  const uint8_t* r8 = ts.ref8.p + t0 * kWarpRefBytes;
  if (V.kind == 4 && V.minb == 3)
    lapmass_warp_pipe_kernel<double, double, 3><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8, r8,
                                                                             x, y);
  else if (V.kind == 4)
    lapmass_warp_pipe_kernel<double, double, 4><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8, r8,
                                                                             x, y);
  else if (V.kind == 3)
    lapmass_warp_kernel<double, double, 4, true><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8, r8,
                                                                              x, y);
  else if (V.minb == 6)
    lapmass_warp_kernel<double, double, 6, false><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8,
                                                                               r8, x, y);
  else if (V.minb == 8)
    lapmass_warp_kernel<double, double, 8, false><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8,
                                                                               r8, x, y);
  else
    lapmass_warp_kernel<double, double, 5, false><<<gw, 32 * kWarpCta, 0, s>>>(wm, a, b, E, nt, tp, ts.nodes.p, e8,
                                                                               r8, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// The pipeline's copies and launches, enqueued on P's three streams (sk last
// waits for sx and sy, so that sk alone marks the end).
static dg_status enqueue_host_pipe(const dg_mat* A, HostPipe& P, const double* hx, double* hy) {
  const dg_da* da = A->da;
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  double* dx = A->host_x.p;
  double* dy = A->host_y.p;
  const int64_t N = da->N;
  const int G = kPipeGroups;
  DG_CUDA(cudaEventRecord(P.efork, P.sk));
  DG_CUDA(cudaStreamWaitEvent(P.sx, P.efork, 0));
  DG_CUDA(cudaStreamWaitEvent(P.sy, P.efork, 0));
  // x: the boundary tail, then the chunks in node order
  if (P.tail < N) DG_CUDA(cudaMemcpyAsync(dx + P.tail, hx + P.tail, 8 * (N - P.tail), cudaMemcpyHostToDevice, P.sx));
  int64_t xs = 0;
  for (int g = 0; g < G; ++g) {
    if (P.xend[g] > xs) {
      DG_CUDA(cudaMemcpyAsync(dx + xs, hx + xs, 8 * (P.xend[g] - xs), cudaMemcpyHostToDevice, P.sx));
      xs = P.xend[g];
    }
    DG_CUDA(cudaEventRecord(P.ex[g], P.sx));
  }
  DG_CUDA(cudaMemsetAsync(dy, 0, 8 * N, P.sk));
  int64_t ys = 0;
  for (int g = 0; g < G; ++g) {
    DG_CUDA(cudaStreamWaitEvent(P.sk, P.ex[g], 0));
    DG_TRY(launch_warp_range(P.variant, da, ca, cb, P.tile0[g], P.tile0[g + 1], dx, dy, P.sk));
    DG_CUDA(cudaEventRecord(P.ek[g], P.sk));
    DG_CUDA(cudaStreamWaitEvent(P.sy, P.ek[g], 0));
    const int64_t ye = g + 1 == G ? N : P.yfinal[g];
    if (ye > ys) {
      DG_CUDA(cudaMemcpyAsync(hy + ys, dy + ys, 8 * (ye - ys), cudaMemcpyDeviceToHost, P.sy));
      ys = ye;
    }
  }
  DG_CUDA(cudaEventRecord(P.ejx, P.sx));
  DG_CUDA(cudaEventRecord(P.ejy, P.sy));
  DG_CUDA(cudaStreamWaitEvent(P.sk, P.ejx, 0));
  DG_CUDA(cudaStreamWaitEvent(P.sk, P.ejy, 0));
  return DG_OK;
}

// True when p is page-locked host memory (registered or allocated by CUDA):
// only then do asynchronous copies from / to it overlap with kernels.
static bool page_locked(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

dg_status lapmass_apply_host_pipelined_f64(dg_mat* A, const double* hx, double* hy) {
  dg_da* da = A->da;
  if (A->kind != 0 || da->E < kPipeMinElements || da->tiles_w.ntiles == 0 || da->tuned_f64 < 0) return DG_ENOTIMPL;
  // pageable buffers: each chunk copy would block the host until its group
  // has run, serialising the pipeline, so the caller copies, applies, copies
  if (!page_locked(hx) || !page_locked(hy)) return DG_ENOTIMPL;
  if (!A->pipe) {
    auto P = std::make_shared<HostPipe>();
    DG_TRY(build_host_pipe(da, *P));
    A->pipe = P;
  }
  HostPipe& P = *A->pipe;
  // the mesh's tuned shape when it is a plain warp-tile one, else the default
  const int kind = kVariants[da->tuned_f64].kind;
  P.variant = (kind >= 2 && kind <= 4) ? da->tuned_f64 : kDefaultVariant;
  DG_TRY(enqueue_host_pipe(A, P, hx, hy));
  DG_CUDA(cudaStreamSynchronize(P.sk));
  return DG_OK;
}

dg_status load_vector(const dg_da* da, const double* force, double* b, cudaStream_t s) {
  DG_CUDA(cudaMemsetAsync(b, 0, 8 * size_t(da->N), s));
  if (da->E) load_vector_kernel<<<grid_for(da->E, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, force, da->E, b);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status lapmass_apply_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s) {
  dg_da* da = A->da;
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  return lapmass_launch<float, float>(da, da->tuned_f32, ca, cb, x, y, s);
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// t = A x into a zero-kept accumulator (every launch shape only adds into y
// or stores whole sums, so no memset), with the mesh's tuned shape.
template <class T, class CT>
static dg_status apply_to_zeroed(const dg_mat* A, const CT* coef, const T* x, T* t, cudaStream_t s) {
  dg_da* da = A->da;
  const CT* ca = A->has_coef ? coef : nullptr;
  const CT* cb = A->has_coef ? coef + da->E : nullptr;
  int& choice = sizeof(T) == 8 ? da->tuned_f64 : da->tuned_f32;
  int v = 0;
  DG_TRY((pick_variant<T, CT>(da, choice, ca, cb, x, t, s, &v)));
  return launch_variant<T, CT>(v, da, ca, cb, x, t, s);
}

template <class T, class CT>
static dg_status type1_add(const dg_mat* A, const Type1Set* t1, const T* x, T* y, cudaStream_t s) {
  if (!t1 || !t1->n) return DG_OK;
  const CT* cf;
  if constexpr (sizeof(CT) == 8) cf = t1->coef.p;
  else cf = t1->coef32.p;
  type1_add_kernel<T, CT><<<grid_for(t1->n, 128, 8), 128, 0, s>>>(A->da->nl.p, A->da->meta.p, A->da->E, t1->elem.p, cf,
                                                                   t1->n, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

template <class T, class CT>
static dg_status smooth_sweep(const dg_mat* A, const CT* coef, T* x, const T* b, const T* dinv, T omega, T* t,
                              cudaStream_t s, const Type1Set* t1 = nullptr) {
  DG_TRY((apply_to_zeroed<T, CT>(A, coef, x, t, s)));
  DG_TRY((type1_add<T, CT>(A, t1, x, t, s)));
  const int64_t n = A->da->N;
  constexpr int W = 16 / sizeof(T);
  const int64_t nv = (aligned16(x) && aligned16(b) && aligned16(dinv) && aligned16(t)) ? n / W : 0;
  if (nv)
    jacobi_from_v<T><<<grid_for((nv + kVecU - 1) / kVecU, 256, 8), 256, 0, s>>>(x, b, dinv, t, omega, nv, n);
  else if (n)
    jacobi_from<T><<<grid_for(n, 256, 16), 256, 0, s>>>(x, b, dinv, t, omega, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

template <class T, class CT>
static dg_status residual(const dg_mat* A, const CT* coef, const T* x, const T* b, T* r, T* t, cudaStream_t s,
                          const Type1Set* t1 = nullptr) {
  DG_TRY((apply_to_zeroed<T, CT>(A, coef, x, t, s)));
  DG_TRY((type1_add<T, CT>(A, t1, x, t, s)));
  const int64_t n = A->da->N;
  constexpr int W = 16 / sizeof(T);
  const int64_t nv = (aligned16(b) && aligned16(t) && aligned16(r)) ? n / W : 0;
  if (nv)
    residual_from_v<T><<<grid_for((nv + kVecU - 1) / kVecU, 256, 8), 256, 0, s>>>(b, t, r, nv, n);
  else if (n)
    residual_from<T><<<grid_for(n, 256, 16), 256, 0, s>>>(b, t, r, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status lapmass_smooth_f64(const dg_mat* A, double* x, const double* b, const double* dinv, double omega,
                             double* acc, cudaStream_t s, const double* coef, const Type1Set* t1) {
  return smooth_sweep<double, double>(A, coef ? coef : A->coef.p, x, b, dinv, omega, acc, s, t1);
}
dg_status lapmass_smooth_f32(const dg_mat* A, float* x, const float* b, const float* dinv, float omega, float* acc,
                             cudaStream_t s, const float* coef, const Type1Set* t1) {
  return smooth_sweep<float, float>(A, coef ? coef : A->coef32.p, x, b, dinv, omega, acc, s, t1);
}
dg_status lapmass_residual_f64(const dg_mat* A, const double* x, const double* b, double* r, double* acc,
                               cudaStream_t s, const double* coef, const Type1Set* t1) {
  return residual<double, double>(A, coef ? coef : A->coef.p, x, b, r, acc, s, t1);
}
dg_status lapmass_residual_f32(const dg_mat* A, const float* x, const float* b, float* r, float* acc,
                               cudaStream_t s, const float* coef, const Type1Set* t1) {
  return residual<float, float>(A, coef ? coef : A->coef32.p, x, b, r, acc, s, t1);
}

dg_status lapmass_apply_j_f64(const dg_mat* A, const double* coef, const Type1Set* t1, const double* x, double* y,
                              cudaStream_t s) {
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * A->da->N, s));
  DG_TRY((apply_to_zeroed<double, double>(A, coef ? coef : A->coef.p, x, y, s)));
  return type1_add<double, double>(A, t1, x, y, s);
}

dg_status lapmass_diag(const dg_mat* A, double* d, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * da->N, s));
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  lapmass_diag_kernel<double><<<grid_for(da->E, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, d);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status lapmass_assemble_dense(const dg_mat* A, double* dense, int64_t dense_size, const uint32_t* row_blk,
                                 const int64_t* boff, const int64_t* bn, const int64_t* baoff, cudaStream_t s,
                                 const double* coef, const Type1Set* t1) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(dense, 0, sizeof(double) * dense_size, s));
  const double* c0 = coef ? coef : A->coef.p;
  const double* ca = A->has_coef ? c0 : nullptr;
  const double* cb = A->has_coef ? c0 + da->E : nullptr;
  lapmass_dense_kernel<double><<<grid_for(da->E * 8, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E,
                                                                          row_blk, boff, bn, baoff, dense);
  if (t1 && t1->n)
    type1_dense_kernel<<<grid_for(t1->n * 8, 128, 8), 128, 0, s>>>(da->nl.p, da->meta.p, da->E, t1->elem.p,
                                                                   t1->coef.p, t1->n, row_blk, boff, bn, baoff, dense);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

namespace {

// 1D operators on [-1,1] along the axis with vertex bit B:
// OP 0: mass M1, 1: stiffness K1 = int phi'_k phi'_j, 2: E1 = int phi'_k phi_j,
// 3: E1^T = int phi_k phi'_j.
template <int OP, int B>
__device__ __forceinline__ void op1(const double (&u)[8], double (&o)[8]) {
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v & B) continue;
    const double u0 = u[v], u1 = u[v | B];
    if (OP == 0) {
      const double s = u0 + u1;
      o[v] = (s + u0) * (1.0 / 3.0);
      o[v | B] = (s + u1) * (1.0 / 3.0);
    } else if (OP == 1) {
      const double d = (u0 - u1) * 0.5;
      o[v] = d;
      o[v | B] = -d;
    } else if (OP == 2) {
      const double s = (u0 + u1) * 0.5;
      o[v] = -s;
      o[v | B] = s;
    } else {
      const double d = (u1 - u0) * 0.5;
      o[v] = d;
      o[v | B] = d;
    }
  }
}

// Block (A, B) of the reference-cube grad-div matrix, int d_A phi_k d_B phi_j,
// as a product of three 1D operators; accumulates w * block * u into r.
template <int A, int B>
__device__ __forceinline__ void graddiv_block(const double (&u)[8], double w, double (&r)[8]) {
  constexpr int o0 = (A == 0 && B == 0) ? 1 : (A == 0) ? 2 : (B == 0) ? 3 : 0;
  constexpr int o1 = (A == 1 && B == 1) ? 1 : (A == 1) ? 2 : (B == 1) ? 3 : 0;
  constexpr int o2 = (A == 2 && B == 2) ? 1 : (A == 2) ? 2 : (B == 2) ? 3 : 0;
  double p[8], q[8], t[8];
  op1<o0, 1>(u, p);
  op1<o1, 2>(p, q);
  op1<o2, 4>(q, t);
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] += w * t[v];
}

// The element in its child-number frame (frame vertex f = vertex f ^ c): the
// hanging vertices are the frame vertices of the frame mask, a hanging frame
// vertex interpolates the raw values at its bit subsets (faces from the raw
// edge values, then edges), and T^T sends w_i r_i to every bit subset of a
// hanging i.  Reflecting axis a negates d/dx_a, so the grad-div block (A, B)
// of the frame is the reference block times s_A s_B (s_a = -1 on the axes
// the child number reflects); K and M are unchanged.  The element operator
// itself runs in the Walsh basis, where it is diagonal plus one shifted term
// per off-diagonal block (below).
__device__ __forceinline__ void frame_interp(double (&u)[8], uint32_t fm) {
#pragma unroll
  for (int f = 3; f < 7; ++f) {
    if (f == 4) continue;
    const int b0 = f & -f, b1 = f ^ b0;
    if ((fm >> f) & 1u) u[f] = ((u[0] + u[f]) + (u[b0] + u[b1])) * 0.25;
  }
#pragma unroll
  for (int f = 1; f <= 4; f <<= 1)
    if ((fm >> f) & 1u) u[f] = (u[0] + u[f]) * 0.5;
}
__device__ __forceinline__ void frame_scatter(double (&r)[8], uint32_t fm) {
  double w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const double wt = (i == 1 || i == 2 || i == 4) ? 0.5 : 0.25;
    w[i] = (i != 0 && i != 7 && ((fm >> i) & 1u)) ? r[i] * wt : 0.0;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    double t = ((fm >> j) & 1u) ? 0.0 : r[j];
#pragma unroll
    for (int i = 1; i < 7; ++i)
      if ((i & j) == j) t += w[i];
    r[j] = t;
  }
}
// r = the element's 24 results in the frame from its 24 raw frame values.
__device__ __forceinline__ void elasticity_frame(double (&u0)[8], double (&u1)[8], double (&u2)[8], uint32_t fm,
                                                 uint32_t cn, double wl, double wg, double (&r0)[8],
                                                 double (&r1)[8], double (&r2)[8]) {
  if (fm) {
    frame_interp(u0, fm);
    frame_interp(u1, fm);
    frame_interp(u2, fm);
  }
  // In the Walsh basis (per axis u^ = (u0 + u1, u0 - u1)) the 1D factors are
  // M1 = diag(1, 1/3), K1 = diag(0, 1), int phi'_k phi_j: u^_1 <- -u^_0 and
  // int phi_k phi'_j: u^_0 <- -u^_1, so every grad-div block (A, B), A != B,
  // is one term per Walsh index w with bit A set and bit B clear:
  // r^_A[w] += m_C(w) u^_B[w ^ bit A ^ bit B] (the two -1 cancel; C the third
  // axis, m_a(w) = 1/3 if bit a of w is set, else 1); the diagonal blocks and
  // mu K are diagonal: mu K eigenvalue n 3^(1-n) (n = popcount w), block
  // (A, A) [bit A of w] times m of the other two axes.  r = WHT(r^) / 8.
  wht8(u0);
  wht8(u1);
  wht8(u2);
  const double s0 = (cn & 1u) ? -1.0 : 1.0, s1 = (cn & 2u) ? -1.0 : 1.0, s2 = (cn & 4u) ? -1.0 : 1.0;
  const double g01 = wg * s0 * s1, g02 = wg * s0 * s2, g12 = wg * s1 * s2;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const int n = (w & 1) + ((w >> 1) & 1) + (w >> 2);
    const double kap = n == 0 ? 0.0 : n == 1 ? 1.0 : n == 2 ? 2.0 / 3.0 : 1.0 / 3.0;
    const double m0 = (w & 1) ? 1.0 / 3.0 : 1.0, m1 = (w & 2) ? 1.0 / 3.0 : 1.0, m2 = (w & 4) ? 1.0 / 3.0 : 1.0;
    double a0 = wl * kap * u0[w], a1 = wl * kap * u1[w], a2 = wl * kap * u2[w];
    if (w & 1) a0 += wg * (m1 * m2) * u0[w];
    if (w & 2) a1 += wg * (m0 * m2) * u1[w];
    if (w & 4) a2 += wg * (m0 * m1) * u2[w];
    if ((w & 1) && !(w & 2)) a0 += g01 * m2 * u1[w ^ 3];
    if ((w & 1) && !(w & 4)) a0 += g02 * m1 * u2[w ^ 5];
    if ((w & 2) && !(w & 1)) a1 += g01 * m2 * u0[w ^ 3];
    if ((w & 2) && !(w & 4)) a1 += g12 * m0 * u2[w ^ 6];
    if ((w & 4) && !(w & 1)) a2 += g02 * m1 * u0[w ^ 5];
    if ((w & 4) && !(w & 2)) a2 += g12 * m0 * u1[w ^ 6];
    r0[w] = a0 * 0.125;
    r1[w] = a1 * 0.125;
    r2[w] = a2 * 0.125;
  }
  wht8(r0);
  wht8(r1);
  wht8(r2);
  if (fm) {
    frame_scatter(r0, fm);
    frame_scatter(r1, fm);
    frame_scatter(r2, fm);
  }
}
__device__ __forceinline__ uint32_t frame_mask(uint32_t mask, uint32_t cn) {
  uint32_t fm = 0;
#pragma unroll
  for (int f = 0; f < 8; ++f) fm |= ((mask >> (uint32_t(f) ^ cn)) & 1u) << f;
  return fm;
}

// y = mu h/2 (K x I3) x + (mu + lambda) h/2 GD x per element (worked in the
// element's child-number frame); Dirichlet nodes contribute nothing (columns
// skipped) and receive nothing (rows handled by elasticity_dirichlet_rows).
// x, y are node-major [N][3].
__global__ void __launch_bounds__(128) elasticity_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                                         const uint8_t* __restrict__ dir, int64_t E, double mu, double lam,
                                                         const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m);
    const uint32_t fm = frame_mask(meta_mask(m), c);
    const double fac = elem_h<double>(lev) / 2.0;
    // in the child-number frame: frame vertex v is vertex v ^ c
    uint32_t id[8];
    bool bd[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      id[v] = __ldg(nl + int64_t(uint32_t(v) ^ c) * E + e);
      bd[v] = __ldg(dir + id[v]) != 0;
    }
    double u0[8], u1[8], u2[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      u0[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]));
      u1[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]) + 1);
      u2[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]) + 2);
    }
    double r0[8], r1[8], r2[8];
    elasticity_frame(u0, u1, u2, fm, c, mu * fac, (mu + lam) * fac, r0, r1, r2);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      if (bd[v]) continue;
      atomicAdd(y + 3 * int64_t(id[v]), r0[v]);
      atomicAdd(y + 3 * int64_t(id[v]) + 1, r1[v]);
      atomicAdd(y + 3 * int64_t(id[v]) + 2, r2[v]);
    }
  }
}

// Chunked form (the octet chunks of the mesh, OctetSet): a CTA per chunk
// stages x at the chunk's nodes (3 components) and their Dirichlet flags in
// shared memory with coalesced loads, applies every element of the chunk's
// octets (one thread per element, the same element arithmetic as above) with
// x read from shared memory and the 24 results added into a shared
// accumulator, then writes the chunk's node sums with stores (nodes no other
// chunk touches) or global reductions.  Dirichlet rows are set afterwards by
// elasticity_dirichlet_rows, as for the kernel above.
constexpr int kElasChunkThreads = 256;
__global__ void __launch_bounds__(kElasChunkThreads, 2) elasticity_chunk_kernel(
    int64_t n, int64_t nchunk, uint32_t node_cap, const uint32_t* __restrict__ oelem, const uint16_t* __restrict__ lnl,
    const uint32_t* __restrict__ cptr, const uint32_t* __restrict__ cnodes, const uint32_t* __restrict__ meta,
    const uint8_t* __restrict__ dir, int64_t E, double mu, double lam, const double* __restrict__ x,
    double* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char el_smem[];
  double* sx = reinterpret_cast<double*>(el_smem);
  double* sy = sx + 3 * size_t(node_cap);
  uint8_t* sd = reinterpret_cast<uint8_t*>(sy + 3 * size_t(node_cap));
  for (int64_t q = blockIdx.x; q < nchunk; q += gridDim.x) {
    const uint32_t p0 = __ldg(cptr + q), nn = __ldg(cptr + q + 1) - p0;
    for (uint32_t k0 = threadIdx.x; k0 < nn; k0 += 4 * kElasChunkThreads) {
      uint32_t id[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t k = k0 + u * kElasChunkThreads;
        id[u] = k < nn ? (__ldg(cnodes + p0 + k) & 0x7fffffffu) : 0u;
      }
      double v[4][3];
      uint8_t dv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool in = k0 + u * kElasChunkThreads < nn;
        dv[u] = in ? __ldg(dir + id[u]) : uint8_t(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) v[u][a] = in ? __ldg(x + 3 * int64_t(id[u]) + a) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t k = k0 + u * kElasChunkThreads;
        if (k >= nn) continue;
        sd[k] = dv[u];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          sx[3 * k + a] = v[u][a];
          sy[3 * k + a] = 0.0;
        }
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * kOctChunk; i += kElasChunkThreads) {
      const int c = i / kOctChunk;
      const int64_t o = q * kOctChunk + (i - c * kOctChunk);
      if (o >= n) continue;
      const uint32_t e = __ldg(oelem + int64_t(c) * n + o);
      if (e == kNoNode) continue;
      const uint32_t m = __ldg(meta + e);
      const uint32_t lev = meta_lev(m), cn = meta_cnum(m);
      const uint32_t fm = frame_mask(meta_mask(m), cn);
      const double fac = elem_h<double>(lev) / 2.0;
      // frame vertex v is vertex v ^ cn: its node's chunk-local index
      uint32_t li[8];
      bool bd[8];
      double u0[8], u1[8], u2[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        li[v] = __ldg(lnl + int64_t(uint32_t(v) ^ cn) * E + e);
        bd[v] = sd[li[v]] != 0;
        u0[v] = bd[v] ? 0.0 : sx[3 * li[v]];
        u1[v] = bd[v] ? 0.0 : sx[3 * li[v] + 1];
        u2[v] = bd[v] ? 0.0 : sx[3 * li[v] + 2];
      }
      double r0[8], r1[8], r2[8];
      elasticity_frame(u0, u1, u2, fm, cn, mu * fac, (mu + lam) * fac, r0, r1, r2);
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        if (bd[v]) continue;
        double* t = sy + 3 * li[v];
        if (r0[v] != 0.0) atomicAdd(t, r0[v]);
        if (r1[v] != 0.0) atomicAdd(t + 1, r1[v]);
        if (r2[v] != 0.0) atomicAdd(t + 2, r2[v]);
      }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nn; k += kElasChunkThreads) {
      const uint32_t id = __ldg(cnodes + p0 + k);
      double* dst = y + 3 * int64_t(id & 0x7fffffffu);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        st_if(dst + a, sy[3 * k + a], !(id >> 31));
        red_add_if(dst + a, sy[3 * k + a], (id >> 31) && sy[3 * k + a] != 0.0);
      }
    }
    __syncthreads();
  }
}

__global__ void elasticity_dirichlet_rows(const uint8_t* __restrict__ dir, int64_t N, const double* __restrict__ x,
                                          double* __restrict__ y) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) {
      y[3 * i] = x[3 * i];
      y[3 * i + 1] = x[3 * i + 1];
      y[3 * i + 2] = x[3 * i + 2];
    }
}

// Diagonal: the element operator applied to each of the 24 node unit vectors.
__global__ void elasticity_diag_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                       const uint8_t* __restrict__ dir, int64_t E, double mu, double lam,
                                       double* __restrict__ d) {
  for (int64_t t = gtid(); t < E * 24; t += gstride()) {
    const int64_t e = t / 24;
    const int j = int(t - e * 24), jn = j / 3, jd = j % 3;
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const uint32_t node = nl[int64_t(jn) * E + e];
    if (dir[node]) continue;
    const double fac = elem_h<double>(lev) / 2.0;
    double u[3][8], r[3][8];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int v = 0; v < 8; ++v) u[a][v] = (a == jd && v == jn) ? 1.0 : 0.0;
    if (mask)
      for (int a = 0; a < 3; ++a) interp_hanging(u[a], c, mask);
    const double wl = mu * fac, wg = (mu + lam) * fac;
    for (int a = 0; a < 3; ++a) lapmass_ref_to(u[a], wl, 0.0, r[a]);
    graddiv_block<0, 0>(u[0], wg, r[0]);
    graddiv_block<0, 1>(u[1], wg, r[0]);
    graddiv_block<0, 2>(u[2], wg, r[0]);
    graddiv_block<1, 0>(u[0], wg, r[1]);
    graddiv_block<1, 1>(u[1], wg, r[1]);
    graddiv_block<1, 2>(u[2], wg, r[1]);
    graddiv_block<2, 0>(u[0], wg, r[2]);
    graddiv_block<2, 1>(u[1], wg, r[2]);
    graddiv_block<2, 2>(u[2], wg, r[2]);
    if (mask)
      for (int a = 0; a < 3; ++a) scatter_hanging(r[a], c, mask);
    atomicAdd(d + 3 * int64_t(node) + jd, r[jd][jn]);
  }
}

// Dense assembly of the operator on a small level (the coarsest level of the
// dof-3 multigrid): per element and non-Dirichlet column (node, component)
// the element operator applied to that unit vector, scattered into the
// non-Dirichlet rows of the row-major n3 x n3 matrix (n3 = 3 N).
__global__ void elasticity_dense_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                        const uint8_t* __restrict__ dir, int64_t E, double mu, double lam,
                                        int64_t n3, double* __restrict__ Ad) {
  for (int64_t t = gtid(); t < E * 24; t += gstride()) {
    const int64_t e = t / 24;
    const int j = int(t - e * 24), jn = j / 3, jd = j % 3;
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    // a hanging vertex's slot holds the parent-corner node the DA lists
    // there, so every one of the 8 slots is a column
    const uint32_t node = nl[int64_t(jn) * E + e];
    if (dir[node]) continue;
    const double fac = elem_h<double>(lev) / 2.0;
    double u[3][8], r[3][8];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int v = 0; v < 8; ++v) u[a][v] = (a == jd && v == jn) ? 1.0 : 0.0;
    if (mask)
      for (int a = 0; a < 3; ++a) interp_hanging(u[a], c, mask);
    const double wl = mu * fac, wg = (mu + lam) * fac;
    for (int a = 0; a < 3; ++a) lapmass_ref_to(u[a], wl, 0.0, r[a]);
    graddiv_block<0, 0>(u[0], wg, r[0]);
    graddiv_block<0, 1>(u[1], wg, r[0]);
    graddiv_block<0, 2>(u[2], wg, r[0]);
    graddiv_block<1, 0>(u[0], wg, r[1]);
    graddiv_block<1, 1>(u[1], wg, r[1]);
    graddiv_block<1, 2>(u[2], wg, r[1]);
    graddiv_block<2, 0>(u[0], wg, r[2]);
    graddiv_block<2, 1>(u[1], wg, r[2]);
    graddiv_block<2, 2>(u[2], wg, r[2]);
    if (mask)
      for (int a = 0; a < 3; ++a) scatter_hanging(r[a], c, mask);
    const int64_t col = 3 * int64_t(node) + jd;
    for (int k = 0; k < 8; ++k) {
      const uint32_t rn = nl[int64_t(k) * E + e];
      if (dir[rn]) continue;
      for (int a = 0; a < 3; ++a)
        if (r[a][k] != 0.0) atomicAdd(Ad + (3 * int64_t(rn) + a) * n3 + col, r[a][k]);
    }
  }
}
__global__ void elasticity_dense_dirichlet(const uint8_t* __restrict__ dir, int64_t N, double* __restrict__ Ad) {
  const int64_t n3 = 3 * N;
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i])
      for (int a = 0; a < 3; ++a) Ad[(3 * i + a) * n3 + 3 * i + a] = 1.0;
}

__global__ void set_dirichlet_diag(const uint8_t* __restrict__ dir, int64_t N, double* __restrict__ d) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) d[3 * i] = d[3 * i + 1] = d[3 * i + 2] = 1.0;
}

// DirichletLaplacianMatMult / DirichletJacobianMatMult (examples/src/backend/
// omgJac.C:859-1056): unit coefficients, h/2 L (+ h^3/8 M for the Jacobian);
// the columns of Dirichlet nodes are dropped (their x entries enter as zero,
// in node space, before the hanging interpolation) and their rows become the
// identity (a pass after the elements).
__global__ void __launch_bounds__(128) dirichlet_scalar_kernel(const uint32_t* __restrict__ nl,
                                                               const uint32_t* __restrict__ meta,
                                                               const uint8_t* __restrict__ dir, int64_t E,
                                                               double mass, const double* __restrict__ x,
                                                               double* __restrict__ y) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(meta_lev(m));
    uint32_t id[8];
    bool bd[8];
    double u[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      id[v] = __ldg(nl + int64_t(v) * E + e);
      bd[v] = __ldg(dir + id[v]) != 0;
      u[v] = bd[v] ? 0.0 : __ldg(x + id[v]);
    }
    if (mask) interp_hanging(u, c, mask);
    lapmass_ref(u, h * 0.5, mass * h * h * h * 0.125);
    if (mask) scatter_hanging(u, c, mask);
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (!bd[v]) atomicAdd(y + id[v], u[v]);
  }
}
__global__ void dirichlet_scalar_rows(const uint8_t* __restrict__ dir, int64_t N, const double* __restrict__ x,
                                      double* __restrict__ y) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) y[i] = x[i];
}
// DirichletLaplacianMatGetDiagonal / DirichletJacobianMatGetDiagonal
// (omgJac.C:1058-1160): one thread per (element, vertex).
__global__ void dirichlet_scalar_diag_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                             const uint8_t* __restrict__ dir, int64_t E, double mass,
                                             double* __restrict__ d) {
  for (int64_t t = gtid(); t < E * 8; t += gstride()) {
    const int64_t e = t >> 3;
    const int j = int(t & 7);
    const uint32_t node = nl[int64_t(j) * E + e];
    if (dir[node]) continue;
    const uint32_t m = meta[e];
    const uint32_t c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(meta_lev(m));
    double u[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) u[v] = v == j ? 1.0 : 0.0;
    if (mask) interp_hanging(u, c, mask);
    lapmass_ref(u, h * 0.5, mass * h * h * h * 0.125);
    if (mask) scatter_hanging(u, c, mask);
    atomicAdd(d + node, u[j]);
  }
}
__global__ void set_dirichlet_diag1(const uint8_t* __restrict__ dir, int64_t N, double* __restrict__ d) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) d[i] = 1.0;
}

}  // namespace

// DG_ELASTICITY_KERNEL=element keeps the one-thread-per-element kernel (testing).
static bool elasticity_chunks_off() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("DG_ELASTICITY_KERNEL");
    v = (e && !strcmp(e, "element")) ? 1 : 0;
  }
  return v == 1;
}

dg_status elasticity_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * 3 * da->N, s));
  const OctetSet& O = da->octs;
  if (O.nchunk > 0 && O.lnl.p && !elasticity_chunks_off()) {
    const size_t smem = 6 * sizeof(double) * O.max_nodes + O.max_nodes;
    DG_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(elasticity_chunk_kernel),
                              (6 * sizeof(double) + 1) * 27 * kOctChunk));
    const unsigned g = unsigned(std::min<int64_t>(O.nchunk, int64_t(sm_count()) * 4));
    elasticity_chunk_kernel<<<g, kElasChunkThreads, smem, s>>>(O.n, O.nchunk, O.max_nodes, O.elem.p, O.lnl.p,
                                                               O.cptr.p, O.cnodes.p, da->meta.p, A->dirichlet.p,
                                                               da->E, A->mu, A->lam, x, y);
  } else {
    elasticity_kernel<<<grid_for(da->E, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E, A->mu,
                                                                 A->lam, x, y);
  }
  elasticity_dirichlet_rows<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dirichlet_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  const dg_da* da = A->da;
  const double mass = A->kind == 3 ? 1.0 : 0.0;
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * da->N, s));
  dirichlet_scalar_kernel<<<grid_for(da->E, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E, mass,
                                                                     x, y);
  dirichlet_scalar_rows<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dirichlet_diag(const dg_mat* A, double* d, cudaStream_t s) {
  const dg_da* da = A->da;
  const double mass = A->kind == 3 ? 1.0 : 0.0;
  DG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * da->N, s));
  dirichlet_scalar_diag_kernel<<<grid_for(da->E * 8, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p,
                                                                              da->E, mass, d);
  set_dirichlet_diag1<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, d);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status elasticity_assemble_dense(const dg_mat* A, double* dense, cudaStream_t s) {
  const dg_da* da = A->da;
  const int64_t n3 = 3 * da->N;
  DG_CUDA(cudaMemsetAsync(dense, 0, sizeof(double) * n3 * n3, s));
  elasticity_dense_kernel<<<grid_for(da->E * 24, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E,
                                                                         A->mu, A->lam, n3, dense);
  elasticity_dense_dirichlet<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, dense);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status elasticity_diag(const dg_mat* A, double* d, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * 3 * da->N, s));
  elasticity_diag_kernel<<<grid_for(da->E * 24, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E,
                                                                         A->mu, A->lam, d);
  set_dirichlet_diag<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, d);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg
