// Octet form of the Laplacian + mass operator (Jacobian2MatMult,
// examples/src/backend/omgNeumann.C:468-557): one thread per parent octant.
//
// Every leaf element is child c of a parent octant P.  The 8 children of P
// share the 3 x 3 x 3 lattice of P's corners, edge midpoints, face centres
// and centre (lattice point p = x + 3 y + 9 z, x, y, z in {0, 1, 2}); vertex v
// of child c is lattice point c + v per axis.  An "octet" is a parent with at
// least one leaf child; a child mask says which children are elements (the
// others are refined further and belong to deeper octets).  Per octet the
// mesh stores the node id of every lattice point that is a node of a present
// child, and kNoNode for points that hang or that no present child touches.
//
// Hanging points are the reference's hanging vertices (the 2:1 balanced
// octree's vertices that lie inside an edge or face of a coarser element,
// odaBuildNlist.C): an edge midpoint of P takes the mean of its edge's two
// corners, a face centre the mean of its face's four corners, exactly the
// interpolation T of the per-element stencils (`T^T L T`, handleType2Stencils.C).
// Corners of P are never hanging (a coarser neighbour of a child is at most
// P's size and aligned with P), and the centre is interior to P.
//
// The thread gathers x at the octet's nodes once, fills the hanging points,
// applies each present child's element operator with compile-time lattice
// indices (all values stay in registers), accumulates the 27 lattice sums,
// folds the hanging points' sums back onto their corners (T^T) and adds each
// node's sum into y with one FP64/FP32 global reduction -- the sums over the
// octet's own children are done in registers, not in memory.
#pragma once

#include "dg_internal.h"
#include "element.cuh"

namespace dg {

constexpr uint32_t kNoNode = 0xffffffffu;

// Lattice point of vertex v of child c.
__host__ __device__ constexpr int oct_lat(int c, int v) {
  return ((c & 1) + (v & 1)) + 3 * (((c >> 1) & 1) + ((v >> 1) & 1)) + 9 * (((c >> 2) & 1) + ((v >> 2) & 1));
}
// Coordinate a (0 x, 1 y, 2 z) of lattice point p, and its stride.
__host__ __device__ constexpr int oct_coord(int p, int a) { return a == 0 ? p % 3 : a == 1 ? (p / 3) % 3 : p / 9; }
__host__ __device__ constexpr int oct_stride(int a) { return a == 0 ? 1 : a == 1 ? 3 : 9; }
// Number of coordinates equal to 1: 0 corner, 1 edge midpoint, 2 face centre, 3 centre.
__host__ __device__ constexpr int oct_free(int p) {
  return (oct_coord(p, 0) == 1) + (oct_coord(p, 1) == 1) + (oct_coord(p, 2) == 1);
}
// The two free axes' strides of a face centre (or the one of an edge midpoint in s0).
__host__ __device__ constexpr int oct_s0(int p) {
  return oct_coord(p, 0) == 1 ? 1 : oct_coord(p, 1) == 1 ? 3 : 9;
}
__host__ __device__ constexpr int oct_s1(int p) {
  return oct_coord(p, 2) == 1 ? 9 : oct_coord(p, 1) == 1 ? 3 : 1;
}

// Per-octet word: level of the children (embedded) | child mask << 8.
__host__ __device__ __forceinline__ uint32_t ometa_lev(uint32_t m) { return m & 31u; }
__host__ __device__ __forceinline__ uint32_t ometa_cmask(uint32_t m) { return (m >> 8) & 255u; }

// The arithmetic of one octet on its 27 lattice values xv: the
// points flagged in `none` (no node: hanging, or not a vertex of a present
// child) are filled from their corners; every present child's element
// operator is applied with compile-time lattice indices; the sums of the
// hanging points are folded back onto their corners (T^T).  yv receives the
// 27 lattice sums (meaningful at the points with a node).  coef(c, f1, f2)
// scales child c's two factors by its coefficients.
// Lattice points that can hang: the 12 edge midpoints and 6 face centres.
__host__ __device__ constexpr uint32_t oct_hangable() {
  uint32_t m = 0;
  for (int p = 0; p < 27; ++p)
    if (oct_free(p) == 1 || oct_free(p) == 2) m |= 1u << p;
  return m;
}

// FULL: the caller knows that all 8 children are present and that no point
// needs filling (a compile-time child loop and no fill or fold).
template <class T, bool FULL = false, class Coef>
__device__ __forceinline__ void octet_apply(T (&xv)[27], T (&yv)[27], uint32_t none, uint32_t m, Coef coef) {
  // octets without a point to fill skip the interpolation and the fold (a
  // branch, uniform when a warp works one octet)
  const bool fill = !FULL && (none & oct_hangable()) != 0u;
  if (fill) {
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        if ((none >> p) & 1u) xv[p] = (xv[p - s0] + xv[p + s0]) * T(0.5);
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        if ((none >> p) & 1u)
          xv[p] = ((xv[p - s0 - s1] + xv[p + s0 - s1]) + (xv[p - s0 + s1] + xv[p + s0 + s1])) * T(0.25);
      }
    }
  }
#pragma unroll
  for (int p = 0; p < 27; ++p) yv[p] = T(0);
  const uint32_t cm = FULL ? 255u : ometa_cmask(m);
  const T h = elem_h<T>(ometa_lev(m));
  const T g1 = h * T(0.5), g2 = h * h * h * T(0.125);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if (FULL || ((cm >> c) & 1u)) {
      T f1 = g1, f2 = g2;
      coef(c, f1, f2);
      T u[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) u[v] = xv[oct_lat(c, v)];
      lapmass_ref(u, f1, f2);
#pragma unroll
      for (int v = 0; v < 8; ++v) yv[oct_lat(c, v)] += u[v];
    }
  }
  if (fill) {
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        const T w = ((none >> p) & 1u) ? yv[p] * T(0.5) : T(0);
        yv[p - s0] += w;
        yv[p + s0] += w;
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        const T w = ((none >> p) & 1u) ? yv[p] * T(0.25) : T(0);
        yv[p - s0 - s1] += w;
        yv[p + s0 - s1] += w;
        yv[p - s0 + s1] += w;
        yv[p + s0 + s1] += w;
      }
    }
  }
}

}  // namespace dg
