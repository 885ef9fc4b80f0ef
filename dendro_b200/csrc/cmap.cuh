// Compressed element-to-node map (the reference's compressLut option of the
// DA, include/oda/oda.txx:1125-1300 and the m_ucpLutRemainders /
// m_uspLutQuotients members, include/oda/oda.h:332-341), in a warp-tile form.
//
// The reference stores per element its sorted node offsets from the element's
// own index, as a remainder byte plus a 16-bit quotient where the offset needs
// one, decoded serially by the element loop.  Here elements come in tiles of
// 32 consecutive elements, one per lane of a warp:
//   base[t]       the smallest node id tile t references;
//   rem[e]        8 bytes, byte v = (id_v - base) & 255 for vertex v of element
//                 e, in the DA's vertex order (no sort to undo);
//   qmask[e]      bit v set when (id_v - base) >> 8 is nonzero;
//   quot[...]     those quotients of the tile, element-major then vertex,
//                 at qoff[t] (bit 31 of qoff: a wide tile, two 16-bit words per
//                 quotient, lower first, used when a quotient of the tile does
//                 not fit the narrow width).
// A lane finds its first quotient by a warp prefix sum of the per-lane
// quotient counts, so a warp decodes 32 elements with one 8-byte and one
// 1-byte load per lane, coalesced, and its share of the quotient words.
#pragma once

#include "dg_internal.h"

namespace dg {

struct CMapView {
  const uint2* rem;
  const uint8_t* qmask;
  const uint32_t* base;
  const uint32_t* qoff;
  const uint16_t* quot;
  int64_t E;
};

constexpr uint32_t kCmapWide = 0x80000000u;

// The 8 node ids of element e = 32 t + lane (vertex order).  Called by all 32
// lanes of a warp for the same tile t; lanes past the last element get
// unspecified ids.
__device__ __forceinline__ void cmap_ids(const CMapView& M, int64_t t, uint32_t lane, uint32_t (&id)[8]) {
  const int64_t e = t * 32 + lane;
  uint2 r = make_uint2(0u, 0u);
  uint32_t mask = 0;
  if (e < M.E) {
    r = __ldg(M.rem + e);
    mask = __ldg(M.qmask + e);
  }
  const uint32_t b = __ldg(M.base + t), qo = __ldg(M.qoff + t);
  const uint32_t wide = qo >> 31;
  const uint32_t cnt = uint32_t(__popc(mask)) << wide;
  uint32_t incl = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= uint32_t(d)) incl += o;
  }
  const uint16_t* q = M.quot + (qo & ~kCmapWide) + (incl - cnt);
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    uint32_t off = ((v < 4 ? r.x : r.y) >> (8 * (v & 3))) & 255u;
    if ((mask >> v) & 1u) {
      uint32_t qq = __ldg(q);
      if (wide) qq |= uint32_t(__ldg(q + 1)) << 16;
      q += 1 + wide;
      off |= qq << 8;
    }
    id[v] = b + off;
  }
}

}  // namespace dg
