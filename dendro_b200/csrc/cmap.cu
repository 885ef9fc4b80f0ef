// Compressed element map: build (two passes over the DA's map and a scan of
// the tiles' quotient counts) and decode (cmap.cuh).
#include "cmap.cuh"
#include "dg_internal.h"

namespace dg {
namespace {

// Per tile (one warp): the base, each lane's remainder bytes and quotient
// mask, and the tile's count of quotient words; wide[t] when a quotient does
// not fit qbits bits.
__device__ __forceinline__ void tile_offsets(const uint32_t* __restrict__ nl, int64_t E, int64_t t, uint32_t lane,
                                             uint32_t (&off)[8], uint32_t& base, bool& live) {
  const int64_t e = t * 32 + lane;
  live = e < E;
  uint32_t mn = 0xffffffffu;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    off[v] = live ? nl[int64_t(v) * E + e] : 0xffffffffu;
    mn = min(mn, off[v]);
  }
  base = __reduce_min_sync(0xffffffffu, mn);
#pragma unroll
  for (int v = 0; v < 8; ++v) off[v] = live ? off[v] - base : 0u;
}

__global__ void cmap_pass1(const uint32_t* __restrict__ nl, int64_t E, int64_t ntiles, uint32_t narrow_lim,
                           uint2* __restrict__ rem, uint8_t* __restrict__ qmask, uint32_t* __restrict__ base,
                           uint32_t* __restrict__ cnt, uint8_t* __restrict__ wide) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t t = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += nw) {
    uint32_t off[8], b;
    bool live;
    tile_offsets(nl, E, t, lane, off, b, live);
    uint32_t m = 0, big = 0;
    uint2 r = make_uint2(0u, 0u);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const uint32_t q = off[v] >> 8;
      if (q) m |= 1u << v;
      big |= q >= narrow_lim;
      const uint32_t byte = (off[v] & 255u) << (8 * (v & 3));
      if (v < 4) r.x |= byte;
      else r.y |= byte;
    }
    const bool w = __any_sync(0xffffffffu, big) != 0;
    const uint32_t words = __reduce_add_sync(0xffffffffu, uint32_t(__popc(m)) << (w ? 1 : 0));
    if (live) {
      rem[t * 32 + lane] = r;
      qmask[t * 32 + lane] = uint8_t(m);
    }
    if (lane == 0) {
      base[t] = b;
      cnt[t] = words;
      wide[t] = w;
    }
  }
}

__global__ void cmap_pass2(const uint32_t* __restrict__ nl, int64_t E, int64_t ntiles,
                           const uint8_t* __restrict__ wide, uint32_t* __restrict__ qoff,
                           uint16_t* __restrict__ quot) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t t = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += nw) {
    uint32_t off[8], b;
    bool live;
    tile_offsets(nl, E, t, lane, off, b, live);
    const uint32_t w = wide[t];
    uint32_t c = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) c += (off[v] >> 8) != 0u;
    c <<= w;
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= uint32_t(d)) incl += o;
    }
    const uint32_t q0 = qoff[t];
    uint16_t* q = quot + q0 + (incl - c);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const uint32_t qq = off[v] >> 8;
      if (qq) {
        q[0] = uint16_t(qq & 0xffffu);
        if (w) q[1] = uint16_t(qq >> 16);
        q += 1 + w;
      }
    }
    __syncwarp();
    if (lane == 0 && w) qoff[t] = q0 | kCmapWide;
  }
}

__global__ void cmap_decode_kernel(CMapView M, int64_t ntiles, uint32_t* __restrict__ out) {
  const uint32_t lane = threadIdx.x & 31u;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t t = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += nw) {
    uint32_t id[8];
    cmap_ids(M, t, lane, id);
    const int64_t e = t * 32 + lane;
    if (e < M.E)
#pragma unroll
      for (int v = 0; v < 8; ++v) out[int64_t(v) * M.E + e] = id[v];
  }
}

}  // namespace

dg_status build_cmap(dg_da* da, int qbits, cudaStream_t s) {
  DG_CHECK(da, DG_EINVAL, "compress_maps: null mesh");
  DG_CHECK(qbits >= 1 && qbits <= 16, DG_EINVAL, "compress_maps: quotient bits must be 1..16");
  CompressedMap& C = da->cmap;
  C = CompressedMap();
  const int64_t E = da->E, nt = (E + 31) / 32;
  if (!E) return DG_OK;
  DBuf<uint32_t> cnt;
  DBuf<uint8_t> wide;
  DG_TRY(C.rem.alloc(E));
  DG_TRY(C.qmask.alloc(E));
  DG_TRY(C.base.alloc(nt));
  DG_TRY(C.qoff.alloc(nt));
  DG_TRY(cnt.alloc(nt));
  DG_TRY(wide.alloc(nt));
  const unsigned g = grid_for(nt * 32, 256, 8);
  cmap_pass1<<<g, 256, 0, s>>>(da->nl.p, E, nt, 1u << qbits, C.rem.p, C.qmask.p, C.base.p, cnt.p, wide.p);
  DG_CUDA(cudaGetLastError());
  uint32_t words = 0;
  DG_TRY(scan_u32(cnt.p, C.qoff.p, nt, &words, s));
  DG_CHECK(words < kCmapWide, DG_EINVAL, "compress_maps: too many quotient words for 31-bit offsets");
  DG_TRY(C.quot.alloc(words > 0 ? words : 1));
  cmap_pass2<<<g, 256, 0, s>>>(da->nl.p, E, nt, wide.p, C.qoff.p, C.quot.p);
  DG_CUDA(cudaGetLastError());
  std::vector<uint8_t> hw(nt);
  DG_CUDA(cudaMemcpyAsync(hw.data(), wide.p, nt, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  int64_t nwide = 0;
  for (uint8_t w : hw) nwide += w;
  C.ntiles = nt;
  C.qbits = qbits;
  C.wide_tiles = nwide;
  // the autotuner times the new launch shape at the next application
  da->tuned_f64 = da->tuned_f32 = -1;
  return DG_OK;
}

dg_status cmap_decode(const dg_da* da, uint32_t* nl_out, cudaStream_t s) {
  DG_CHECK(da && da->cmap.qbits, DG_EINVAL, "decompress_maps: the mesh has no compressed map");
  const CompressedMap& C = da->cmap;
  const CMapView M{C.rem.p, C.qmask.p, C.base.p, C.qoff.p, C.quot.p, da->E};
  cmap_decode_kernel<<<grid_for(C.ntiles * 32, 256, 8), 256, 0, s>>>(M, C.ntiles, nl_out);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg
