// Mesh (ot::DA) construction on the GPU for one level:
//  * embed the balanced octree at maxDepth+1 and add the positive-boundary
//    pseudo-octants (addBoundaryNodesType1, src/oct/OctFunctions.C:636-716);
//  * flag octants whose anchor is a non-hanging node (flagNodesType3,
//    OctFunctions.C:1501-2025);
//  * number the nodes in DA order (the Vec order of DA::vecGetBuffer,
//    include/oda/oda.txx:948-970) and build the element->node map with
//    hanging masks, child numbers and element types (DA::buildNodeList,
//    src/oda/private/odaBuildNlist.C:47-856; GET_ETYPE_BLOCK,
//    include/oda/odaUtils.h:334).
#include "dg_internal.h"

namespace dg {

// (childNum, hanging mask) -> element type in [0,18), 255 when the mask is not
// one of the 18 configurations of include/oda/cnumEtypes.h:19-229.
__constant__ uint8_t c_etype_lut[8][256];

namespace {

// Hanging masks of the 18 element types per child number (cnumEtypes.h).
const uint8_t kEtypeMask[8][18] = {
    {0, 4, 2, 6, 16, 20, 18, 22, 14, 30, 84, 86, 94, 50, 54, 62, 118, 126},
    {0, 1, 8, 9, 32, 33, 40, 41, 13, 45, 49, 57, 61, 168, 169, 173, 185, 189},
    {0, 8, 1, 9, 64, 72, 65, 73, 11, 75, 200, 201, 203, 81, 89, 91, 217, 219},
    {0, 2, 4, 6, 128, 130, 132, 134, 7, 135, 162, 166, 167, 196, 198, 199, 230, 231},
    {0, 1, 32, 33, 64, 65, 96, 97, 35, 99, 69, 101, 103, 224, 225, 227, 229, 231},
    {0, 2, 128, 130, 16, 18, 144, 146, 138, 154, 19, 147, 155, 208, 210, 218, 211, 219},
    {0, 4, 16, 20, 128, 132, 144, 148, 21, 149, 140, 156, 157, 176, 180, 181, 188, 189},
    {0, 8, 64, 72, 32, 40, 96, 104, 76, 108, 42, 106, 110, 112, 120, 124, 122, 126}};

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

__device__ __forceinline__ int64_t find_exact(const uint64_t* __restrict__ a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < n && a[lo] == key) ? lo : -1;
}

// Embedded element keys (level + 1, same anchors) and pseudo-octant counts.
__global__ void embed_and_count(const uint64_t* __restrict__ k, int64_t n, uint32_t D, uint64_t* __restrict__ ekey,
                                uint32_t* __restrict__ cnt) {
  const uint32_t top = 1u << D;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint64_t m = okey_m(k[i]);
    uint32_t l = okey_l(k[i]);
    ekey[i] = okey(m, l + 1);
    uint32_t x, y, z;
    demorton(m, x, y, z);
    uint32_t blen = top - (1u << (D - l));
    uint32_t px = x == blen, py = y == blen, pz = z == blen;
    cnt[i] = px + py + pz + (px & py) + (px & pz) + (py & pz) + (px & py & pz);
  }
}

__global__ void emit_pseudo(const uint64_t* __restrict__ k, int64_t n, uint32_t D, const uint32_t* __restrict__ pos,
                            uint64_t* __restrict__ out) {
  const uint32_t top = 1u << D;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint64_t m = okey_m(k[i]);
    uint32_t l = okey_l(k[i]);
    uint32_t x, y, z;
    demorton(m, x, y, z);
    uint32_t blen = top - (1u << (D - l));
    bool px = x == blen, py = y == blen, pz = z == blen;
    uint64_t* o = out + pos[i];
    int c = 0;
    if (px) o[c++] = okey(morton(top, y, z), l + 1);
    if (py) o[c++] = okey(morton(x, top, z), l + 1);
    if (pz) o[c++] = okey(morton(x, y, top), l + 1);
    if (px && py) o[c++] = okey(morton(top, top, z), l + 1);
    if (px && pz) o[c++] = okey(morton(top, y, top), l + 1);
    if (py && pz) o[c++] = okey(morton(x, top, top), l + 1);
    if (px && py && pz) o[c++] = okey(morton(top, top, top), l + 1);
  }
}

// NODE flag: the anchor is hanging when the parent of a same-level neighbour
// across the parent's faces/edges holding the anchor is an octant.
__global__ void flag_nodes(const uint64_t* __restrict__ all, int64_t n, uint32_t Dp, uint32_t* __restrict__ flag) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint64_t k = all[i];
    uint32_t m = okey_l(k);
    bool hanging = false;
    if (m != 1 && m != 0) {
      uint32_t x, y, z;
      demorton(okey_m(k), x, y, z);
      uint32_t s = 1u << (Dp - m);
      uint32_t c = ((x >> (Dp - m)) & 1u) | (((y >> (Dp - m)) & 1u) << 1) | (((z >> (Dp - m)) & 1u) << 2);
      if (c != 0 && c != 7) {
        uint32_t zero = (~c) & 7u;
        uint32_t pmask = ~((2u * s) - 1u);
        for (uint32_t S = 1; S < 8 && !hanging; ++S) {
          if ((S & zero) != S) continue;
          if (((S & 1) && !x) || ((S & 2) && !y) || ((S & 4) && !z)) continue;
          uint32_t nx = x - ((S & 1) ? s : 0), ny = y - ((S & 2) ? s : 0), nz = z - ((S & 4) ? s : 0);
          uint64_t pk = okey(morton(nx & pmask, ny & pmask, nz & pmask), m - 1);
          if (find_exact(all, n, pk) >= 0) hanging = true;
        }
      }
    }
    flag[i] = hanging ? 0u : 1u;
  }
}

__global__ void emit_node_keys(const uint64_t* __restrict__ all, int64_t n, const uint32_t* __restrict__ flag,
                               const uint32_t* __restrict__ pos, uint64_t* __restrict__ nkey) {
  for (int64_t i = gtid(); i < n; i += gstride())
    if (flag[i]) nkey[pos[i]] = okey_m(all[i]);
}

// Element -> node map, hanging mask, child number, element type.
__global__ void build_nlist(const uint64_t* __restrict__ ekey, int64_t E, uint32_t Dp, const uint64_t* __restrict__ nkey,
                            int64_t N, uint32_t* __restrict__ nl, uint32_t* __restrict__ meta, uint32_t* __restrict__ err) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    uint64_t k = ekey[e];
    uint32_t m = okey_l(k);
    uint32_t x, y, z;
    demorton(okey_m(k), x, y, z);
    uint32_t s = 1u << (Dp - m);
    uint32_t pm = ~((2u * s) - 1u);
    uint32_t px = x & pm, py = y & pm, pz = z & pm;
    uint32_t mask = 0;
    for (uint32_t v = 0; v < 8; ++v) {
      uint32_t vx = x + ((v & 1) ? s : 0), vy = y + ((v & 2) ? s : 0), vz = z + ((v & 4) ? s : 0);
      int64_t id = find_exact(nkey, N, morton(vx, vy, vz));
      if (id < 0) {
        mask |= 1u << v;
        id = find_exact(nkey, N, morton(px + ((v & 1) ? 2 * s : 0), py + ((v & 2) ? 2 * s : 0),
                                        pz + ((v & 4) ? 2 * s : 0)));
        if (id < 0) {
          atomicOr(err, 1u);
          id = 0;
        }
      }
      nl[int64_t(v) * E + e] = uint32_t(id);
    }
    uint32_t c = ((x >> (Dp - m)) & 1u) | (((y >> (Dp - m)) & 1u) << 1) | (((z >> (Dp - m)) & 1u) << 2);
    uint32_t t = mask ? c_etype_lut[c][mask] : 0u;
    if (t == 255u) {
      atomicOr(err, 2u);
      t = 0;
    }
    meta[e] = meta_pack(m, c, mask, t);
  }
}

// Per tile of kTile consecutive elements: min node id and the window span.
__global__ void tile_ranges(const uint32_t* __restrict__ nl, int64_t E, int tile, int64_t ntiles,
                            uint32_t* __restrict__ lo_out, uint32_t* __restrict__ span_out) {
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    uint32_t lo = 0xffffffffu, hi = 0;
    const int64_t e0 = t * tile;
    for (int v = 0; v < 8; ++v)
      for (int i = threadIdx.x; i < tile; i += blockDim.x) {
        const int64_t e = e0 + i;
        if (e < E) {
          const uint32_t id = nl[int64_t(v) * E + e];
          lo = min(lo, id);
          hi = max(hi, id);
        }
      }
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_down_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_down_sync(0xffffffffu, hi, o));
    }
    __shared__ uint32_t slo[32], shi[32];
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      slo[w] = lo;
      shi[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int i = 1; i < int(blockDim.x >> 5); ++i) {
        lo = min(lo, slo[i]);
        hi = max(hi, shi[i]);
      }
      lo_out[t] = lo;
      span_out[t] = hi >= lo ? hi - lo + 1 : 0;
    }
    __syncthreads();
  }
}

}  // namespace

static dg_status upload_etype_lut() {
  static bool done = false;
  if (done) return DG_OK;
  uint8_t lut[8][256];
  memset(lut, 255, sizeof lut);
  for (int c = 0; c < 8; ++c)
    for (int t = 0; t < 18; ++t) lut[c][kEtypeMask[c][t]] = uint8_t(t);
  DG_CUDA(cudaMemcpyToSymbol(c_etype_lut, lut, sizeof lut));
  done = true;
  return DG_OK;
}

dg_status build_mesh(const dg_octree* tree, dg_da* da, cudaStream_t s) {
  const uint32_t D = tree->max_depth;
  const int64_t E = tree->n;
  DG_CHECK(D + 1 <= kMaxEmbeddedDepth, DG_EDEPTH, "maxDepth above 19 is not supported");
  DG_CHECK(E >= 1, DG_EINVAL, "empty octree");
  DG_TRY(upload_etype_lut());
  const uint32_t Dp = D + 1;
  da->D = Dp;
  da->E = E;
  DBuf<uint32_t> cnt;
  DG_TRY(cnt.alloc(E));
  DBuf<uint64_t> ekey;
  DG_TRY(ekey.alloc(E));
  unsigned g = grid_for(E, 256);
  embed_and_count<<<g, 256, 0, s>>>(tree->keys.p, E, D, ekey.p, cnt.p);
  uint32_t P = 0;
  DG_TRY(scan_u32(cnt.p, cnt.p, E, &P, s));
  da->P = P;
  const int64_t n = E + P;
  DBuf<uint64_t> all, tmp;
  DG_TRY(all.alloc(n));
  DG_TRY(tmp.alloc(P > 0 ? P : 1));
  DG_CUDA(cudaMemcpyAsync(all.p, ekey.p, 8 * E, cudaMemcpyDeviceToDevice, s));
  emit_pseudo<<<g, 256, 0, s>>>(tree->keys.p, E, D, cnt.p, all.p + E);
  DG_CUDA(cudaGetLastError());
  // pseudo-octants lie outside the domain child of the embedded root, so they
  // sort after every element; sorting them alone keeps `all` sorted
  DG_TRY(radix_sort_u64(all.p + E, tmp.p, P, int(3 * Dp + 5), s));
  DBuf<uint32_t> flag, pos;
  DG_TRY(flag.alloc(n));
  DG_TRY(pos.alloc(n));
  flag_nodes<<<grid_for(n, 256), 256, 0, s>>>(all.p, n, Dp, flag.p);
  uint32_t N = 0;
  DG_TRY(scan_u32(flag.p, pos.p, n, &N, s));
  da->N = N;
  DG_TRY(da->nkey.alloc(N));
  emit_node_keys<<<grid_for(n, 256), 256, 0, s>>>(all.p, n, flag.p, pos.p, da->nkey.p);
  DG_TRY(da->nl.alloc(8 * E));
  DG_TRY(da->meta.alloc(E));
  DBuf<uint32_t> err;
  DG_TRY(err.alloc(1));
  DG_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
  build_nlist<<<g, 256, 0, s>>>(ekey.p, E, Dp, da->nkey.p, N, da->nl.p, da->meta.p, err.p);
  DG_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  DG_CUDA(cudaMemcpyAsync(&herr, err.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  DG_CHECK(!(herr & 1u), DG_EUNBALANCED, "hanging vertex without a parent node: octree not 2:1 balanced");
  DG_CHECK(!(herr & 2u), DG_EUNBALANCED, "hanging configuration outside the 18 element types");
  da->ekey = std::move(ekey);
  return build_tiles(da, s);
}

dg_status build_tiles(dg_da* da, cudaStream_t s) {
  const int tile = 512;  // elements per tile of the shared-memory operator kernel
  da->tile_elems = tile;
  da->ntiles = (da->E + tile - 1) / tile;
  DG_TRY(da->tile_lo.alloc(da->ntiles));
  DG_TRY(da->tile_span.alloc(da->ntiles));
  tile_ranges<<<grid_for(da->ntiles, 256, 16), 256, 0, s>>>(da->nl.p, da->E, tile, da->ntiles, da->tile_lo.p,
                                                             da->tile_span.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  return DG_OK;
}

}  // namespace dg
