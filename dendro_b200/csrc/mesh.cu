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

// Exclusive scan of one value per thread over a block of TE threads (every
// thread calls it); the block total is returned through `total`.
template <int TE>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* wsum, uint32_t& total) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  uint32_t base = 0;
  total = 0;
  for (int i = 0; i < TE / 32; ++i) {
    if (i < w) base += wsum[i];
    total += wsum[i];
  }
  __syncthreads();
  return base + incl - v;
}

// Per tile of TE consecutive elements (one CTA of TE threads per tile): the
// 8 TE (node id, position v * TE + element) pairs are sorted in shared memory
// by a bitonic network; the sorted positions are the tile's references
// grouped by node (inc), the distinct ids its node list (to tmp, count to
// cnt) and the run ends per node nend.
template <int TE>
__global__ void __launch_bounds__(TE) tile_lists(const uint32_t* __restrict__ nl, int64_t E, int64_t ntiles,
                                                 uint32_t* __restrict__ tmp, uint32_t* __restrict__ cnt,
                                                 uint16_t* __restrict__ nend, uint16_t* __restrict__ inc,
                                                 uint4* __restrict__ eloc, uint8_t* __restrict__ eloc8) {
  constexpr int S = 8 * TE;
  constexpr int kPer = 8;  // sorted entries per thread
  static_assert(S <= 4096, "positions are 12-bit");
  extern __shared__ __align__(16) unsigned char tl_smem[];
  uint64_t* key = reinterpret_cast<uint64_t*>(tl_smem);
  uint16_t* slot = reinterpret_cast<uint16_t*>(key + S);  // position -> node rank
  __shared__ uint32_t wsum[TE / 32];
  const int tid = threadIdx.x;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    for (int i = tid; i < S; i += TE) {
      const int v = i / TE, el = i % TE;
      const int64_t e = t * TE + el;
      key[i] = e < E ? (uint64_t(nl[int64_t(v) * E + e]) << 12) | uint64_t(i) : ~0ull;
    }
    __syncthreads();
    for (int k = 2; k <= S; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int p = tid; p < S / 2; p += TE) {
          const int i = 2 * p - (p & (j - 1));  // lower index of the pair, bit j clear
          const int l = i + j;
          const bool up = (i & k) == 0;
          const uint64_t a = key[i], b = key[l];
          if ((a > b) == up) {
            key[i] = b;
            key[l] = a;
          }
        }
        __syncthreads();
      }
    uint32_t first_f = 0, nfirst = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int j = tid * kPer + q;
      const uint64_t kj = key[j];
      const bool first = kj != ~0ull && (j == 0 || (key[j - 1] >> 12) != (kj >> 12));
      first_f |= uint32_t(first) << q;
      nfirst += first;
    }
    uint32_t total = 0;
    uint32_t run = block_excl_scan<TE>(nfirst, wsum, total);
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int j = tid * kPer + q;
      const uint64_t kj = key[j];
      if (kj == ~0ull) continue;
      if ((first_f >> q) & 1u) {
        tmp[t * S + run] = uint32_t(kj >> 12);
        ++run;
      }
      inc[t * S + j] = uint16_t(kj & 4095u);
      slot[kj & 4095u] = uint16_t(run - 1);
      const bool last = j + 1 == S || (key[j + 1] >> 12) != (kj >> 12);  // padding keys end every run
      if (last) nend[t * S + run - 1] = uint16_t(j + 1);
    }
    if (tid == 0) cnt[t] = total;
    __syncthreads();
    if (eloc) {  // per element the node ranks of its eight vertices
      const int64_t e = t * TE + tid;
      if (e < E) {
        uint4 o;
        o.x = uint32_t(slot[0 * TE + tid]) | (uint32_t(slot[1 * TE + tid]) << 16);
        o.y = uint32_t(slot[2 * TE + tid]) | (uint32_t(slot[3 * TE + tid]) << 16);
        o.z = uint32_t(slot[4 * TE + tid]) | (uint32_t(slot[5 * TE + tid]) << 16);
        o.w = uint32_t(slot[6 * TE + tid]) | (uint32_t(slot[7 * TE + tid]) << 16);
        eloc[e] = o;
      }
      __syncthreads();
    }
    if (eloc8) {  // the same as bytes (tiles of at most 256 nodes)
      const int64_t e = t * TE + tid;
      if (e < E) {
        uint2 o;
        o.x = uint32_t(slot[0 * TE + tid]) | (uint32_t(slot[1 * TE + tid]) << 8) |
              (uint32_t(slot[2 * TE + tid]) << 16) | (uint32_t(slot[3 * TE + tid]) << 24);
        o.y = uint32_t(slot[4 * TE + tid]) | (uint32_t(slot[5 * TE + tid]) << 8) |
              (uint32_t(slot[6 * TE + tid]) << 16) | (uint32_t(slot[7 * TE + tid]) << 24);
        reinterpret_cast<uint2*>(eloc8)[e] = o;
      }
      __syncthreads();
    }
  }
}

// Copy each tile's node list (capacity S per tile) to its final place.
__global__ void tile_compact(const uint32_t* __restrict__ tmp, int S, const uint32_t* __restrict__ ptr,
                             int64_t ntiles, uint32_t* __restrict__ out) {
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t p0 = ptr[t], n = ptr[t + 1] - p0;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) out[p0 + k] = tmp[t * S + k];
  }
}

// Warp-tile reference lists in bytes, per tile of kWarpTile elements (768
// bytes): the 8 * kWarpTile references sorted by node as positions
// v * kWarpTile + element, the node's rank in the tile list, and flags for
// the kernel's segmented sum, which gives each lane 8 consecutive references:
// 1 = a new sum starts here, 2 = the sum leaves after this reference, 4 = it
// leaves as a store (the node's whole run lies in this lane and no other
// tile uses the node), 8 = valid reference.  One warp per tile, one lane per
// node; runs after the nodes shared between tiles are marked.
__global__ void warp_refs(const uint16_t* __restrict__ inc, const uint16_t* __restrict__ nend,
                          const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ nodes,
                          const uint32_t* __restrict__ meta, int64_t ntiles, uint8_t* __restrict__ tmp,
                          uint8_t* __restrict__ out) {
  constexpr int S = 8 * kWarpTile;
  const int lane = threadIdx.x & 31;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x / 32);
  for (int64_t t = blockIdx.x * int64_t(blockDim.x / 32) + (threadIdx.x >> 5); t < ntiles; t += nw) {
    uint8_t* o = tmp + t * 3 * S;  // positions, ranks, flag bytes (8 valid, 1 start, 2 leave, 4 store)
    for (int j = lane; j < S; j += 32) o[2 * S + j] = 0;  // invalid until written
    __syncwarp();
    const uint32_t p0 = ptr[t], nt = ptr[t + 1] - p0;
    for (uint32_t k = lane; k < nt; k += 32) {
      const uint32_t beg = k ? nend[t * S + k - 1] : 0u, end = nend[t * S + k];
      const bool excl = !(nodes[p0 + k] & 0x80000000u);
      for (uint32_t j = beg; j < end; ++j) {
        o[j] = uint8_t(inc[t * S + j]);
        o[S + j] = uint8_t(k);
        const bool lane_first = (j & 7u) == 0u, lane_last = (j & 7u) == 7u;
        const bool start = j == beg || lane_first;
        const bool flush = j + 1 == end || lane_last;
        const bool whole = (beg >> 3) == ((end - 1) >> 3);  // the run does not cross a lane boundary
        o[2 * S + j] = uint8_t(8u | (start ? 1u : 0u) | (flush ? 2u : 0u) | (flush && whole && excl ? 4u : 0u));
      }
    }
    __syncwarp();
    // per lane its 8 references: positions v * 32 + element become frame
    // positions (v ^ c) * 32 + element, the flag bytes one word of bit masks
    uint8_t* f = out + t * kWarpRefBytes;
    uint32_t word = 0;
    for (int q = 0; q < 8; ++q) {
      const int j = lane * 8 + q;
      const uint32_t fl = o[2 * S + j];
      uint32_t pf = 0, rk = 0;
      if (fl & 8u) {
        const uint32_t pos = o[j];
        const uint32_t c = meta_cnum(meta[t * kWarpTile + (pos & 31u)]);
        pf = (((pos >> 5) ^ c) << 5) | (pos & 31u);
        rk = o[S + j];
        word |= (1u << q) | ((fl & 1u) << (8 + q)) | (((fl >> 1) & 1u) << (16 + q)) | (((fl >> 2) & 1u) << (24 + q));
      }
      f[j] = uint8_t(pf);
      f[S + j] = uint8_t(rk);
    }
    reinterpret_cast<uint32_t*>(f + 2 * S)[lane] = word;
    __syncwarp();
  }
}

// Warp tiles: node ranks in the child-number frame and the per-element word
// (level, frame hanging mask).
__global__ void warp_frame(const uint32_t* __restrict__ meta, int64_t E, uint2* __restrict__ eloc8,
                           uint32_t* __restrict__ wmeta) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    eloc8[e] = xor_perm_bytes(eloc8[e], meta_cnum(m));
    wmeta[e] = wmeta_pack(m);
  }
}

// Per node, the number of tiles whose list holds it.
// An entry whose bit 31 is already set (a warp-tile node whose references
// span two lanes of the segmented sum) counts twice, so that it is treated
// like a node shared between tiles.
__global__ void tile_touch(const uint32_t* __restrict__ nodes, int64_t n, uint32_t* __restrict__ touch) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = nodes[i];
    atomicAdd(touch + (id & 0x7fffffffu), (id & 0x80000000u) ? 2u : 1u);
  }
}

// Warp tiles: mark (bit 31) the nodes whose run of sorted references crosses
// a boundary between two lanes' groups of 8, since their sums arrive in parts.
__global__ void warp_split_runs(const uint16_t* __restrict__ nend, const uint32_t* __restrict__ ptr, int64_t ntiles,
                                uint32_t* __restrict__ nodes) {
  constexpr int S = 8 * kWarpTile;
  const int lane = threadIdx.x & 31;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x / 32);
  for (int64_t t = blockIdx.x * int64_t(blockDim.x / 32) + (threadIdx.x >> 5); t < ntiles; t += nw) {
    const uint32_t p0 = ptr[t], nt = ptr[t + 1] - p0;
    for (uint32_t k = lane; k < nt; k += 32) {
      const uint32_t beg = k ? nend[t * S + k - 1] : 0u, end = nend[t * S + k];
      if ((beg >> 3) != ((end - 1) >> 3)) nodes[p0 + k] |= 0x80000000u;
    }
  }
}

// Bit 31 of a list entry: the node is referenced by more than one tile, so its
// sum must be accumulated with a global atomic.  The shared nodes are also
// flagged per node for the compact list of them.
__global__ void tile_local_mark(uint32_t* __restrict__ nodes, int64_t n, const uint32_t* __restrict__ touch) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = nodes[i] & 0x7fffffffu;
    if (touch[id] > 1u) nodes[i] = id | 0x80000000u;
  }
}
__global__ void shared_flag(uint32_t* __restrict__ touch, int64_t N) {
  for (int64_t i = gtid(); i < N; i += gstride()) touch[i] = touch[i] > 1u ? 1u : 0u;
}
__global__ void shared_emit(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, int64_t N,
                            uint32_t* __restrict__ out) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (flag[i]) out[pos[i]] = uint32_t(i);
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
  DG_CHECK(D + 1 <= kMaxEmbeddedDepth, DG_EDEPTH,
           "mesh: maxDepth above 18 is not supported (the embedded depth's keys would exceed 64 bits)");
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
  DG_TRY(build_tiles(da, s));
  return build_octets(da, s);
}

template <int TE>
static dg_status launch_tile_lists(const dg_da* da, int64_t nt, uint32_t* tmp, uint32_t* cnt, uint16_t* nend,
                                   uint16_t* inc, uint4* eloc, uint8_t* eloc8, cudaStream_t s) {
  const size_t smem = size_t(8 + 2) * 8 * TE;
  static bool set = false;
  if (!set && smem > 48 * 1024) {
    DG_CUDA(cudaFuncSetAttribute(tile_lists<TE>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  }
  set = true;
  tile_lists<TE><<<grid_for(nt, TE, 2048 / TE), TE, smem, s>>>(da->nl.p, da->E, nt, tmp, cnt, nend, inc, eloc, eloc8);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status build_tile_set(const dg_da* da, int te, TileSet& ts, cudaStream_t s) {
  DG_CHECK(da->N < (int64_t(1) << 31), DG_EINVAL, "mesh above 2^31 nodes");
  DG_CHECK(te == kMultiTile || te == kWarpTile, DG_EINVAL, "unsupported tile size");
  const int64_t E = da->E, nt = (E + te - 1) / te, S = 8 * int64_t(te);
  ts.te = te;
  ts.ntiles = nt;
  DBuf<uint32_t> tmp, cnt, touch;
  DG_TRY(tmp.alloc(nt * S));
  DG_TRY(cnt.alloc(nt));
  DG_TRY(ts.nend.alloc(nt * S));
  DG_TRY(ts.inc.alloc(nt * S));
  if (te == kWarpTile) {
    DG_TRY(ts.eloc8.alloc(8 * nt * kWarpTile));  // whole tiles
    DG_TRY(launch_tile_lists<kWarpTile>(da, nt, tmp.p, cnt.p, ts.nend.p, ts.inc.p, nullptr, ts.eloc8.p, s));
  } else {
    DG_TRY(ts.eloc.alloc(E));
    DG_TRY(launch_tile_lists<kMultiTile>(da, nt, tmp.p, cnt.p, ts.nend.p, ts.inc.p, ts.eloc.p, nullptr, s));
  }
  std::vector<uint32_t> hc(nt);
  DG_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, 4 * nt, cudaMemcpyDeviceToHost, s));
  uint32_t total = 0;
  DG_TRY(ts.ptr.alloc(nt + 1));
  DG_TRY(scan_u32(cnt.p, ts.ptr.p, nt, &total, s));
  DG_CUDA(cudaMemcpyAsync(ts.ptr.p + nt, &total, 4, cudaMemcpyHostToDevice, s));
  DG_CUDA(cudaStreamSynchronize(s));
  uint32_t mx = 0;
  for (uint32_t c : hc) mx = c > mx ? c : mx;
  ts.max_nodes = mx;
  DG_TRY(ts.nodes.alloc(total + kNodePad));
  tile_compact<<<grid_for(nt, 256, 8), 256, 0, s>>>(tmp.p, int(S), ts.ptr.p, nt, ts.nodes.p);
  DG_TRY(touch.alloc(da->N));
  DG_CUDA(cudaMemsetAsync(touch.p, 0, 4 * da->N, s));
  if (te == kWarpTile)
    warp_split_runs<<<grid_for(nt * 32, 256, 8), 256, 0, s>>>(ts.nend.p, ts.ptr.p, nt, ts.nodes.p);
  tile_touch<<<grid_for(total, 256), 256, 0, s>>>(ts.nodes.p, total, touch.p);
  tile_local_mark<<<grid_for(total, 256), 256, 0, s>>>(ts.nodes.p, total, touch.p);
  shared_flag<<<grid_for(da->N, 256), 256, 0, s>>>(touch.p, da->N);
  DG_CUDA(cudaGetLastError());
  DBuf<uint32_t> pos;
  DG_TRY(pos.alloc(da->N));
  uint32_t ns = 0;
  DG_TRY(scan_u32(touch.p, pos.p, da->N, &ns, s));
  ts.nshared = ns;
  DG_TRY(ts.shared.alloc(ns > 0 ? ns : 1));
  shared_emit<<<grid_for(da->N, 256), 256, 0, s>>>(touch.p, pos.p, da->N, ts.shared.p);
  if (te == kWarpTile) {  // byte lists with flags replace the uint16 ones
    DBuf<uint8_t> r3;
    DG_TRY(r3.alloc(nt * 3 * S));
    DG_TRY(ts.ref8.alloc(nt * kWarpRefBytes));
    warp_refs<<<grid_for(nt * 32, 256, 8), 256, 0, s>>>(ts.inc.p, ts.nend.p, ts.ptr.p, ts.nodes.p, da->meta.p, nt,
                                                         r3.p, ts.ref8.p);
    DG_TRY(ts.wmeta.alloc(nt * kWarpTile));  // whole tiles
    warp_frame<<<grid_for(E, 256), 256, 0, s>>>(da->meta.p, E, reinterpret_cast<uint2*>(ts.eloc8.p), ts.wmeta.p);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaStreamSynchronize(s));  // r3 is freed on return
  }
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  if (te == kWarpTile) {
    ts.inc.reset();
    ts.nend.reset();
  }
  return DG_OK;
}

dg_status build_tiles(dg_da* da, cudaStream_t s) { return build_tile_set(da, kWarpTile, da->tiles_w, s); }

uint32_t etype_mask(int c, int t) { return kEtypeMask[c & 7][t % 18]; }

}  // namespace dg
