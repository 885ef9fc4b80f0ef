// Shared device/host helpers for the B200 octree-FEM library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/dendro_b200.h"

namespace dg {

// ----------------------------------------------------------------- errors --
void set_error(const char* file, int line, const std::string& msg);

#define DG_CUDA(call)                                                         \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) {                                                  \
      ::dg::set_error(__FILE__, __LINE__, cudaGetErrorString(_e));            \
      return DG_ECUDA;                                                        \
    }                                                                         \
  } while (0)

#define DG_CHECK(cond, code, msg)                                             \
  do {                                                                        \
    if (!(cond)) {                                                            \
      ::dg::set_error(__FILE__, __LINE__, msg);                               \
      return code;                                                            \
    }                                                                         \
  } while (0)

#define DG_TRY(expr)                                                          \
  do {                                                                        \
    dg_status _s = (expr);                                                    \
    if (_s != DG_OK) return _s;                                               \
  } while (0)

// ------------------------------------------------------------- octant bits --
// Octant flags follow the reference layout (include/oct/TreeNode.h:77-78).
constexpr uint32_t kLevelMask = 31u;
constexpr uint32_t kBoundary = 64u;
constexpr uint32_t kNode = 128u;
// Deepest supported depths.  A key is the Morton anchor shifted left by 5
// with the level (up to the depth, 5 bits) below it: 3 depth + 5 <= 64 bits.
// Octrees go to maxDepth 19 (62 bits); a mesh embeds its octree one level
// deeper (addBoundaryNodesType1), so meshes go to maxDepth 18 (embedded
// depth 19, 62 bits).
constexpr uint32_t kMaxDepth = 19;
constexpr uint32_t kMaxEmbeddedDepth = 19;

// Morton key of an anchor: bits interleaved z>y>x within each triple, so that
// integer order equals the reference's Morton comparator for distinct anchors
// (src/hilbert/morton.cpp:18-60).
__host__ __device__ __forceinline__ uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
__host__ __device__ __forceinline__ uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x | (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x | (x >> 4)) & 0x100f00f00f00f00full;
  x = (x | (x >> 8)) & 0x1f0000ff0000ffull;
  x = (x | (x >> 16)) & 0x1f00000000ffffull;
  x = (x | (x >> 32)) & 0x1fffffull;
  return uint32_t(x);
}
__host__ __device__ __forceinline__ uint64_t morton(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
__host__ __device__ __forceinline__ void demorton(uint64_t k, uint32_t& x, uint32_t& y, uint32_t& z) {
  x = compact3(k);
  y = compact3(k >> 1);
  z = compact3(k >> 2);
}

// Octant key: Morton anchor key shifted left by 5, level in the low 5 bits.
// Integer order of octant keys is the reference's octant order: Morton order
// of anchors, coarser first for equal anchors (include/oct/TreeNode.txx:186).
__host__ __device__ __forceinline__ uint64_t okey(uint64_t m, uint32_t lev) { return (m << 5) | lev; }
__host__ __device__ __forceinline__ uint64_t okey_m(uint64_t k) { return k >> 5; }
__host__ __device__ __forceinline__ uint32_t okey_l(uint64_t k) { return uint32_t(k & 31u); }

// --------------------------------------------------------------- elements --
// Packed per-element metadata: level (5 b) | child number (3 b) << 5 |
// hanging mask (8 b) << 8 | element type (5 b) << 16.
__host__ __device__ __forceinline__ uint32_t meta_pack(uint32_t lev, uint32_t c, uint32_t mask, uint32_t t) {
  return lev | (c << 5) | (mask << 8) | (t << 16);
}
__host__ __device__ __forceinline__ uint32_t meta_lev(uint32_t m) { return m & 31u; }
__host__ __device__ __forceinline__ uint32_t meta_cnum(uint32_t m) { return (m >> 5) & 7u; }
__host__ __device__ __forceinline__ uint32_t meta_mask(uint32_t m) { return (m >> 8) & 255u; }
__host__ __device__ __forceinline__ uint32_t meta_type(uint32_t m) { return (m >> 16) & 31u; }

// Child-number frame of the warp-tile kernels: frame vertex j is vertex j ^ c
// of the element (c its child number), so the element's own corner of its
// parent is frame vertex 0 and the hanging structure no longer depends on c.
// Bytes j <- j ^ c of a vertex-indexed byte vector (8 node ranks in a uint2).
__device__ __forceinline__ uint2 xor_perm_bytes(uint2 r, uint32_t c) {
  if (c & 1u) {
    r.x = __byte_perm(r.x, 0, 0x2301);
    r.y = __byte_perm(r.y, 0, 0x2301);
  }
  if (c & 2u) {
    r.x = __byte_perm(r.x, 0, 0x1032);
    r.y = __byte_perm(r.y, 0, 0x1032);
  }
  if (c & 4u) {
    const uint32_t t = r.x;
    r.x = r.y;
    r.y = t;
  }
  return r;
}
// byte j of a uint2, zero-extended (one byte permute)
__device__ __forceinline__ uint32_t byte_of(uint2 r, int j) {
  return __byte_perm(j < 4 ? r.x : r.y, 0u, 0x4440u | uint32_t(j & 3));
}
// The hanging mask in the same frame: bit j <- bit j ^ c.
__host__ __device__ __forceinline__ uint32_t xor_perm_mask(uint32_t m, uint32_t c) {
  if (c & 1u) m = ((m & 0x55u) << 1) | ((m & 0xAAu) >> 1);
  if (c & 2u) m = ((m & 0x33u) << 2) | ((m & 0xCCu) >> 2);
  if (c & 4u) m = ((m & 0x0Fu) << 4) | ((m & 0xF0u) >> 4);
  return m;
}
// The 18 element types are 18 hanging patterns in the child-number frame
// (the same set for every child number, listed in a different order per
// child), so an element's stencil in that frame depends on the pattern only.
constexpr uint8_t kFrameMasks[18] = {0, 2, 4, 6, 14, 16, 18, 20, 22, 30, 50, 54, 62, 84, 86, 94, 118, 126};
__host__ __device__ __forceinline__ uint32_t frame_type(uint32_t mp) {
  const uint8_t fm[18] = {0, 2, 4, 6, 14, 16, 18, 20, 22, 30, 50, 54, 62, 84, 86, 94, 118, 126};
  uint32_t t = 0;
#pragma unroll
  for (uint32_t i = 0; i < 18; ++i)
    if (fm[i] == mp) t = i;
  return t;
}
// Per-element word of the warp-tile kernels: level | frame hanging mask << 8
// | frame type (index into kFrameMasks) << 16.
__host__ __device__ __forceinline__ uint32_t wmeta_pack(uint32_t m) {
  const uint32_t mp = xor_perm_mask(meta_mask(m), meta_cnum(m));
  return meta_lev(m) | (mp << 8) | (frame_type(mp) << 16);
}
__host__ __device__ __forceinline__ uint32_t wmeta_ftype(uint32_t w) { return (w >> 16) & 31u; }
__host__ __device__ __forceinline__ uint32_t wmeta_mask(uint32_t w) { return (w >> 8) & 255u; }

// ----------------------------------------------------------------- launch --
int sm_count();
inline unsigned grid_for(int64_t n, int block, int per_sm = 8) {
  int64_t b = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count()) * per_sm;
  if (b > cap) b = cap;
  return unsigned(b < 1 ? 1 : b);
}

// Device buffer with RAII ownership.
template <class T>
struct DBuf {
  T* p = nullptr;
  int64_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { reset(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  dg_status alloc(int64_t count) {
    reset();
    if (count <= 0) return DG_OK;
    cudaError_t e = cudaMalloc(&p, sizeof(T) * size_t(count));
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(__FILE__, __LINE__, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return DG_ENOMEM;
    }
    n = count;
    return DG_OK;
  }
};

}  // namespace dg
