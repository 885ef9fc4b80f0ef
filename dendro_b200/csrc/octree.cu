// Octree construction on the GPU: points -> linear octree (points2OctreeSeq /
// p2oLocal, src/oct/Construct.C:880-1015), 2:1 balance with corners
// (balanceOctree -> comboRipple, src/oct/Balance.C:31,767,1162) and one level
// of coarsening (coarsenOctree, src/oct/Coarsen.C:53-104).
//
// All three are integer key manipulations on Morton keys: sort, adjacent
// unique, per-key arithmetic and binary search.  Outputs are bit-exact with
// the reference's octant lists (anchors and levels, Morton order).
#include "dg_internal.h"

namespace dg {

namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

// --------------------------------------------------------------- points --
// Construct.C:897-911: px = (uint)(x * 2^D / gLen) with gLen = 1.
__global__ void quantise_points(const double* __restrict__ pts, int64_t n, uint32_t D,
                                uint64_t* __restrict__ keys, uint32_t* __restrict__ bad) {
  const double scale = double(1u << D);
  const uint32_t top = 1u << D;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    double vx = pts[3 * i] * scale / 1.0, vy = pts[3 * i + 1] * scale / 1.0, vz = pts[3 * i + 2] * scale / 1.0;
    if (!(vx >= 0.0 && vy >= 0.0 && vz >= 0.0 && vx < double(top) && vy < double(top) && vz < double(top))) {
      atomicExch(bad, 1u);
      vx = vy = vz = 0.0;
    }
    keys[i] = morton(uint32_t(vx), uint32_t(vy), uint32_t(vz));
  }
}

__device__ __forceinline__ uint32_t common_level(uint64_t a, uint64_t b, uint32_t D) {
  uint64_t x = a ^ b;
  if (!x) return D;
  uint32_t lz = uint32_t(__clzll(x)) - (64u - 3u * D);
  return lz / 3u;
}

// Leaf of each sorted point: the octant at level l containing point i is
// split iff some window of m+1 consecutive points holding i lies inside it,
// i.e. iff keys j and j+m share the level-l prefix.  The leaf is one level
// below the deepest split ancestor (never deeper than D).
__global__ void point_leaves(const uint64_t* __restrict__ pk, int64_t n, uint32_t D, uint32_t m,
                             uint64_t* __restrict__ leaf) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    int64_t lo = i - int64_t(m) > 0 ? i - int64_t(m) : 0;
    int64_t hi = i < n - 1 - int64_t(m) ? i : n - 1 - int64_t(m);
    uint32_t best = 0;
    for (int64_t j = lo; j <= hi; ++j) {
      uint32_t c = common_level(pk[j], pk[j + m], D);
      c = c < D - 1 ? c : D - 1;
      best = c > best ? c : best;
    }
    uint32_t L = best + 1;
    uint64_t anchor = pk[i] & ~((1ull << (3u * (D - L))) - 1ull);
    leaf[i] = okey(anchor, L);
  }
}

// Number of maximal aligned octants covering the Morton cell range [lo, hi).
__device__ __forceinline__ uint32_t gap_blocks(uint64_t lo, uint64_t hi, uint32_t D, uint64_t* out) {
  uint32_t c = 0;
  while (lo < hi) {
    uint32_t k = lo ? (uint32_t(__ffsll(lo)) - 1u) / 3u : D;
    if (k > D) k = D;
    uint64_t span = hi - lo;
    while (k > 0 && (1ull << (3u * k)) > span) --k;
    if (out) out[c] = okey(lo, D - k);
    ++c;
    lo += 1ull << (3u * k);
  }
  return c;
}

__device__ __forceinline__ void gap_bounds(const uint64_t* __restrict__ lk, int64_t u, int64_t k, uint32_t D,
                                           uint64_t& lo, uint64_t& hi) {
  if (k == 0) {
    lo = 0;
  } else {
    uint64_t p = lk[k - 1];
    lo = okey_m(p) + (1ull << (3u * (D - okey_l(p))));
  }
  hi = (k == u) ? (1ull << (3u * D)) : okey_m(lk[k]);
}

__global__ void count_gaps(const uint64_t* __restrict__ lk, int64_t u, uint32_t D, uint32_t* __restrict__ cnt) {
  for (int64_t k = gtid(); k <= u; k += gstride()) {
    uint64_t lo, hi;
    gap_bounds(lk, u, k, D, lo, hi);
    cnt[k] = gap_blocks(lo, hi, D, nullptr) + (k < u ? 1u : 0u);
  }
}

__global__ void emit_gaps(const uint64_t* __restrict__ lk, int64_t u, uint32_t D, const uint32_t* __restrict__ pos,
                          uint64_t* __restrict__ out) {
  for (int64_t k = gtid(); k <= u; k += gstride()) {
    uint64_t lo, hi;
    gap_bounds(lk, u, k, D, lo, hi);
    uint32_t c = gap_blocks(lo, hi, D, out + pos[k]);
    if (k < u) out[pos[k] + c] = lk[k];
  }
}

// -------------------------------------------------------------- balance --
__global__ void level_composite(const uint64_t* __restrict__ ok, int64_t n, uint32_t D, uint64_t* __restrict__ out,
                                uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[32];
  if (threadIdx.x < 32) h[threadIdx.x] = 0;
  __syncthreads();
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint32_t l = okey_l(ok[i]);
    uint64_t lk = okey_m(ok[i]) >> (3u * (D - l));
    out[i] = (uint64_t(l) << 59) | lk;
    atomicAdd(&h[l], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void strip_level(uint64_t* __restrict__ k, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) k[i] &= (1ull << 59) - 1ull;
}

// Adjacent-unique parents of sorted level-l keys (parent key = key >> 3).
__global__ void mark_parent_unique(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ flag) {
  for (int64_t i = gtid(); i < n; i += gstride()) flag[i] = (i == 0 || (k[i] >> 3) != (k[i - 1] >> 3)) ? 1u : 0u;
}
__global__ void scatter_parents(const uint64_t* __restrict__ k, int64_t n, const uint32_t* __restrict__ flag,
                                const uint32_t* __restrict__ pos, uint64_t* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride())
    if (flag[i]) out[pos[i]] = k[i] >> 3;
}

// The 3x3x3 block of level-l octants around each parent (the parent and its
// 26 same-level neighbours), clipped to the domain; sentinel ~0 elsewhere.
__global__ void block27(const uint64_t* __restrict__ u, int64_t nu, uint32_t l, uint64_t* __restrict__ out) {
  const int64_t side = int64_t(1) << l;
  for (int64_t t = gtid(); t < nu * 27; t += gstride()) {
    int64_t i = t / 27;
    int r = int(t - i * 27);
    int dx = r % 3 - 1, dy = (r / 3) % 3 - 1, dz = r / 9 - 1;
    uint32_t x, y, z;
    demorton(u[i], x, y, z);
    int64_t nx = int64_t(x) + dx, ny = int64_t(y) + dy, nz = int64_t(z) + dz;
    bool ok = nx >= 0 && ny >= 0 && nz >= 0 && nx < side && ny < side && nz < side;
    out[t] = ok ? morton(uint32_t(nx), uint32_t(ny), uint32_t(nz)) : ~0ull;
  }
}

__device__ __forceinline__ bool contains_sorted(const uint64_t* __restrict__ a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo < n && a[lo] == key;
}

// Leaves at level l: children of internal level-(l-1) octants that are not
// internal themselves.  Writes octant keys at depth D, or ~0 for internal.
__global__ void emit_children(const uint64_t* __restrict__ up, int64_t nup, const uint64_t* __restrict__ uc,
                              int64_t nuc, uint32_t l, uint32_t D, uint64_t* __restrict__ out) {
  for (int64_t t = gtid(); t < nup * 8; t += gstride()) {
    uint64_t ck = (up[t >> 3] << 3) | uint64_t(t & 7);
    bool internal = contains_sorted(uc, nuc, ck);
    out[t] = internal ? ~0ull : okey(ck << (3u * (D - l)), l);
  }
}

// -------------------------------------------------------------- coarsen --
__device__ __forceinline__ uint32_t child_of(uint64_t ok, uint32_t D) {
  uint32_t l = okey_l(ok);
  if (l == 0) return 0;
  return uint32_t((okey_m(ok) >> (3u * (D - l))) & 7u);
}
__device__ __forceinline__ uint64_t parent_key(uint64_t ok, uint32_t D) {
  uint32_t l = okey_l(ok);
  uint32_t pl = l ? l - 1 : 0;
  uint64_t m = okey_m(ok) & ~((1ull << (3u * (D - pl))) - 1ull);
  return okey(m, pl);
}

// family start: a child-0 leaf followed by its 7 siblings as leaves
__global__ void coarsen_mark(const uint64_t* __restrict__ k, int64_t n, uint32_t D, uint32_t* __restrict__ start) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint32_t s = 0;
    if (i + 7 < n && okey_l(k[i]) > 0 && child_of(k[i], D) == 0 && okey_l(k[i + 7]) == okey_l(k[i]) &&
        parent_key(k[i + 7], D) == parent_key(k[i], D))
      s = 1;
    start[i] = s;
  }
}
__global__ void coarsen_keep(const uint32_t* __restrict__ start, int64_t n, uint32_t* __restrict__ keep) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    uint32_t kp = 1;
    for (int d = 1; d <= 7 && i - d >= 0; ++d)
      if (start[i - d]) kp = 0;
    keep[i] = kp;
  }
}
__global__ void coarsen_emit(const uint64_t* __restrict__ k, int64_t n, uint32_t D, const uint32_t* __restrict__ start,
                             const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, uint64_t* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride())
    if (keep[i]) out[pos[i]] = start[i] ? parent_key(k[i], D) : k[i];
}

__global__ void count_not_sentinel(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ flag) {
  for (int64_t i = gtid(); i < n; i += gstride()) flag[i] = k[i] != ~0ull ? 1u : 0u;
}

__global__ void scatter_flagged(const uint64_t* __restrict__ k, int64_t n, const uint32_t* __restrict__ flag,
                                const uint32_t* __restrict__ pos, uint64_t* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride())
    if (flag[i]) out[pos[i]] = k[i];
}

}  // namespace

// Keep the entries of keys[0, n) whose flag is set, in order; keys is
// reallocated to the compacted length.
static dg_status compact_by_flag(DBuf<uint64_t>& keys, int64_t n, const uint32_t* flag, int64_t* n_out,
                                 cudaStream_t s) {
  DBuf<uint32_t> pos;
  DBuf<uint64_t> out;
  DG_TRY(pos.alloc(n));
  uint32_t total = 0;
  DG_TRY(scan_u32(flag, pos.p, n, &total, s));
  DG_TRY(out.alloc(total > 0 ? total : 1));
  scatter_flagged<<<grid_for(n, 256), 256, 0, s>>>(keys.p, n, flag, pos.p, out.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  keys = std::move(out);
  *n_out = total;
  return DG_OK;
}

static dg_status drop_sentinels(DBuf<uint64_t>& keys, int64_t n, int64_t* n_out, cudaStream_t s) {
  if (n == 0) {
    *n_out = 0;
    return DG_OK;
  }
  DBuf<uint32_t> flag;
  DG_TRY(flag.alloc(n));
  count_not_sentinel<<<grid_for(n, 256), 256, 0, s>>>(keys.p, n, flag.p);
  return compact_by_flag(keys, n, flag.p, n_out, s);
}

static dg_status set_root(dg_octree* out, uint32_t D, cudaStream_t s) {
  out->max_depth = D;
  DG_TRY(out->keys.alloc(1));
  uint64_t root = okey(0, 0);
  DG_CUDA(cudaMemcpyAsync(out->keys.p, &root, 8, cudaMemcpyHostToDevice, s));
  DG_CUDA(cudaStreamSynchronize(s));
  out->n = 1;
  return DG_OK;
}

dg_status points_to_octree(const double* d_pts, int64_t n, uint32_t D, uint32_t m, dg_octree* out, cudaStream_t s) {
  DG_CHECK(D <= kMaxDepth, DG_EDEPTH, "maxDepth above 19 is not supported");
  DG_CHECK(m >= 1, DG_EINVAL, "maxNumPts must be >= 1");
  DG_CHECK(n >= 0, DG_EINVAL, "negative point count");
  if (D == 0 || n <= int64_t(m)) return set_root(out, D, s);  // Construct.C:884-888,915-919
  DBuf<uint64_t> pk, tmp;
  DBuf<uint32_t> bad;
  DG_TRY(pk.alloc(n));
  DG_TRY(tmp.alloc(n));
  DG_TRY(bad.alloc(1));
  DG_CUDA(cudaMemsetAsync(bad.p, 0, 4, s));
  quantise_points<<<grid_for(n, 256), 256, 0, s>>>(d_pts, n, D, pk.p, bad.p);
  DG_CUDA(cudaGetLastError());
  uint32_t hbad = 0;
  DG_CUDA(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  DG_CHECK(!hbad, DG_EINVAL, "points must lie in [0,1)^3");
  DG_TRY(radix_sort_u64(pk.p, tmp.p, n, int(3 * D), s));
  // leaf of every point, then adjacent-unique
  point_leaves<<<grid_for(n, 256), 256, 0, s>>>(pk.p, n, D, m, tmp.p);
  DG_CUDA(cudaGetLastError());
  int64_t u = 0;
  DG_TRY(unique_u64(tmp.p, n, &u, s));
  // complete the gaps with the coarsest octants
  DBuf<uint32_t> cnt;
  DG_TRY(cnt.alloc(u + 1));
  count_gaps<<<grid_for(u + 1, 256), 256, 0, s>>>(tmp.p, u, D, cnt.p);
  uint32_t total = 0;
  DG_TRY(scan_u32(cnt.p, cnt.p, u + 1, &total, s));
  DG_TRY(out->keys.alloc(total));
  emit_gaps<<<grid_for(u + 1, 256), 256, 0, s>>>(tmp.p, u, D, cnt.p, out->keys.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  out->n = total;
  out->max_depth = D;
  return DG_OK;
}

// Coarsest 2:1 balanced refinement.  W_l (the octants that must exist at
// level l) is the union of the input leaves at level l and the 3x3x3 blocks
// around U_l = parents of W_{l+1}; the balanced leaves at level l are the
// children of U_{l-1} that are not in U_l.
dg_status balance_octree(const dg_octree* in, dg_octree* out, cudaStream_t s) {
  const uint32_t D = in->max_depth;
  const int64_t n = in->n;
  DG_CHECK(D <= kMaxDepth, DG_EDEPTH, "maxDepth above 19 is not supported");
  if (n <= 1) {
    out->max_depth = D;
    DG_TRY(out->keys.alloc(n > 0 ? n : 1));
    if (n) DG_CUDA(cudaMemcpyAsync(out->keys.p, in->keys.p, 8 * n, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(cudaStreamSynchronize(s));
    out->n = n;
    return DG_OK;
  }
  // leaves grouped by level (stable sort on the level bits of a composite key)
  DBuf<uint64_t> byl, tmp;
  DBuf<uint32_t> hist;
  DG_TRY(byl.alloc(n));
  DG_TRY(tmp.alloc(n));
  DG_TRY(hist.alloc(32));
  DG_CUDA(cudaMemsetAsync(hist.p, 0, 128, s));
  level_composite<<<grid_for(n, 256), 256, 0, s>>>(in->keys.p, n, D, byl.p, hist.p);
  DG_CUDA(cudaGetLastError());
  DG_TRY(radix_sort_u64(byl.p, tmp.p, n, 5, s, 59));
  strip_level<<<grid_for(n, 256), 256, 0, s>>>(byl.p, n);
  uint32_t h[32];
  DG_CUDA(cudaMemcpyAsync(h, hist.p, 128, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  int64_t off[33];
  off[0] = 0;
  for (int l = 0; l < 32; ++l) off[l + 1] = off[l] + h[l];

  std::vector<DBuf<uint64_t>> U(D + 1);  // U[l]: internal octants at level l (sorted level keys)
  std::vector<int64_t> nU(D + 1, 0);
  DBuf<uint64_t> W;
  int64_t nW = h[D];
  DG_TRY(W.alloc(nW > 0 ? nW : 1));
  if (nW) DG_CUDA(cudaMemcpyAsync(W.p, byl.p + off[D], 8 * nW, cudaMemcpyDeviceToDevice, s));
  for (uint32_t l = D; l >= 1; --l) {
    // U_{l-1} = unique parents of W_l
    if (nW > 0) {
      DBuf<uint32_t> flag, pos;
      DG_TRY(flag.alloc(nW));
      DG_TRY(pos.alloc(nW));
      mark_parent_unique<<<grid_for(nW, 256), 256, 0, s>>>(W.p, nW, flag.p);
      uint32_t tot = 0;
      DG_TRY(scan_u32(flag.p, pos.p, nW, &tot, s));
      DG_TRY(U[l - 1].alloc(tot));
      scatter_parents<<<grid_for(nW, 256), 256, 0, s>>>(W.p, nW, flag.p, pos.p, U[l - 1].p);
      DG_CUDA(cudaGetLastError());
      DG_CUDA(cudaStreamSynchronize(s));
      nU[l - 1] = tot;
    }
    if (l - 1 == 0) break;
    // W_{l-1} = unique(block27(U_{l-1}) + leaves at level l-1)
    const uint32_t lp = l - 1;
    int64_t nc = nU[lp] * 27 + int64_t(h[lp]);
    DBuf<uint64_t> cand, ctmp;
    DG_TRY(cand.alloc(nc > 0 ? nc : 1));
    DG_TRY(ctmp.alloc(nc > 0 ? nc : 1));
    if (nU[lp]) block27<<<grid_for(nU[lp] * 27, 256), 256, 0, s>>>(U[lp].p, nU[lp], lp, cand.p);
    if (h[lp]) DG_CUDA(cudaMemcpyAsync(cand.p + nU[lp] * 27, byl.p + off[lp], 8 * int64_t(h[lp]),
                                       cudaMemcpyDeviceToDevice, s));
    DG_CUDA(cudaGetLastError());
    // the sentinel needs all 64 bits to sort last
    DG_TRY(radix_sort_u64(cand.p, ctmp.p, nc, 64, s));
    int64_t nu = 0;
    DG_TRY(unique_u64(cand.p, nc, &nu, s));
    if (nu > 0) {
      uint64_t last = 0;
      DG_CUDA(cudaMemcpyAsync(&last, cand.p + nu - 1, 8, cudaMemcpyDeviceToHost, s));
      DG_CUDA(cudaStreamSynchronize(s));
      if (last == ~0ull) --nu;
    }
    W = std::move(cand);
    nW = nu;
  }
  if (nU[0] == 0) return set_root(out, D, s);
  // assemble the leaves level by level
  std::vector<DBuf<uint64_t>> leaves(D + 1);
  std::vector<int64_t> nleaf(D + 1, 0);
  int64_t total = 0;
  for (uint32_t l = 1; l <= D; ++l) {
    if (nU[l - 1] == 0) continue;
    int64_t nk = nU[l - 1] * 8;
    DG_TRY(leaves[l].alloc(nk));
    const uint64_t* uc = nU[l] ? U[l].p : nullptr;
    emit_children<<<grid_for(nk, 256), 256, 0, s>>>(U[l - 1].p, nU[l - 1], uc, nU[l], l, D, leaves[l].p);
    DG_CUDA(cudaGetLastError());
    DG_TRY(drop_sentinels(leaves[l], nk, &nleaf[l], s));
    total += nleaf[l];
  }
  DBuf<uint64_t> all, atmp;
  DG_TRY(all.alloc(total));
  DG_TRY(atmp.alloc(total));
  int64_t o = 0;
  for (uint32_t l = 1; l <= D; ++l) {
    if (nleaf[l]) DG_CUDA(cudaMemcpyAsync(all.p + o, leaves[l].p, 8 * nleaf[l], cudaMemcpyDeviceToDevice, s));
    o += nleaf[l];
  }
  DG_TRY(radix_sort_u64(all.p, atmp.p, total, int(3 * D + 5), s));
  out->keys = std::move(all);
  out->n = total;
  out->max_depth = D;
  return DG_OK;
}

dg_status coarsen_octree(const dg_octree* in, dg_octree* out, cudaStream_t s) {
  const uint32_t D = in->max_depth;
  const int64_t n = in->n;
  out->max_depth = D;
  if (n < 8) {  // Coarsen.C:66-70
    DG_TRY(out->keys.alloc(n > 0 ? n : 1));
    if (n) DG_CUDA(cudaMemcpyAsync(out->keys.p, in->keys.p, 8 * n, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(cudaStreamSynchronize(s));
    out->n = n;
    return DG_OK;
  }
  DBuf<uint32_t> start, keep, pos;
  DG_TRY(start.alloc(n));
  DG_TRY(keep.alloc(n));
  DG_TRY(pos.alloc(n));
  unsigned g = grid_for(n, 256);
  coarsen_mark<<<g, 256, 0, s>>>(in->keys.p, n, D, start.p);
  coarsen_keep<<<g, 256, 0, s>>>(start.p, n, keep.p);
  uint32_t total = 0;
  DG_TRY(scan_u32(keep.p, pos.p, n, &total, s));
  DG_TRY(out->keys.alloc(total));
  coarsen_emit<<<g, 256, 0, s>>>(in->keys.p, n, D, start.p, keep.p, pos.p, out->keys.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  out->n = total;
  return DG_OK;
}

}  // namespace dg
