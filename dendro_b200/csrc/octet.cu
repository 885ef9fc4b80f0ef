// Builds the octet tables of a mesh (OctetSet, octet.cuh): elements grouped by
// their parent octant, the node id of every lattice point of the parent, the
// element id of every present child.  One-time set-up after the element ->
// node map (build_nlist, mesh.cu) exists.
#include <algorithm>
#include <vector>

#include "octet.cuh"

namespace dg {
namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

__device__ __forceinline__ int64_t find_key(const uint64_t* __restrict__ a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && a[lo] == key) ? lo : -1;
}

// Parent octant key of element e (embedded level m >= 1, so the parent has
// level m - 1 >= 0 and lies inside the embedded domain).
__device__ __forceinline__ uint64_t parent_key(uint64_t ek, uint32_t Dp) {
  const uint32_t m = okey_l(ek);
  uint32_t x, y, z;
  demorton(okey_m(ek), x, y, z);
  const uint32_t pm = ~((2u << (Dp - m)) - 1u);
  return okey(morton(x & pm, y & pm, z & pm), m - 1);
}

__global__ void octet_parent_keys(const uint64_t* __restrict__ ekey, int64_t E, uint32_t Dp,
                                  uint64_t* __restrict__ pk) {
  for (int64_t e = gtid(); e < E; e += gstride()) pk[e] = parent_key(ekey[e], Dp);
}

// Per element: its octet, child bit, level, element id, and the node ids of
// its non-hanging vertices at their lattice points; hanging and non-hanging
// lattice points are recorded separately so that the two can be checked to
// agree (a lattice point's hanging status is a property of the point).
__global__ void octet_fill(const uint64_t* __restrict__ ekey, int64_t E, uint32_t Dp,
                           const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                           const uint64_t* __restrict__ okeys, int64_t n, uint32_t* __restrict__ ometa,
                           uint32_t* __restrict__ oid, uint32_t* __restrict__ oelem, uint32_t* __restrict__ hang,
                           uint32_t* __restrict__ node, uint32_t* __restrict__ err) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const int64_t o = find_key(okeys, n, parent_key(ekey[e], Dp));
    if (o < 0) {
      atomicOr(err, 1u);
      continue;
    }
    const uint32_t m = meta[e];
    const uint32_t c = meta_cnum(m), mask = meta_mask(m);
    atomicOr(ometa + o, meta_lev(m) | (1u << (8 + c)));
    oelem[int64_t(c) * n + o] = uint32_t(e);
    uint32_t hb = 0, nb = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      // lattice point of vertex v of child c (c is a run-time value here)
      const int p = int(((c & 1u) + (v & 1)) + 3 * (((c >> 1) & 1u) + ((v >> 1) & 1)) +
                        9 * (((c >> 2) & 1u) + ((v >> 2) & 1)));
      if ((mask >> v) & 1u) {
        hb |= 1u << p;
        // the DA lists a hanging vertex v as the parent's vertex v, the
        // octet corner at lattice point 2 v, one of the corners its
        // interpolation reads
        const int pc = 2 * (v & 1) + 6 * ((v >> 1) & 1) + 18 * ((v >> 2) & 1);
        oid[int64_t(pc) * n + o] = nl[int64_t(v) * E + e];
      } else {
        nb |= 1u << p;
        oid[int64_t(p) * n + o] = nl[int64_t(v) * E + e];
      }
    }
    if (hb) atomicOr(hang + o, hb);
    atomicOr(node + o, nb);
  }
}

// Checks that no lattice point is both hanging for one child and a node for
// another and that no corner hangs; corners a hanging point needs and no
// element listed (none expected) are looked up among the node anchors.
__global__ void octet_corners(const uint64_t* __restrict__ okeys, int64_t n, uint32_t Dp,
                              const uint64_t* __restrict__ nkey, int64_t N, const uint32_t* __restrict__ hang,
                              const uint32_t* __restrict__ node, uint32_t* __restrict__ oid,
                              uint32_t* __restrict__ err) {
  constexpr uint32_t kCornerBits = (1u << 0) | (1u << 2) | (1u << 6) | (1u << 8) | (1u << 18) | (1u << 20) |
                                   (1u << 24) | (1u << 26);
  for (int64_t o = gtid(); o < n; o += gstride()) {
    const uint32_t hb = hang[o], nb = node[o];
    if ((hb & nb) || (hb & kCornerBits) || (hb & (1u << 13))) {
      atomicOr(err, 2u);
      continue;
    }
    uint32_t need = 0;
    for (int p = 0; p < 27; ++p) {
      if (!((hb >> p) & 1u)) continue;
      const int cx = p % 3, cy = (p / 3) % 3, cz = p / 9;
      for (int b = 0; b < 8; ++b) {
        // corners of p: free axes (coordinate 1) take 0 or 2, the others stay
        if (((b & 1) && cx != 1) || ((b & 2) && cy != 1) || ((b & 4) && cz != 1)) continue;
        const int qx = cx == 1 ? 2 * (b & 1) : cx, qy = cy == 1 ? (b & 2) : cy, qz = cz == 1 ? (b & 4) / 2 : cz;
        need |= 1u << (qx + 3 * qy + 9 * qz);
      }
    }
    // corners still without an id (none: every element lists its hanging
    // vertices' corners) are looked up among the node anchors
    for (int p = 0; p < 27; ++p)
      if (((need >> p) & 1u) && oid[int64_t(p) * n + o] != kNoNode) need &= ~(1u << p);
    if (!need) continue;
    const uint64_t k = okeys[o];
    const uint32_t pl = okey_l(k);
    uint32_t x, y, z;
    demorton(okey_m(k), x, y, z);
    const uint32_t S = 1u << (Dp - pl);  // parent size, embedded units
    for (int p = 0; p < 27; ++p) {
      if (!((need >> p) & 1u)) continue;
      const uint32_t qx = x + (p % 3 ? S : 0), qy = y + ((p / 3) % 3 ? S : 0), qz = z + (p / 9 ? S : 0);
      const int64_t id = find_key(nkey, N, morton(qx, qy, qz));
      if (id < 0) {
        atomicOr(err, 4u);
        continue;
      }
      oid[int64_t(p) * n + o] = uint32_t(id);
    }
  }
}

// ---------------------------------------------------------------- chunks --
// One CTA per chunk of kOctChunk octets: the ids of the chunk's lattice nodes
// (27 per octet, kNoNode included) sorted in shared memory by a bitonic sort.
constexpr int kChunkKeys = 4096;  // >= 27 kOctChunk, a power of two
constexpr int kChunkThreads = 256;
static_assert(kChunkKeys >= 27 * kOctChunk, "chunk key buffer");

__device__ void chunk_sorted_ids(int64_t q, int64_t n, const uint32_t* __restrict__ oid, uint32_t* keys) {
  const int64_t o0 = q * kOctChunk;
  const int no = int(n - o0 < kOctChunk ? n - o0 : kOctChunk);
  for (int t = threadIdx.x; t < kChunkKeys; t += kChunkThreads) {
    uint32_t v = kNoNode;
    if (t < 27 * no) {
      const int p = t / no, j = t - p * no;
      v = oid[int64_t(p) * n + o0 + j];
    }
    keys[t] = v;
  }
  __syncthreads();
  for (int k = 2; k <= kChunkKeys; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < kChunkKeys; i += kChunkThreads) {
        const int l = i ^ j;
        if (l > i) {
          const uint32_t a = keys[i], b = keys[l];
          if ((a > b) == ((i & k) == 0)) {
            keys[i] = b;
            keys[l] = a;
          }
        }
      }
      __syncthreads();
    }
}

__device__ __forceinline__ bool chunk_first(const uint32_t* keys, int i) {
  return keys[i] != kNoNode && (i == 0 || keys[i] != keys[i - 1]);
}

// Per chunk: number of distinct nodes, first element id and element range.
__global__ void __launch_bounds__(kChunkThreads) chunk_count(int64_t n, const uint32_t* __restrict__ oid,
                                                             const uint32_t* __restrict__ oelem,
                                                             uint32_t* __restrict__ count, uint32_t* __restrict__ cel) {
  __shared__ uint32_t keys[kChunkKeys];
  __shared__ uint32_t red[3];
  const int64_t q = blockIdx.x;
  chunk_sorted_ids(q, n, oid, keys);
  if (threadIdx.x == 0) {
    red[0] = 0;
    red[1] = 0xffffffffu;
    red[2] = 0;
  }
  __syncthreads();
  uint32_t c = 0;
  for (int i = threadIdx.x; i < kChunkKeys; i += kChunkThreads) c += chunk_first(keys, i);
  const int64_t o0 = q * kOctChunk;
  const int no = int(n - o0 < kOctChunk ? n - o0 : kOctChunk);
  uint32_t emin = 0xffffffffu, emax = 0;
  for (int t = threadIdx.x; t < 8 * no; t += kChunkThreads) {
    const int cc = t / no, j = t - cc * no;
    const uint32_t e = oelem[int64_t(cc) * n + o0 + j];
    if (e != kNoNode) {
      emin = min(emin, e);
      emax = max(emax, e);
    }
  }
  atomicAdd(&red[0], c);
  atomicMin(&red[1], emin);
  atomicMax(&red[2], emax);
  __syncthreads();
  if (threadIdx.x == 0) {
    count[q] = red[0];
    cel[2 * q] = red[1];
    cel[2 * q + 1] = red[2] - red[1] + 1;
  }
}

// Per chunk: its distinct node ids into cnodes, a count per node of the
// chunks that touch it, and the chunk-local indices of every octet's lattice
// nodes and children's elements.
__global__ void __launch_bounds__(kChunkThreads) chunk_emit(int64_t n, const uint32_t* __restrict__ oid,
                                                            const uint32_t* __restrict__ oelem,
                                                            const uint32_t* __restrict__ cptr,
                                                            const uint32_t* __restrict__ cel,
                                                            uint32_t* __restrict__ cnodes,
                                                            uint32_t* __restrict__ ncount,
                                                            uint16_t* __restrict__ lidx,
                                                            uint16_t* __restrict__ lelem,
                                                            const uint32_t* __restrict__ nl, int64_t E,
                                                            uint16_t* __restrict__ lnl) {
  __shared__ uint32_t keys[kChunkKeys];
  __shared__ uint32_t uniq[kChunkKeys];
  __shared__ uint32_t tsum[kChunkThreads];
  const int64_t q = blockIdx.x;
  chunk_sorted_ids(q, n, oid, keys);
  // compaction: thread t owns keys [16 t, 16 t + 16)
  constexpr int per = kChunkKeys / kChunkThreads;
  const int i0 = threadIdx.x * per;
  uint32_t c = 0;
  for (int i = i0; i < i0 + per; ++i) c += chunk_first(keys, i);
  tsum[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int t = 0; t < kChunkThreads; ++t) {
      const uint32_t v = tsum[t];
      tsum[t] = acc;
      acc += v;
    }
  }
  __syncthreads();
  uint32_t r = tsum[threadIdx.x];
  const uint32_t base = cptr[q];
  for (int i = i0; i < i0 + per; ++i)
    if (chunk_first(keys, i)) {
      uniq[r] = keys[i];
      cnodes[base + r] = keys[i];
      atomicAdd(ncount + keys[i], 1u);
      ++r;
    }
  __syncthreads();
  const int nu = int(cptr[q + 1] - base);
  const int64_t o0 = q * kOctChunk;
  const int no = int(n - o0 < kOctChunk ? n - o0 : kOctChunk);
  for (int t = threadIdx.x; t < 27 * no; t += kChunkThreads) {
    const int p = t / no, j = t - p * no;
    const int64_t g = int64_t(p) * n + o0 + j;
    const uint32_t id = oid[g];
    uint16_t li = 0xffffu;
    if (id != kNoNode) {
      int lo = 0, hi = nu;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (uniq[mid] < id) lo = mid + 1;
        else hi = mid;
      }
      li = uint16_t(lo);
    }
    lidx[g] = li;
  }
  const uint32_t e0 = cel[2 * q];
  for (int t = threadIdx.x; t < 8 * no; t += kChunkThreads) {
    const int cc = t / no, j = t - cc * no;
    const int64_t g = int64_t(cc) * n + o0 + j;
    const uint32_t e = oelem[g];
    lelem[g] = e == kNoNode ? uint16_t(0xffffu) : uint16_t(e - e0);
    if (e == kNoNode) continue;
    // the element's 8 nodes as listed by the DA (a hanging vertex lists the
    // parent's vertex node, a corner of the octet and so in the chunk's list)
    for (int v = 0; v < 8; ++v) {
      const uint32_t id = nl[int64_t(v) * E + e];
      int lo = 0, hi = nu;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (uniq[mid] < id) lo = mid + 1;
        else hi = mid;
      }
      lnl[int64_t(v) * E + e] = uint16_t(lo < nu && uniq[lo] == id ? lo : 0xffff);
    }
  }
}

__global__ void count_u16_ffff(const uint16_t* __restrict__ a, int64_t n, uint32_t* __restrict__ out) {
  for (int64_t i = gtid(); i < n; i += gstride())
    if (a[i] == 0xffffu) atomicAdd(out, 1u);
}

__global__ void chunk_flag_shared(uint32_t* __restrict__ cnodes, int64_t total, const uint32_t* __restrict__ ncount) {
  for (int64_t i = gtid(); i < total; i += gstride()) {
    const uint32_t id = cnodes[i];
    if (ncount[id] > 1u) cnodes[i] = id | 0x80000000u;
  }
}

dg_status build_chunks(dg_da* da, cudaStream_t s) {
  OctetSet& O = da->octs;
  const int64_t n = O.n;
  const int64_t nq = (n + kOctChunk - 1) / kOctChunk;
  DBuf<uint32_t> count;
  DG_TRY(count.alloc(nq));
  DG_TRY(O.cel.alloc(2 * nq));
  chunk_count<<<unsigned(nq), kChunkThreads, 0, s>>>(n, O.id.p, O.elem.p, count.p, O.cel.p);
  DG_CUDA(cudaGetLastError());
  std::vector<uint32_t> hc(nq), hel(2 * nq);
  DG_CUDA(cudaMemcpyAsync(hc.data(), count.p, 4 * nq, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaMemcpyAsync(hel.data(), O.cel.p, 8 * nq, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> hp(nq + 1, 0);
  uint32_t mx = 0, mr = 0;
  for (int64_t q = 0; q < nq; ++q) {
    hp[q + 1] = hp[q] + hc[q];
    mx = std::max(mx, hc[q]);
    mr = std::max(mr, hel[2 * q + 1]);
  }
  // element offsets are 16-bit: a chunk whose children span more element ids
  // leaves the chunked kernel off for this mesh
  if (mr >= 0xffffu) {
    O.nchunk = 0;
    O.cel.reset();
    return DG_OK;
  }
  DG_TRY(O.cptr.alloc(nq + 1));
  DG_TRY(O.cnodes.alloc(int64_t(hp[nq]) > 0 ? int64_t(hp[nq]) : 1));
  DG_TRY(O.lidx.alloc(27 * n));
  DG_TRY(O.lelem.alloc(8 * n));
  DG_TRY(O.lnl.alloc(8 * da->E));
  DG_CUDA(cudaMemsetAsync(O.lnl.p, 0xff, 2 * 8 * da->E, s));
  DBuf<uint32_t> ncount;
  DG_TRY(ncount.alloc(da->N));
  DG_CUDA(cudaMemsetAsync(ncount.p, 0, 4 * da->N, s));
  DG_CUDA(cudaMemcpyAsync(O.cptr.p, hp.data(), 4 * (nq + 1), cudaMemcpyHostToDevice, s));
  chunk_emit<<<unsigned(nq), kChunkThreads, 0, s>>>(n, O.id.p, O.elem.p, O.cptr.p, O.cel.p, O.cnodes.p, ncount.p,
                                                     O.lidx.p, O.lelem.p, da->nl.p, da->E, O.lnl.p);
  // every node an element lists must be in its chunk's list
  DBuf<uint32_t> miss;
  DG_TRY(miss.alloc(1));
  DG_CUDA(cudaMemsetAsync(miss.p, 0, 4, s));
  count_u16_ffff<<<grid_for(8 * da->E, 256), 256, 0, s>>>(O.lnl.p, 8 * da->E, miss.p);
  uint32_t hmiss = 0;
  DG_CUDA(cudaMemcpyAsync(&hmiss, miss.p, 4, cudaMemcpyDeviceToHost, s));
  chunk_flag_shared<<<grid_for(hp[nq], 256), 256, 0, s>>>(O.cnodes.p, hp[nq], ncount.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  DG_CHECK(!hmiss, DG_EUNBALANCED, "octet chunks: an element's node is missing from its chunk's node list");
  O.nchunk = nq;
  O.max_nodes = mx;
  O.max_erange = mr;
  return DG_OK;
}

}  // namespace

// Per octet one 128-byte record (and a padding octet at index n with no
// children): the 27 lattice node ids, the mask of lattice points without a
// node, the meta word, three words of padding.
__global__ void octet_records(int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oid,
                              uint32_t* __restrict__ rec) {
  for (int64_t o = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; o <= n; o += int64_t(gridDim.x) * blockDim.x) {
    uint32_t* r = rec + o * kOctRec;
    uint32_t none = 0;
    for (int p = 0; p < 27; ++p) {
      const uint32_t id = o < n ? oid[int64_t(p) * n + o] : kNoNode;
      r[p] = id;
      none |= id == kNoNode ? (1u << p) : 0u;
    }
    r[27] = none;
    r[28] = o < n ? ometa[o] : 0u;
    r[29] = r[30] = r[31] = 0u;
  }
}

dg_status build_octets(dg_da* da, cudaStream_t s) {
  const int64_t E = da->E;
  const uint32_t Dp = da->D;
  OctetSet& O = da->octs;
  DBuf<uint64_t> pk, tmp;
  DG_TRY(pk.alloc(E));
  DG_TRY(tmp.alloc(E));
  octet_parent_keys<<<grid_for(E, 256), 256, 0, s>>>(da->ekey.p, E, Dp, pk.p);
  DG_CUDA(cudaGetLastError());
  DG_TRY(radix_sort_u64(pk.p, tmp.p, E, int(3 * Dp + 5), s));
  int64_t n = 0;
  DG_TRY(unique_u64(pk.p, E, &n, s));
  O.n = n;
  DG_TRY(O.meta.alloc(n));
  DG_TRY(O.id.alloc(27 * n));
  DG_TRY(O.elem.alloc(8 * n));
  DBuf<uint32_t> hang, node, err;
  DG_TRY(hang.alloc(n));
  DG_TRY(node.alloc(n));
  DG_TRY(err.alloc(1));
  DG_CUDA(cudaMemsetAsync(O.meta.p, 0, 4 * n, s));
  DG_CUDA(cudaMemsetAsync(O.id.p, 0xff, 4 * 27 * n, s));
  DG_CUDA(cudaMemsetAsync(O.elem.p, 0xff, 4 * 8 * n, s));
  DG_CUDA(cudaMemsetAsync(hang.p, 0, 4 * n, s));
  DG_CUDA(cudaMemsetAsync(node.p, 0, 4 * n, s));
  DG_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
  octet_fill<<<grid_for(E, 256), 256, 0, s>>>(da->ekey.p, E, Dp, da->nl.p, da->meta.p, pk.p, n, O.meta.p, O.id.p,
                                             O.elem.p, hang.p, node.p, err.p);
  octet_corners<<<grid_for(n, 256), 256, 0, s>>>(pk.p, n, Dp, da->nkey.p, da->N, hang.p, node.p, O.id.p, err.p);
  DG_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  DG_CUDA(cudaMemcpyAsync(&herr, err.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  DG_CHECK(!(herr & 1u), DG_EUNBALANCED, "octets: element without its parent entry");
  DG_CHECK(!(herr & 2u), DG_EUNBALANCED, "octets: a lattice point hangs for one child and is a node for another");
  DG_CHECK(!(herr & 4u), DG_EUNBALANCED, "octets: a parent corner needed by a hanging point is not a node");
  DG_TRY(O.rec.alloc((n + 1) * kOctRec));
  octet_records<<<grid_for(n + 1, 256), 256, 0, s>>>(n, O.meta.p, O.id.p, O.rec.p);
  DG_CUDA(cudaGetLastError());
  return build_chunks(da, s);
}

}  // namespace dg
