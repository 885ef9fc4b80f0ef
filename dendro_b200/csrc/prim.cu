// Device-wide primitives: exclusive scan, LSD radix sort of 64-bit keys,
// adjacent-duplicate removal.  Hand-written; no CUB/Thrust on the path.
#include "dg_internal.h"

namespace dg {

namespace {

constexpr int kScanBlock = 1024;  // elements per scan block (256 threads x 4)

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-level exclusive scan of 4 items per thread (256 threads).
__device__ void block_scan4(uint32_t (&v)[4], uint32_t& block_total) {
  __shared__ uint32_t warp_sums[8];
  uint32_t t0 = v[0], t1 = t0 + v[1], t2 = t1 + v[2], t3 = t2 + v[3];
  uint32_t incl = warp_incl_scan(t3);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < 8 ? warp_sums[lane] : 0;
    uint32_t wi = warp_incl_scan(w);
    if (lane < 8) warp_sums[lane] = wi - w;
  }
  __syncthreads();
  uint32_t base = warp_sums[wid] + (incl - t3);
  block_total = 0;
  v[3] = base + t2;
  v[2] = base + t1;
  v[1] = base + t0;
  v[0] = base;
}

__global__ void scan_block_sums(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums) {
  int64_t base = int64_t(blockIdx.x) * kScanBlock + threadIdx.x * 4;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (base + i < n) s += in[base + i];
  // block reduce
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ uint32_t ws[8];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int i = 0; i < 8; ++i) t += ws[i];
    sums[blockIdx.x] = t;
  }
}

__global__ void scan_apply(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t n,
                           const uint32_t* __restrict__ block_off) {
  int64_t base = int64_t(blockIdx.x) * kScanBlock + threadIdx.x * 4;
  uint32_t v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = (base + i < n) ? in[base + i] : 0u;
  uint32_t tot;
  block_scan4(v, tot);
  uint32_t off = block_off ? block_off[blockIdx.x] : 0u;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (base + i < n) out[base + i] = v[i] + off;
}

// ------------------------------------------------------------ radix sort --
constexpr int kRadixBits = 8;
constexpr int kBins = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;  // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void __launch_bounds__(kSortThreads)
radix_hist(const uint64_t* __restrict__ keys, int64_t n, int shift, uint32_t* __restrict__ hist, int nblocks) {
  __shared__ uint32_t h[kBins];
  for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int64_t base = int64_t(blockIdx.x) * kSortTile;
  for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
    int64_t k = base + i;
    if (k < n) atomicAdd(&h[(keys[k] >> shift) & (kBins - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kBins; i += blockDim.x) hist[int64_t(i) * nblocks + blockIdx.x] = h[i];
}

// Stable scatter.  Warp w owns keys [base + w*512, base + (w+1)*512) in
// slot-major, lane-minor order; ranks within the warp come from
// __match_any_sync, and per-(warp, digit) counters give the warp offsets.
__global__ void __launch_bounds__(kSortThreads)
radix_scatter(const uint64_t* __restrict__ in, uint64_t* __restrict__ out, int64_t n, int shift,
              const uint32_t* __restrict__ offs, int nblocks) {
  __shared__ uint32_t cnt[kSortThreads / 32][kBins];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < (kSortThreads / 32) * kBins; i += blockDim.x) (&cnt[0][0])[i] = 0;
  __syncthreads();
  int64_t base = int64_t(blockIdx.x) * kSortTile + int64_t(wid) * (kSortItems * 32);
  uint64_t key[kSortItems];
  uint32_t rank[kSortItems];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int s = 0; s < kSortItems; ++s) {
    int64_t k = base + s * 32 + lane;
    bool valid = k < n;
    key[s] = valid ? in[k] : ~0ull;
    uint32_t d = valid ? uint32_t((key[s] >> shift) & (kBins - 1)) : uint32_t(kBins);  // kBins = invalid
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t pre = (d < kBins) ? cnt[wid][d] : 0u;
    __syncwarp();
    int leader = __ffs(peers) - 1;
    if (lane == leader && d < kBins) cnt[wid][d] = pre + __popc(peers);
    __syncwarp();
    rank[s] = pre + __popc(peers & lt);
  }
  __syncthreads();
  // exclusive prefix over warps for each digit, plus the global block offset
  for (int d = threadIdx.x; d < kBins; d += blockDim.x) {
    uint32_t run = offs[int64_t(d) * nblocks + blockIdx.x];
    for (int w = 0; w < kSortThreads / 32; ++w) {
      uint32_t c = cnt[w][d];
      cnt[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < kSortItems; ++s) {
    int64_t k = base + s * 32 + lane;
    if (k < n) {
      uint32_t d = uint32_t((key[s] >> shift) & (kBins - 1));
      out[cnt[wid][d] + rank[s]] = key[s];
    }
  }
}

__global__ void mark_unique(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    flag[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}
__global__ void scatter_unique(const uint64_t* __restrict__ k, int64_t n, const uint32_t* __restrict__ flag,
                               const uint32_t* __restrict__ pos, uint64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (flag[i]) out[pos[i]] = k[i];
}

}  // namespace

dg_status scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, cudaStream_t s) {
  if (n <= 0) {
    if (total) *total = 0;
    return DG_OK;
  }
  DG_CHECK(n < (int64_t(1) << 31), DG_EINVAL, "scan: too many elements");
  int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  uint32_t last_in = 0;
  if (total) DG_CUDA(cudaMemcpyAsync(&last_in, in + n - 1, 4, cudaMemcpyDeviceToHost, s));
  if (nb == 1) {
    scan_apply<<<1, 256, 0, s>>>(in, out, n, nullptr);
  } else {
    DBuf<uint32_t> sums;
    DG_TRY(sums.alloc(nb));
    scan_block_sums<<<unsigned(nb), 256, 0, s>>>(in, n, sums.p);
    DG_TRY(scan_u32(sums.p, sums.p, nb, nullptr, s));
    scan_apply<<<unsigned(nb), 256, 0, s>>>(in, out, n, sums.p);
    DG_CUDA(cudaGetLastError());
    if (total) {
      uint32_t last_out = 0;
      DG_CUDA(cudaMemcpyAsync(&last_out, out + n - 1, 4, cudaMemcpyDeviceToHost, s));
      DG_CUDA(cudaStreamSynchronize(s));
      *total = last_out + last_in;
    }
    // `sums` is released when this scope ends: finish the work that reads it first
    DG_CUDA(cudaStreamSynchronize(s));
    return DG_OK;
  }
  DG_CUDA(cudaGetLastError());
  if (total) {
    uint32_t last_out = 0;
    DG_CUDA(cudaMemcpyAsync(&last_out, out + n - 1, 4, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    *total = last_out + last_in;
  }
  return DG_OK;
}

dg_status radix_sort_u64(uint64_t* keys, uint64_t* tmp, int64_t n, int bits, cudaStream_t s, int start_bit) {
  if (n <= 1) return DG_OK;
  DG_CHECK(n < (int64_t(1) << 31), DG_EINVAL, "radix sort: too many keys");
  int nblocks = int((n + kSortTile - 1) / kSortTile);
  DBuf<uint32_t> hist;
  DG_TRY(hist.alloc(int64_t(kBins) * nblocks));
  int passes = (bits + kRadixBits - 1) / kRadixBits;
  uint64_t* src = keys;
  uint64_t* dst = tmp;
  for (int p = 0; p < passes; ++p) {
    int shift = start_bit + p * kRadixBits;
    radix_hist<<<nblocks, kSortThreads, 0, s>>>(src, n, shift, hist.p, nblocks);
    DG_TRY(scan_u32(hist.p, hist.p, int64_t(kBins) * nblocks, nullptr, s));
    radix_scatter<<<nblocks, kSortThreads, 0, s>>>(src, dst, n, shift, hist.p, nblocks);
    DG_CUDA(cudaGetLastError());
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  if (src != keys) DG_CUDA(cudaMemcpyAsync(keys, src, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
  DG_CUDA(cudaStreamSynchronize(s));
  return DG_OK;
}

dg_status unique_u64(uint64_t* keys, int64_t n, int64_t* n_out, cudaStream_t s) {
  if (n <= 1) {
    *n_out = n;
    return DG_OK;
  }
  DBuf<uint32_t> flag, pos;
  DBuf<uint64_t> out;
  DG_TRY(flag.alloc(n));
  DG_TRY(pos.alloc(n));
  DG_TRY(out.alloc(n));
  unsigned g = grid_for(n, 256);
  mark_unique<<<g, 256, 0, s>>>(keys, n, flag.p);
  uint32_t total = 0;
  DG_TRY(scan_u32(flag.p, pos.p, n, &total, s));
  scatter_unique<<<g, 256, 0, s>>>(keys, n, flag.p, pos.p, out.p);
  DG_CUDA(cudaMemcpyAsync(keys, out.p, sizeof(uint64_t) * total, cudaMemcpyDeviceToDevice, s));
  DG_CUDA(cudaStreamSynchronize(s));
  *n_out = total;
  return DG_OK;
}

}  // namespace dg
