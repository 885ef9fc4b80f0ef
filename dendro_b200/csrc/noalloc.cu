// FP64 inner product that performs no device allocation.
//
// dg_vec_dot allocates its block partial sums with cudaMalloc on every call.
// Some callers cannot do that: a KSP convergence test or monitor that runs
// every iteration inside a solver whose device memory belongs to another
// allocator (a caching pool that has already reserved the free HBM, or a
// process capped by an MPS memory limit), and loops that cannot afford the
// device-wide synchronisation that cudaMalloc / cudaFree imply.  This variant
// keeps its partial sums in a fixed array in the library's own device memory.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds kNoAllocMaxPartials doubles (512 KiB) of it until the process
// exits.  Host code must not pass the symbol itself to a kernel -- on the
// host it is only a stand-in, not a device address -- so the device address
// is looked up with cudaGetSymbolAddress once per device (on that device's
// first call, with the device current) and that pointer is what the kernels
// receive.
#include <mutex>

#include "dg_internal.h"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int64_t kNoAllocChunk = 4096;        // elements reduced by one block
constexpr int kNoAllocMaxPartials = 65536;      // one partial sum per block
constexpr int64_t kNoAllocMaxN = kNoAllocChunk * kNoAllocMaxPartials;  // 268,435,456
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxPartials];

__device__ __forceinline__ double noalloc_block_sum(double v) {
  __shared__ double ws[kNoAllocThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  v = 0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (kNoAllocThreads / 32) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Block b writes the sum over elements [b*chunk, (b+1)*chunk) to partial[b];
// every slot that the second kernel reads is written first, so the array
// never needs clearing between calls.
__global__ void __launch_bounds__(kNoAllocThreads)
noalloc_dot_chunks(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                   double* __restrict__ partial) {
  const int64_t base = int64_t(blockIdx.x) * kNoAllocChunk;
  double v = 0;
  for (int64_t i = threadIdx.x; i < kNoAllocChunk; i += kNoAllocThreads) {
    const int64_t k = base + i;
    if (k < n) v += x[k] * y[k];
  }
  v = noalloc_block_sum(v);
  if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

// One block adds the partial sums in a fixed order (deterministic result).
__global__ void __launch_bounds__(kNoAllocThreads)
noalloc_sum_partials(const double* __restrict__ partial, int nb, double* __restrict__ out) {
  double v = 0;
  for (int i = threadIdx.x; i < nb; i += kNoAllocThreads) v += partial[i];
  v = noalloc_block_sum(v);
  if (threadIdx.x == 0) *out = v;
}

std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_partials on the current device (looked up once).
// The address belongs to the device's primary context at the time of the
// lookup: cudaDeviceReset destroys that context and the module holding the
// array, after which the cached address is stale, so a process that resets a
// device must not call dg_vec_dot_noalloc on it again.
dg_status noalloc_scratch(double** out) {
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CHECK(dev >= 0 && dev < kMaxDevices, DG_EINVAL, "vec_dot_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      dg::set_error(__FILE__, __LINE__, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return DG_ECUDA;
    }
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_addr[dev];
  return DG_OK;
}

}  // namespace

extern "C" dg_status dg_vec_dot_noalloc(const double* x, const double* y, int64_t n, double* result,
                                        void* stream) {
  DG_CHECK(result && n >= 0 && (n == 0 || (x && y)), DG_EINVAL, "vec_dot_noalloc: bad arguments");
  DG_CHECK(n <= kNoAllocMaxN, DG_EINVAL,
           "vec_dot_noalloc: n exceeds 268435456 elements (65536 partial sums of 4096 elements); "
           "use dg_vec_dot for longer vectors");
  double* partial = nullptr;
  DG_TRY(noalloc_scratch(&partial));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int nb = int((n + kNoAllocChunk - 1) / kNoAllocChunk);
  if (nb > 0) noalloc_dot_chunks<<<nb, kNoAllocThreads, 0, s>>>(x, y, n, partial);
  noalloc_sum_partials<<<1, kNoAllocThreads, 0, s>>>(partial, nb, result);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
