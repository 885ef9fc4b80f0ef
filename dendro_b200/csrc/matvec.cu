// Matrix-free elemental operators on the GPU (the PETSc MatShell callbacks):
//  * Laplacian + mass, JAC_TYPE2_ELEM_MULT_BLOCK / Jacobian2MatMult
//    (examples/src/backend/omgNeumann.C:468-557),
//  * its diagonal, JAC_TYPE2_ELEM_DIAG_BLOCK (omgNeumann.C:396-465),
//  * 3-dof linear elasticity, ELASTICITY_ELEM_MULT_BLOCK
//    (examples/src/backend/elasticityJac.C:130-230).
//
// The reference multiplies by precomputed tables L[c][t], M[c][t] (8x8) and
// GD[c][t] (24x24) per (child number, element type).  Each table equals
// T^T A T, where A is the reference-cube Q1 matrix and T interpolates the
// element's vertex values from its node values (a hanging vertex takes the
// mean of the parent vertices on its edge or face).  The kernels apply T,
// the tensor-product form of A on [-1,1]^3, then T^T, which needs no tables
// and about 150 flops per scalar element instead of 256.
#include <cstdlib>
#include <cstring>

#include "dg_internal.h"

namespace dg {

namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

// h = 2^-(lev-1) for embedded level lev (omgNeumann.C:470-471).
template <class T>
__device__ __forceinline__ T elem_h(uint32_t lev) {
  return T(__longlong_as_double(int64_t(1023 + 1 - int(lev)) << 52));
}

// 1D reference matrices on [-1,1]: mass M1 = [[2,1],[1,2]]/3, stiffness
// K1 = [[1,-1],[-1,1]]/2, applied along the axis whose vertex bit is B.
template <int B, class T>
__device__ __forceinline__ void mass1(const T (&u)[8], T (&o)[8]) {
  const T third = T(1.0 / 3.0);
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v & B) continue;
    T s = u[v] + u[v | B];
    o[v] = (s + u[v]) * third;
    o[v | B] = (s + u[v | B]) * third;
  }
}
template <int B, class T>
__device__ __forceinline__ void stiff1(const T (&u)[8], T (&o)[8]) {
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v & B) continue;
    T d = (u[v] - u[v | B]) * T(0.5);
    o[v] = d;
    o[v | B] = -d;
  }
}

// r = f1 * K u + f2 * M u with K = K1(x)M1(x)M1 + M1(x)K1(x)M1 + M1(x)M1(x)K1
// and M = M1(x)M1(x)M1 on the reference cube.
template <class T>
__device__ __forceinline__ void lapmass_ref(const T (&u)[8], T f1, T f2, T (&r)[8]) {
  T P[8], Q[8], A[8], B[8];
  mass1<1>(u, P);   // Mx u
  mass1<2>(P, Q);   // My Mx u
  mass1<4>(Q, A);   // Mz My Mx u        (mass)
  stiff1<4>(Q, B);  // Kz My Mx u
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] = f2 * A[v] + f1 * B[v];
  mass1<4>(P, Q);   // Mz Mx u
  stiff1<2>(Q, A);  // Ky Mz Mx u
  mass1<2>(u, P);   // My u
  mass1<4>(P, Q);   // Mz My u
  stiff1<1>(Q, B);  // Kx Mz My u
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] += f1 * (A[v] + B[v]);
}

// Hanging interpolation u_vertex = T u_node, in place.  A hanging vertex i
// takes the mean of the nodes j that differ from i only on the axes where i
// and the child number c differ (2 nodes on an edge, 4 on a face).  All array
// indices are compile-time constants so the values stay in registers.
template <class T>
__device__ __forceinline__ void interp_hanging(T (&u)[8], uint32_t c, uint32_t mask) {
  T un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) un[v] = u[v];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if ((mask >> i) & 1u) {
      const uint32_t keep = ~((uint32_t(i) ^ c)) & 7u;  // axes on which j must equal i
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < 8; ++j) acc += (((uint32_t(j ^ i)) & keep) == 0u) ? un[j] : T(0);
      u[i] = acc * ((__popc(keep) == 2) ? T(0.5) : T(0.25));
    }
  }
}
// r_node = T^T r_vertex, in place.
template <class T>
__device__ __forceinline__ void scatter_hanging(T (&r)[8], uint32_t c, uint32_t mask) {
  T rn[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) rn[v] = ((mask >> v) & 1u) ? T(0) : r[v];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if ((mask >> i) & 1u) {
      const uint32_t keep = ~((uint32_t(i) ^ c)) & 7u;
      const T w = r[i] * ((__popc(keep) == 2) ? T(0.5) : T(0.25));
#pragma unroll
      for (int j = 0; j < 8; ++j) rn[j] += (((uint32_t(j ^ i)) & keep) == 0u) ? w : T(0);
    }
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] = rn[v];
}

// One thread per element: gather, apply, scatter with atomics.  BLOCK and
// MINB set the launch bounds (registers per thread) of each tuned variant.
template <class T, class CT, int BLOCK = 256, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) lapmass_kernel(const uint32_t* __restrict__ nl,
                                                              const uint32_t* __restrict__ meta,
                                                              const CT* __restrict__ ca, const CT* __restrict__ cb,
                                                              int64_t E, const T* __restrict__ x, T* __restrict__ y) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const T h = elem_h<T>(lev);
    const T a = ca ? T(ca[e]) : T(1), b = cb ? T(cb[e]) : T(1);
    const T f1 = a * h / T(2), f2 = b * h * h * h / T(8);
    uint32_t id[8];
    T u[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) id[v] = __ldg(nl + int64_t(v) * E + e);
#pragma unroll
    for (int v = 0; v < 8; ++v) u[v] = __ldg(x + id[v]);
    if (mask) interp_hanging(u, c, mask);
    T r[8];
    lapmass_ref(u, f1, f2, r);
    if (mask) scatter_hanging(r, c, mask);
#pragma unroll
    for (int v = 0; v < 8; ++v) atomicAdd(y + id[v], r[v]);
  }
}

// Tiled variant: a CTA owns kTileElems consecutive elements (Morton order) and
// a window of kWindow consecutive node ids starting at the tile's smallest
// node id.  x over the window is staged in shared memory with coalesced
// loads; element results for window nodes accumulate in shared memory and are
// flushed with one global atomic per touched node.  References outside the
// window (about 8% on log-normal meshes) go straight to global memory.
constexpr int kTileThreads = 256;
constexpr int kTileElems = 512;
constexpr int kWindow = 2048;

template <class T, class CT>
__global__ void __launch_bounds__(kTileThreads) lapmass_tiled_kernel(
    const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta, const CT* __restrict__ ca,
    const CT* __restrict__ cb, int64_t E, int64_t N, const uint32_t* __restrict__ tile_lo, int64_t ntiles,
    const T* __restrict__ x, T* __restrict__ y) {
  __shared__ T xs[kWindow];
  __shared__ T ys[kWindow];
  __shared__ uint32_t touched[kWindow / 32];
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t lo = tile_lo[tile];
    const int64_t wn = (N - int64_t(lo)) < kWindow ? (N - int64_t(lo)) : kWindow;
    for (int i = threadIdx.x; i < kWindow; i += kTileThreads) {
      xs[i] = i < wn ? x[lo + i] : T(0);
      ys[i] = T(0);
    }
    for (int i = threadIdx.x; i < kWindow / 32; i += kTileThreads) touched[i] = 0;
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < kTileElems / kTileThreads; ++k) {
      const int64_t e = tile * kTileElems + k * kTileThreads + threadIdx.x;
      if (e >= E) break;
      const uint32_t m = meta[e];
      const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
      const T h = elem_h<T>(lev);
      const T a = ca ? T(ca[e]) : T(1), b = cb ? T(cb[e]) : T(1);
      const T f1 = a * h / T(2), f2 = b * h * h * h / T(8);
      uint32_t id[8];
      T u[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) id[v] = __ldg(nl + int64_t(v) * E + e);
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const uint32_t o = id[v] - lo;
        u[v] = o < uint32_t(wn) ? xs[o] : __ldg(x + id[v]);
      }
      if (mask) interp_hanging(u, c, mask);
      T r[8];
      lapmass_ref(u, f1, f2, r);
      if (mask) scatter_hanging(r, c, mask);
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const uint32_t o = id[v] - lo;
        if (o < uint32_t(wn)) {
          atomicAdd(ys + o, r[v]);
          atomicOr(touched + (o >> 5), 1u << (o & 31));
        } else {
          atomicAdd(y + id[v], r[v]);
        }
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kWindow; i += kTileThreads)
      if ((touched[i >> 5] >> (i & 31)) & 1u) atomicAdd(y + lo + i, ys[i]);
    __syncthreads();
  }
}

template <class CT>
__global__ void lapmass_diag_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                    const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
                                    double* __restrict__ d) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(lev);
    const double a = ca ? double(ca[e]) : 1.0, b = cb ? double(cb[e]) : 1.0;
    const double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    for (int j = 0; j < 8; ++j) {
      double u[8], r[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) u[v] = v == j ? 1.0 : 0.0;
      if (mask) interp_hanging(u, c, mask);
      lapmass_ref(u, f1, f2, r);
      if (mask) scatter_hanging(r, c, mask);
      atomicAdd(d + nl[int64_t(j) * E + e], r[j]);
    }
  }
}

// Dense assembly of a small level into per-mesh row-major blocks: node r of
// block b = row_blk[r] lands at dense[aoff[b] + (r - off[b]) * n[b] + ...].
template <class CT>
__global__ void lapmass_dense_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                     const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
                                     const uint32_t* __restrict__ row_blk, const int64_t* __restrict__ boff,
                                     const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                                     double* __restrict__ A) {
  for (int64_t t = gtid(); t < E * 8; t += gstride()) {
    int64_t e = t >> 3;
    int j = int(t & 7);
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const double h = elem_h<double>(lev);
    const double a = ca ? double(ca[e]) : 1.0, b = cb ? double(cb[e]) : 1.0;
    const double f1 = a * h / 2.0, f2 = b * h * h * h / 8.0;
    double u[8], r[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) u[v] = v == j ? 1.0 : 0.0;
    if (mask) interp_hanging(u, c, mask);
    lapmass_ref(u, f1, f2, r);
    if (mask) scatter_hanging(r, c, mask);
    const uint32_t col = nl[int64_t(j) * E + e];
    const uint32_t blk = row_blk[col];
    const int64_t o = boff[blk], n = bn[blk];
    double* Ab = A + baoff[blk];
    for (int k = 0; k < 8; ++k)
      atomicAdd(Ab + (int64_t(nl[int64_t(k) * E + e]) - o) * n + (int64_t(col) - o), r[k]);
  }
}

}  // namespace

// Launch shapes tried by the autotuner: one thread per element with
// different block sizes / register caps / grid sizes, and the tiled
// shared-memory form.  The first application on a mesh times each once
// (after one untimed launch) and keeps the fastest for that mesh and
// precision; DG_MATVEC_KERNEL=<index> forces one (testing).
struct MatvecVariant {
  int block, per_sm;  // threads per CTA, CTAs per SM in the grid (0: one thread per element)
  int kind;           // 0 atomic (BLOCK, MINB), 1 tiled
  int minb;
  const char* name;
};
constexpr MatvecVariant kVariants[] = {
    {256, 8, 0, 1, "atomic b256 grid 8/SM"},  {256, 0, 0, 1, "atomic b256 grid E"},
    {256, 8, 0, 4, "atomic b256 minB4"},      {128, 16, 0, 8, "atomic b128 minB8"},
    {512, 4, 0, 2, "atomic b512 minB2"},      {256, 0, 1, 1, "tiled 512 elems / 2048-node window"},
};
constexpr int kNumVariants = int(sizeof(kVariants) / sizeof(kVariants[0]));

template <class T, class CT>
static dg_status launch_variant(int v, const dg_da* da, const CT* ca, const CT* cb, const T* x, T* y,
                                cudaStream_t s) {
  const MatvecVariant& V = kVariants[v];
  const unsigned g = V.per_sm ? grid_for(da->E, V.block, V.per_sm)
                              : unsigned((da->E + V.block - 1) / V.block > 0 ? (da->E + V.block - 1) / V.block : 1);
  if (V.kind == 1) {
    const unsigned gt = unsigned(da->ntiles < int64_t(sm_count()) * 16 ? da->ntiles : int64_t(sm_count()) * 16);
    lapmass_tiled_kernel<T, CT><<<gt > 0 ? gt : 1, kTileThreads, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, da->N,
                                                                      da->tile_lo.p, da->ntiles, x, y);
  } else if (V.block == 256 && V.minb == 1) {
    lapmass_kernel<T, CT, 256, 1><<<g, 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else if (V.block == 256 && V.minb == 4) {
    lapmass_kernel<T, CT, 256, 4><<<g, 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else if (V.block == 128) {
    lapmass_kernel<T, CT, 128, 8><<<g, 128, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  } else {
    lapmass_kernel<T, CT, 512, 2><<<g, 512, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

static int forced_variant() {
  static int v = -2;
  if (v == -2) {
    const char* e = getenv("DG_MATVEC_KERNEL");
    v = -1;
    if (e && *e) {
      if (!strcmp(e, "atomic")) v = 0;
      else if (!strcmp(e, "tiled")) v = kNumVariants - 1;
      else v = atoi(e) % kNumVariants;
    }
  }
  return v;
}

template <class T, class CT>
static dg_status lapmass_launch(const dg_da* da, int& choice, const CT* ca, const CT* cb, const T* x, T* y,
                                cudaStream_t s) {
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
  if (forced_variant() >= 0) return launch_variant<T, CT>(forced_variant(), da, ca, cb, x, y, s);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  DG_CUDA(cudaStreamIsCapturing(s, &cap));
  if (choice < 0 && cap != cudaStreamCaptureStatusNone)  // no timing inside a graph capture
    return launch_variant<T, CT>(0, da, ca, cb, x, y, s);
  if (choice < 0) {
    // autotune: one untimed launch, then per variant the best of two timed
    // launches, each after overwriting a buffer larger than L2 so that the
    // mesh streams from HBM as it does for meshes larger than L2
    cudaEvent_t e0, e1;
    DG_CUDA(cudaEventCreate(&e0));
    DG_CUDA(cudaEventCreate(&e1));
    DBuf<uint8_t> flush;
    const int64_t flush_bytes = int64_t(192) << 20;
    DG_TRY(flush.alloc(flush_bytes));
    float best = 1e30f;
    int bi = 0;
    DG_TRY((launch_variant<T, CT>(0, da, ca, cb, x, y, s)));
    for (int v = 0; v < kNumVariants; ++v) {
      if (kVariants[v].kind == 1 && da->ntiles == 0) continue;
      for (int trial = 0; trial < 2; ++trial) {
        DG_CUDA(cudaMemsetAsync(flush.p, trial + 1, flush_bytes, s));
        DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
        DG_CUDA(cudaEventRecord(e0, s));
        DG_TRY((launch_variant<T, CT>(v, da, ca, cb, x, y, s)));
        DG_CUDA(cudaEventRecord(e1, s));
        DG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        DG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          bi = v;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    choice = bi;
    DG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * da->N, s));
  }
  return launch_variant<T, CT>(choice, da, ca, cb, x, y, s);
}

const char* matvec_variant_name(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].name : "untuned"; }

dg_status lapmass_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  dg_da* da = A->da;
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  return lapmass_launch<double, double>(da, da->tuned_f64, ca, cb, x, y, s);
}

dg_status lapmass_apply_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s) {
  dg_da* da = A->da;
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  return lapmass_launch<float, float>(da, da->tuned_f32, ca, cb, x, y, s);
}

dg_status lapmass_diag(const dg_mat* A, double* d, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * da->N, s));
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  lapmass_diag_kernel<double><<<grid_for(da->E, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, d);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status lapmass_assemble_dense(const dg_mat* A, double* dense, int64_t dense_size, const uint32_t* row_blk,
                                 const int64_t* boff, const int64_t* bn, const int64_t* baoff, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(dense, 0, sizeof(double) * dense_size, s));
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  lapmass_dense_kernel<double><<<grid_for(da->E * 8, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E,
                                                                          row_blk, boff, bn, baoff, dense);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

namespace {

// 1D operators on [-1,1] along the axis with vertex bit B:
// OP 0: mass M1, 1: stiffness K1 = int phi'_k phi'_j, 2: E1 = int phi'_k phi_j,
// 3: E1^T = int phi_k phi'_j.
template <int OP, int B>
__device__ __forceinline__ void op1(const double (&u)[8], double (&o)[8]) {
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    if (v & B) continue;
    const double u0 = u[v], u1 = u[v | B];
    if (OP == 0) {
      const double s = u0 + u1;
      o[v] = (s + u0) * (1.0 / 3.0);
      o[v | B] = (s + u1) * (1.0 / 3.0);
    } else if (OP == 1) {
      const double d = (u0 - u1) * 0.5;
      o[v] = d;
      o[v | B] = -d;
    } else if (OP == 2) {
      const double s = (u0 + u1) * 0.5;
      o[v] = -s;
      o[v | B] = s;
    } else {
      const double d = (u1 - u0) * 0.5;
      o[v] = d;
      o[v | B] = d;
    }
  }
}

// Block (A, B) of the reference-cube grad-div matrix, int d_A phi_k d_B phi_j,
// as a product of three 1D operators; accumulates w * block * u into r.
template <int A, int B>
__device__ __forceinline__ void graddiv_block(const double (&u)[8], double w, double (&r)[8]) {
  constexpr int o0 = (A == 0 && B == 0) ? 1 : (A == 0) ? 2 : (B == 0) ? 3 : 0;
  constexpr int o1 = (A == 1 && B == 1) ? 1 : (A == 1) ? 2 : (B == 1) ? 3 : 0;
  constexpr int o2 = (A == 2 && B == 2) ? 1 : (A == 2) ? 2 : (B == 2) ? 3 : 0;
  double p[8], q[8], t[8];
  op1<o0, 1>(u, p);
  op1<o1, 2>(p, q);
  op1<o2, 4>(q, t);
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] += w * t[v];
}

// y = mu h/2 (K x I3) x + (mu + lambda) h/2 GD x per element; Dirichlet nodes
// contribute nothing (columns skipped) and receive nothing (rows handled by
// elasticity_dirichlet_rows).  x, y are node-major [N][3].
__global__ void __launch_bounds__(128) elasticity_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                                         const uint8_t* __restrict__ dir, int64_t E, double mu, double lam,
                                                         const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const double fac = elem_h<double>(lev) / 2.0;
    uint32_t id[8];
    bool bd[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      id[v] = __ldg(nl + int64_t(v) * E + e);
      bd[v] = __ldg(dir + id[v]) != 0;
    }
    double u0[8], u1[8], u2[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      u0[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]));
      u1[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]) + 1);
      u2[v] = bd[v] ? 0.0 : __ldg(x + 3 * int64_t(id[v]) + 2);
    }
    if (mask) {
      interp_hanging(u0, c, mask);
      interp_hanging(u1, c, mask);
      interp_hanging(u2, c, mask);
    }
    double r0[8], r1[8], r2[8];
    const double wl = mu * fac, wg = (mu + lam) * fac;
    lapmass_ref(u0, wl, 0.0, r0);
    lapmass_ref(u1, wl, 0.0, r1);
    lapmass_ref(u2, wl, 0.0, r2);
    graddiv_block<0, 0>(u0, wg, r0);
    graddiv_block<0, 1>(u1, wg, r0);
    graddiv_block<0, 2>(u2, wg, r0);
    graddiv_block<1, 0>(u0, wg, r1);
    graddiv_block<1, 1>(u1, wg, r1);
    graddiv_block<1, 2>(u2, wg, r1);
    graddiv_block<2, 0>(u0, wg, r2);
    graddiv_block<2, 1>(u1, wg, r2);
    graddiv_block<2, 2>(u2, wg, r2);
    if (mask) {
      scatter_hanging(r0, c, mask);
      scatter_hanging(r1, c, mask);
      scatter_hanging(r2, c, mask);
    }
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      if (bd[v]) continue;
      atomicAdd(y + 3 * int64_t(id[v]), r0[v]);
      atomicAdd(y + 3 * int64_t(id[v]) + 1, r1[v]);
      atomicAdd(y + 3 * int64_t(id[v]) + 2, r2[v]);
    }
  }
}

__global__ void elasticity_dirichlet_rows(const uint8_t* __restrict__ dir, int64_t N, const double* __restrict__ x,
                                          double* __restrict__ y) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) {
      y[3 * i] = x[3 * i];
      y[3 * i + 1] = x[3 * i + 1];
      y[3 * i + 2] = x[3 * i + 2];
    }
}

// Diagonal: the element operator applied to each of the 24 node unit vectors.
__global__ void elasticity_diag_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                       const uint8_t* __restrict__ dir, int64_t E, double mu, double lam,
                                       double* __restrict__ d) {
  for (int64_t t = gtid(); t < E * 24; t += gstride()) {
    const int64_t e = t / 24;
    const int j = int(t - e * 24), jn = j / 3, jd = j % 3;
    const uint32_t m = meta[e];
    const uint32_t lev = meta_lev(m), c = meta_cnum(m), mask = meta_mask(m);
    const uint32_t node = nl[int64_t(jn) * E + e];
    if (dir[node]) continue;
    const double fac = elem_h<double>(lev) / 2.0;
    double u[3][8], r[3][8];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int v = 0; v < 8; ++v) u[a][v] = (a == jd && v == jn) ? 1.0 : 0.0;
    if (mask)
      for (int a = 0; a < 3; ++a) interp_hanging(u[a], c, mask);
    const double wl = mu * fac, wg = (mu + lam) * fac;
    for (int a = 0; a < 3; ++a) lapmass_ref(u[a], wl, 0.0, r[a]);
    graddiv_block<0, 0>(u[0], wg, r[0]);
    graddiv_block<0, 1>(u[1], wg, r[0]);
    graddiv_block<0, 2>(u[2], wg, r[0]);
    graddiv_block<1, 0>(u[0], wg, r[1]);
    graddiv_block<1, 1>(u[1], wg, r[1]);
    graddiv_block<1, 2>(u[2], wg, r[1]);
    graddiv_block<2, 0>(u[0], wg, r[2]);
    graddiv_block<2, 1>(u[1], wg, r[2]);
    graddiv_block<2, 2>(u[2], wg, r[2]);
    if (mask)
      for (int a = 0; a < 3; ++a) scatter_hanging(r[a], c, mask);
    atomicAdd(d + 3 * int64_t(node) + jd, r[jd][jn]);
  }
}

__global__ void set_dirichlet_diag(const uint8_t* __restrict__ dir, int64_t N, double* __restrict__ d) {
  for (int64_t i = gtid(); i < N; i += gstride())
    if (dir[i]) d[3 * i] = d[3 * i + 1] = d[3 * i + 2] = 1.0;
}

}  // namespace

dg_status elasticity_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * 3 * da->N, s));
  elasticity_kernel<<<grid_for(da->E, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E, A->mu,
                                                               A->lam, x, y);
  elasticity_dirichlet_rows<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status elasticity_diag(const dg_mat* A, double* d, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * 3 * da->N, s));
  elasticity_diag_kernel<<<grid_for(da->E * 24, 128, 16), 128, 0, s>>>(da->nl.p, da->meta.p, A->dirichlet.p, da->E,
                                                                         A->mu, A->lam, d);
  set_dirichlet_diag<<<grid_for(da->N, 256), 256, 0, s>>>(A->dirichlet.p, da->N, d);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg
