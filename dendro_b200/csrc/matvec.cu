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

// Hanging interpolation u_vertex = T u_node, in place.
template <class T>
__device__ __forceinline__ void interp_hanging(T (&u)[8], uint32_t c, uint32_t mask) {
  T un[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) un[v] = u[v];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (!((mask >> i) & 1u)) continue;
    uint32_t mid = (uint32_t(i) ^ c) & 7u;
    T acc = T(0);
    int cnt = 0;
    for (uint32_t sub = mid;; sub = (sub - 1) & mid) {  // all subsets of mid
      acc += un[i ^ sub];
      ++cnt;
      if (!sub) break;
    }
    u[i] = acc * (cnt == 2 ? T(0.5) : T(0.25));
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
    if (!((mask >> i) & 1u)) continue;
    uint32_t mid = (uint32_t(i) ^ c) & 7u;
    T w = r[i] * (__popc(mid) == 1 ? T(0.5) : T(0.25));
    for (uint32_t sub = mid;; sub = (sub - 1) & mid) {
      rn[i ^ sub] += w;
      if (!sub) break;
    }
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] = rn[v];
}

// One thread per element: gather, apply, scatter with atomics.
template <class T, class CT>
__global__ void __launch_bounds__(256) lapmass_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                                      const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E,
                                                      const T* __restrict__ x, T* __restrict__ y) {
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

// Dense assembly of a small level (row-major N x N).
template <class CT>
__global__ void lapmass_dense_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta,
                                     const CT* __restrict__ ca, const CT* __restrict__ cb, int64_t E, int64_t N,
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
    for (int k = 0; k < 8; ++k) atomicAdd(A + int64_t(nl[int64_t(k) * E + e]) * N + col, r[k]);
  }
}

}  // namespace

dg_status lapmass_apply_f64(const dg_mat* A, const double* x, double* y, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * da->N, s));
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  lapmass_kernel<double, double><<<grid_for(da->E, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status lapmass_apply_f32(const dg_mat* A, const float* x, float* y, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * da->N, s));
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  lapmass_kernel<float, float><<<grid_for(da->E, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E, x, y);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
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

dg_status lapmass_assemble_dense(const dg_mat* A, double* dense, cudaStream_t s) {
  const dg_da* da = A->da;
  DG_CUDA(cudaMemsetAsync(dense, 0, sizeof(double) * da->N * da->N, s));
  const double* ca = A->has_coef ? A->coef.p : nullptr;
  const double* cb = A->has_coef ? A->coef.p + da->E : nullptr;
  lapmass_dense_kernel<double><<<grid_for(da->E * 8, 256, 8), 256, 0, s>>>(da->nl.p, da->meta.p, ca, cb, da->E,
                                                                          da->N, dense);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status elasticity_apply_f64(const dg_mat*, const double*, double*, cudaStream_t) {
  set_error(__FILE__, __LINE__, "elasticity operator not built yet");
  return DG_ENOTIMPL;
}
dg_status elasticity_diag(const dg_mat*, double*, cudaStream_t) {
  set_error(__FILE__, __LINE__, "elasticity operator not built yet");
  return DG_ENOTIMPL;
}

}  // namespace dg
