// Multigrid hierarchy and solver on the GPU (ot::DAMG):
//  * levels by coarsenOctree + balanceOctree until the requested count or a
//    level below 500 octants (DAMGCreateAndSetDA, src/omg/omg.C:1306-1420);
//  * coarse coefficients copied or averaged from the 8 children
//    (ASSIGN_MAT_PROP_FINE_TO_COARSE_ELEM_BLOCK, omgNeumann.C:73-113);
//  * prolongation P = the coarse conforming FE function at the fine nodes,
//    restriction R = P^T (prolongMatVecType1 / restrictMatVecType1,
//    src/omg/ProlongMatVec.C:154-284, RestrictMatVec.C:486-619);
//  * V(nu_pre, nu_post) cycle with Richardson(omega)+Jacobi smoothing and a
//    dense FP64 direct coarse solve, inside CG (bin/options:50-53,182-207).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include <type_traits>

#include "dg_internal.h"

#include <cuda_bf16.h>

namespace dg {
dg_status node_boundary_flags(const dg_da* da, uint8_t* d_out, cudaStream_t s);
dg_status convert_f64_to_f32(const double* a, float* b, int64_t n, cudaStream_t s);
dg_status smoother_node_data(const dg_da* da, const float* dinv32, float* refs, float* hang, float* dlogbar,
                             cudaStream_t s);
dg_status mlp_smooth_step(const float* params, const dg_da* da, const float* r, float* s2, const float* dinv32,
                          float dlogbar, float level_feat, const float* hang, const float* inv_refs, float* nsum,
                          float* nmax, float* x, cudaStream_t s);
dg_status mlp_features_f64(const dg_da* da, const double* r, float* s2, const float* dinv32, float dlogbar,
                           float level_feat, const float* hang, const float* inv_refs, float* nsum, float* nmax,
                           float* F, float* scale_out, cudaStream_t s);
}  // namespace dg

using namespace dg;

namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

__device__ __forceinline__ int64_t lower_bound(const uint64_t* __restrict__ a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;  // first index with a[i] >= key
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int64_t max_lower_bound(const uint64_t* __restrict__ a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;  // first index with a[i] > key
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo - 1;
}

// ---------------------------------------------------------- coefficients --
__global__ void coarse_coef_kernel(const uint64_t* __restrict__ fk, int64_t Ef, const double* __restrict__ fa,
                                   const double* __restrict__ fb, const uint64_t* __restrict__ ck, int64_t Ec,
                                   double* __restrict__ ca, double* __restrict__ cb, uint32_t* __restrict__ err) {
  for (int64_t e = gtid(); e < Ec; e += gstride()) {
    uint64_t m = okey_m(ck[e]);
    uint32_t l = okey_l(ck[e]);
    int64_t f = lower_bound(fk, Ef, okey(m, 0));  // first fine element anchored at or after m
    if (f >= Ef || okey_m(fk[f]) != m) {
      atomicOr(err, 1u);
      continue;
    }
    if (okey_l(fk[f]) == l) {
      ca[e] = fa[f];
      cb[e] = fb[f];
    } else {
      double a = 0, b = 0;
      for (int k = 0; k < 8 && f + k < Ef; ++k) {
        a += fa[f + k];
        b += fb[f + k];
      }
      ca[e] = a / 8.0;
      cb[e] = b / 8.0;
    }
  }
}

// Coarse elements split into 8 fine children whose coefficients differ by more
// than tol relative to their maximum (a or b): JAC_TYPE3_MULT_BLOCK's test
// (examples/src/backend/omgJac.C:2167-2207, -tolToCoarsenMatProp default 1e-12).
// flag[e] = 1 for those, with the children's a, b in child[16 e ..].
__global__ void type1_detect_kernel(const uint64_t* __restrict__ fk, int64_t Ef, const double* __restrict__ fa,
                                    const double* __restrict__ fb, const uint64_t* __restrict__ ck, int64_t Ec,
                                    double tol, uint8_t* __restrict__ flag, double* __restrict__ child) {
  for (int64_t e = gtid(); e < Ec; e += gstride()) {
    const uint64_t m = okey_m(ck[e]);
    const int64_t f = lower_bound(fk, Ef, okey(m, 0));
    flag[e] = 0;
    if (f + 8 > Ef || okey_m(fk[f]) != m || okey_l(fk[f]) == okey_l(ck[e])) continue;
    double mx1 = fa[f], mn1 = fa[f], mx2 = fb[f], mn2 = fb[f];
    for (int k = 1; k < 8; ++k) {
      mx1 = fmax(mx1, fa[f + k]);
      mn1 = fmin(mn1, fa[f + k]);
      mx2 = fmax(mx2, fb[f + k]);
      mn2 = fmin(mn2, fb[f + k]);
    }
    if (mx1 - mn1 <= tol * mx1 && mx2 - mn2 <= tol * mx2) continue;
    flag[e] = 1;
    for (int k = 0; k < 8; ++k) {
      child[16 * e + k] = fa[f + k];
      child[16 * e + 8 + k] = fb[f + k];
    }
  }
}
__global__ void gather16(const double* __restrict__ src, const uint32_t* __restrict__ idx, int64_t n,
                         double* __restrict__ dst) {
  for (int64_t i = gtid(); i < 16 * n; i += gstride()) dst[i] = src[16 * int64_t(idx[i / 16]) + i % 16];
}
__global__ void zero_elems(double* __restrict__ coef, int64_t E, const uint32_t* __restrict__ idx, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    coef[idx[i]] = 0.0;
    coef[E + idx[i]] = 0.0;
  }
}

// concatenation helpers for batches of meshes
__global__ void copy_add_u32(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, int64_t n, uint32_t add) {
  for (int64_t i = gtid(); i < n; i += gstride()) dst[i] = src[i] + add;
}
__global__ void fill_u16(uint16_t* __restrict__ d, int64_t n0, int64_t n1, uint16_t v) {
  for (int64_t i = n0 + gtid(); i < n1; i += gstride()) d[i] = v;
}
// per-mesh squared norms (acc zeroed by the caller), one shared slot per mesh
__global__ void seg_sqnorm(const double* __restrict__ r, int64_t n, const uint16_t* __restrict__ node_mesh, int nmesh,
                           double* __restrict__ acc) {
  extern __shared__ double sh[];
  for (int i = threadIdx.x; i < nmesh; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (int64_t i = gtid(); i < n; i += gstride()) atomicAdd(sh + node_mesh[i], r[i] * r[i]);
  __syncthreads();
  for (int i = threadIdx.x; i < nmesh; i += blockDim.x)
    if (sh[i] != 0.0) atomicAdd(acc + i, sh[i]);
}

// ----------------------------------------------------------- prolongation --
// Weights of the coarse element holding fine node f: the 8 trilinear values
// at the node, mapped through T^T to the element's node slots.
__device__ __forceinline__ bool prolong_row(const uint64_t* __restrict__ fnk, int64_t f, const uint64_t* __restrict__ cek,
                                            int64_t Ec, const uint32_t* __restrict__ cmeta, uint32_t top, uint32_t Dp,
                                            int64_t& e, double (&w)[8]) {
  uint32_t px, py, pz;
  demorton(fnk[f], px, py, pz);
  uint32_t qx = px == top ? px - 1 : px, qy = py == top ? py - 1 : py, qz = pz == top ? pz - 1 : pz;
  e = max_lower_bound(cek, Ec, okey(morton(qx, qy, qz), 31));
  if (e < 0) return false;
  uint32_t ox, oy, oz;
  demorton(okey_m(cek[e]), ox, oy, oz);
  uint32_t s = 1u << (Dp - okey_l(cek[e]));
  if (qx < ox || qy < oy || qz < oz || qx >= ox + s || qy >= oy + s || qz >= oz + s) return false;
  double inv = 1.0 / double(s);
  double lx = double(px - ox) * inv, ly = double(py - oy) * inv, lz = double(pz - oz) * inv;
  double phi[8];
#pragma unroll
  for (int v = 0; v < 8; ++v)
    phi[v] = ((v & 1) ? lx : 1 - lx) * ((v & 2) ? ly : 1 - ly) * ((v & 4) ? lz : 1 - lz);
  uint32_t m = cmeta[e], c = meta_cnum(m), mask = meta_mask(m);
#pragma unroll
  for (int v = 0; v < 8; ++v) w[v] = ((mask >> v) & 1u) ? 0.0 : phi[v];
  for (int i = 0; i < 8; ++i) {
    if (!((mask >> i) & 1u)) continue;
    uint32_t mid = (uint32_t(i) ^ c) & 7u;
    double wi = phi[i] * (__popc(mid) == 1 ? 0.5 : 0.25);
    for (uint32_t sub = mid;; sub = (sub - 1) & mid) {
      w[i ^ sub] += wi;
      if (!sub) break;
    }
  }
  return true;
}

__global__ void prolong_count(const uint64_t* __restrict__ fnk, int64_t Nf, const uint64_t* __restrict__ cek, int64_t Ec,
                              const uint32_t* __restrict__ cmeta, uint32_t top, uint32_t Dp, uint32_t* __restrict__ cnt,
                              uint32_t* __restrict__ err) {
  for (int64_t f = gtid(); f < Nf; f += gstride()) {
    int64_t e;
    double w[8];
    uint32_t c = 0;
    if (!prolong_row(fnk, f, cek, Ec, cmeta, top, Dp, e, w)) {
      atomicOr(err, 1u);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) c += w[j] != 0.0;
    }
    cnt[f] = c;
  }
}

__global__ void prolong_fill(const uint64_t* __restrict__ fnk, int64_t Nf, const uint64_t* __restrict__ cek, int64_t Ec,
                             const uint32_t* __restrict__ cmeta, const uint32_t* __restrict__ cnl, uint32_t top,
                             uint32_t Dp, const uint32_t* __restrict__ ptr, uint32_t* __restrict__ col,
                             double* __restrict__ val) {
  for (int64_t f = gtid(); f < Nf; f += gstride()) {
    int64_t e;
    double w[8];
    if (!prolong_row(fnk, f, cek, Ec, cmeta, top, Dp, e, w)) continue;
    uint32_t p = ptr[f];
    for (int j = 0; j < 8; ++j)
      if (w[j] != 0.0) {
        col[p] = cnl[int64_t(j) * Ec + e];
        val[p] = w[j];
        ++p;
      }
  }
}

// xf += P xc
template <class T>
__global__ void prolong_add(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                            const T* __restrict__ val, int64_t Nf, const T* __restrict__ xc, T* __restrict__ xf) {
  #pragma unroll 4
  for (int64_t f = gtid(); f < Nf; f += gstride()) {
    T s = 0;
    for (uint32_t k = ptr[f]; k < ptr[f + 1]; ++k) s += val[k] * xc[col[k]];
    xf[f] += s;
  }
}

// rc = R rf with R = P^T stored by coarse rows (a gather: no atomics, and the
// sum order is the same on every run)
template <class T>
__global__ void restrict_gather(const uint32_t* __restrict__ rptr, const uint32_t* __restrict__ rcol,
                                const T* __restrict__ rval, int64_t Nc, const T* __restrict__ rf,
                                T* __restrict__ rc) {
  for (int64_t c = gtid(); c < Nc; c += gstride()) {
    T acc = T(0);
    for (uint32_t k = rptr[c]; k < rptr[c + 1]; ++k) acc += rval[k] * rf[rcol[k]];
    rc[c] = acc;
  }
}
// The same two products with the weights as 8-bit codes k = 128 w.  The
// weights are dyadic (trilinear interpolation at a coarse element's corners,
// edge midpoints, face centres and centre, with the hanging corners' halves
// and quarters folded in), so k is exact; code * x is w * x scaled by 128
// exactly, every partial sum is the uncoded one scaled by 128, and the final
// scaling by 1/128 gives the uncoded result bit for bit while each entry
// moves 5 bytes instead of 12 (FP64) or 8 (FP32).
constexpr double kWeightCode = 128.0;
template <class T>
__global__ void prolong_add_coded(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                  const uint8_t* __restrict__ code, int64_t Nf, const T* __restrict__ xc,
                                  T* __restrict__ xf) {
  #pragma unroll 4
  for (int64_t f = gtid(); f < Nf; f += gstride()) {
    T s = 0;
    for (uint32_t k = ptr[f]; k < ptr[f + 1]; ++k) s += T(code[k]) * xc[col[k]];
    xf[f] += s * T(1.0 / kWeightCode);
  }
}
template <class T>
__global__ void restrict_gather_coded(const uint32_t* __restrict__ rptr, const uint32_t* __restrict__ rcol,
                                      const uint8_t* __restrict__ code, int64_t Nc, const T* __restrict__ rf,
                                      T* __restrict__ rc) {
  for (int64_t c = gtid(); c < Nc; c += gstride()) {
    T acc = T(0);
    for (uint32_t k = rptr[c]; k < rptr[c + 1]; ++k) acc += T(code[k]) * rf[rcol[k]];
    rc[c] = acc * T(1.0 / kWeightCode);
  }
}
// k = 128 w for every weight; flags a weight that has no exact code.
__global__ void weight_codes(const double* __restrict__ w, int64_t n, uint8_t* __restrict__ code,
                             uint32_t* __restrict__ bad) {
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const double k = w[i] * kWeightCode;
    const bool ok = k >= 0.0 && k <= 255.0 && k == floor(k);
    if (!ok) atomicOr(bad, 1u);
    code[i] = ok ? uint8_t(k) : uint8_t(0);
  }
}
// The dof-3 forms: the scalar transfer applied to each of the 3 interleaved
// components (node-major [N][3]), as the reference's transfer loops apply
// the same R entry to every dof (RestrictMatVec.C:109-115, ProlongMatVec.C).
__global__ void prolong_add3(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                             const double* __restrict__ val, int64_t Nf, const double* __restrict__ xc,
                             double* __restrict__ xf) {
  for (int64_t f = gtid(); f < Nf; f += gstride()) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (uint32_t k = ptr[f]; k < ptr[f + 1]; ++k) {
      const double w = val[k];
      const int64_t c = 3 * int64_t(col[k]);
      s0 += w * xc[c];
      s1 += w * xc[c + 1];
      s2 += w * xc[c + 2];
    }
    xf[3 * f] += s0;
    xf[3 * f + 1] += s1;
    xf[3 * f + 2] += s2;
  }
}
__global__ void restrict_gather3(const uint32_t* __restrict__ rptr, const uint32_t* __restrict__ rcol,
                                 const double* __restrict__ rval, int64_t Nc, const double* __restrict__ rf,
                                 double* __restrict__ rc) {
  for (int64_t c = gtid(); c < Nc; c += gstride()) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (uint32_t k = rptr[c]; k < rptr[c + 1]; ++k) {
      const double w = rval[k];
      const int64_t f = 3 * int64_t(rcol[k]);
      s0 += w * rf[f];
      s1 += w * rf[f + 1];
      s2 += w * rf[f + 2];
    }
    rc[3 * c] = s0;
    rc[3 * c + 1] = s1;
    rc[3 * c + 2] = s2;
  }
}
// x += omega dinv (b - t), elementwise (the dof-3 sweep after the operator)
__global__ void jacobi_update(double* __restrict__ x, const double* __restrict__ b, const double* __restrict__ dinv,
                              const double* __restrict__ t, double omega, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) x[i] += omega * dinv[i] * (b[i] - t[i]);
}
__global__ void residual_update(const double* __restrict__ b, const double* __restrict__ t, double* __restrict__ r,
                                int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) r[i] = b[i] - t[i];
}

// transpose of P: keys (coarse column << 32 | entry index) and counts per column
__global__ void ptrans_keys(const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col, int64_t Nf,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ frow, uint32_t* __restrict__ cnt) {
  for (int64_t f = gtid(); f < Nf; f += gstride())
    for (uint32_t k = ptr[f]; k < ptr[f + 1]; ++k) {
      keys[k] = (uint64_t(col[k]) << 32) | k;
      frow[k] = uint32_t(f);
      atomicAdd(cnt + col[k], 1u);
    }
}
__global__ void ptrans_fill(const uint64_t* __restrict__ keys, int64_t nnz, const uint32_t* __restrict__ frow,
                            const double* __restrict__ pval, uint32_t* __restrict__ rcol,
                            double* __restrict__ rval) {
  for (int64_t j = gtid(); j < nnz; j += gstride()) {
    const uint32_t k = uint32_t(keys[j] & 0xffffffffu);
    rcol[j] = frow[k];
    rval[j] = pval[k];
  }
}

// --------------------------------------------------------------- smoother --
// x = omega dinv b on 16-byte chunks (4 floats or 2 doubles; level vectors
// are whole allocations, so 16-byte aligned); the remainder by thread 0.
template <class T>
__global__ void jacobi_first(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv, T omega,
                             int64_t n) {
  constexpr int W = 16 / sizeof(T);
  constexpr int U = 4;  // steps per thread, all loads first (streams at ~0.9 of HBM; one step: a third)
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const int64_t nv = n / W, S = gstride();
  for (int64_t i0 = gtid(); i0 < nv; i0 += S * U) {
    V bv[U], dv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * S;
      if (i < nv) {
        bv[u] = reinterpret_cast<const V*>(b)[i];
        dv[u] = reinterpret_cast<const V*>(dinv)[i];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * S;
      if (i >= nv) continue;
      T* bp = reinterpret_cast<T*>(&bv[u]);
      const T* dp = reinterpret_cast<const T*>(&dv[u]);
#pragma unroll
      for (int k = 0; k < W; ++k) bp[k] = omega * dp[k] * bp[k];
      reinterpret_cast<V*>(x)[i] = bv[u];
    }
  }
  if (gtid() == 0)
    for (int64_t i = nv * W; i < n; ++i) x[i] = omega * dinv[i] * b[i];
}
// b = a converted, two values per thread and step (whole allocations)
template <class A, class B>
__global__ void convert(const A* __restrict__ a, B* __restrict__ b, int64_t n) {
  using VA = typename std::conditional<sizeof(A) == 4, float2, double2>::type;
  using VB = typename std::conditional<sizeof(B) == 4, float2, double2>::type;
  const int64_t n2 = n / 2;
  #pragma unroll 2
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    const VA v = reinterpret_cast<const VA*>(a)[i];
    VB o;
    o.x = B(v.x);
    o.y = B(v.y);
    reinterpret_cast<VB*>(b)[i] = o;
  }
  if (gtid() == 0 && (n & 1)) b[n - 1] = B(a[n - 1]);
}
// Coefficients stored in BF16: round the FP32 copy to the nearest BF16 value.
__global__ void to_bf16_values(float* __restrict__ a, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) a[i] = __bfloat162float(__float2bfloat16_rn(a[i]));
}
__global__ void invert(double* __restrict__ d, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) d[i] = 1.0 / d[i];
}

// ------------------------------------------------------------ coarse solve --
// Gauss-Jordan inversion of SPD blocks, all blocks advancing one pivot k per
// launch (blockIdx.y = block; blocks with n <= k skip).
__global__ void gj_col(double* __restrict__ A, const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                       int64_t k, double* __restrict__ colk, const int64_t* __restrict__ boff) {
  const int64_t n = bn[blockIdx.y];
  if (k >= n) return;
  const double* Ab = A + baoff[blockIdx.y];
  double* ck = colk + boff[blockIdx.y];
  for (int64_t i = gtid(); i < n; i += gstride()) ck[i] = Ab[i * n + k];
}
__global__ void gj_row(double* __restrict__ A, const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                       int64_t k, const double* __restrict__ colk, const int64_t* __restrict__ boff) {
  const int64_t n = bn[blockIdx.y];
  if (k >= n) return;
  double* Ab = A + baoff[blockIdx.y];
  const double piv = colk[boff[blockIdx.y] + k];
  for (int64_t j = gtid(); j < n; j += gstride()) Ab[k * n + j] = (j == k ? 1.0 : Ab[k * n + j]) / piv;
}
__global__ void gj_elim(double* __restrict__ A, const int64_t* __restrict__ bn, const int64_t* __restrict__ baoff,
                        int64_t k, const double* __restrict__ colk, const int64_t* __restrict__ boff) {
  const int64_t n = bn[blockIdx.y];
  if (k >= n) return;
  double* Ab = A + baoff[blockIdx.y];
  const double* ck = colk + boff[blockIdx.y];
  for (int64_t t = gtid(); t < n * n; t += gstride()) {
    int64_t i = t / n, j = t - i * n;
    if (i == k) continue;
    Ab[t] = (j == k ? 0.0 : Ab[t]) - ck[i] * Ab[k * n + j];
  }
}
// Blocked Gauss-Jordan inversion of one SPD matrix A (n x n, row-major, in
// place) for coarse levels too large for one pivot per launch: per pivot
// block K of kGjB rows (P = A[K,K], row panel R = A[K,J], column panel
// C = A[I,K], the rest S = A[I,J]) one sweep replaces
//   P <- P^-1,  R <- P^-1 R,  S <- S - C (P^-1 R),  C <- -C P^-1,
// which after every block has been swept leaves A^-1 (the block form of the
// scalar sweep of gj_col / gj_row / gj_elim).  SPD keeps every pivot block
// invertible without pivoting.  The S update is the n^2 kGjB multiply-add
// product that carries the cost: 64 x 64 output tiles, 4 x 4 per thread,
// the panels staged through shared memory.
constexpr int kGjB = 64;

// P^-1 of the pivot block into Pinv (kb x kb, leading dimension kGjB), by the
// unblocked sweep in shared memory (one CTA of 256 threads).
__global__ void __launch_bounds__(256) gjb_pivot(const double* __restrict__ A, int64_t n, int64_t k0, int kb,
                                                 double* __restrict__ Pinv) {
  __shared__ double P[kGjB][kGjB + 1];
  __shared__ double ck[kGjB];
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int i = t / kb, j = t - i * kb;
    P[i][j] = A[(k0 + i) * n + k0 + j];
  }
  __syncthreads();
  for (int k = 0; k < kb; ++k) {
    if (threadIdx.x < kb) ck[threadIdx.x] = P[threadIdx.x][k];
    __syncthreads();
    const double piv = ck[k];
    if (threadIdx.x < kb) P[k][threadIdx.x] = (threadIdx.x == k ? 1.0 : P[k][threadIdx.x]) / piv;
    __syncthreads();
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
      const int i = t / kb, j = t - i * kb;
      if (i != k) P[i][j] = (j == k ? 0.0 : P[i][j]) - ck[i] * P[k][j];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
    const int i = t / kb, j = t - i * kb;
    Pinv[i * kGjB + j] = P[i][j];
  }
}

// R <- P^-1 R: CTA = one strip of 64 columns outside the pivot block.
__global__ void __launch_bounds__(256) gjb_row(double* __restrict__ A, int64_t n, int64_t k0, int kb,
                                               const double* __restrict__ Pinv) {
  extern __shared__ double gj_smem[];  // two kGjB x (kGjB + 1) panels
  double(*Pi)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(gj_smem);
  double(*R)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(gj_smem + kGjB * (kGjB + 1));
  const int64_t j0 = int64_t(blockIdx.x) * kGjB;
  if (j0 == k0) return;  // the pivot block's own columns
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int i = t / kGjB, j = t - i * kGjB;
    Pi[i][j] = (i < kb && j < kb) ? Pinv[i * kGjB + j] : 0.0;
    R[i][j] = (i < kb && j0 + j < n) ? A[(k0 + i) * n + j0 + j] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int i = t / kGjB, j = t - i * kGjB;
    if (i >= kb || j0 + j >= n) continue;
    double acc = 0;
    for (int k = 0; k < kb; ++k) acc += Pi[i][k] * R[k][j];
    A[(k0 + i) * n + j0 + j] = acc;
  }
}

// S <- S - C R for every 64 x 64 tile outside the pivot rows and columns
// (blockIdx.x: column tile, blockIdx.y: row tile).
__global__ void __launch_bounds__(256) gjb_update(double* __restrict__ A, int64_t n, int64_t k0, int kb) {
  extern __shared__ double gj_smem[];
  double(*Cs)[kGjB + 2] = reinterpret_cast<double(*)[kGjB + 2]>(gj_smem);                      // Cs[k][row]
  double(*Rs)[kGjB + 2] = reinterpret_cast<double(*)[kGjB + 2]>(gj_smem + kGjB * (kGjB + 2));  // Rs[k][col]
  const int64_t i0 = int64_t(blockIdx.y) * kGjB, j0 = int64_t(blockIdx.x) * kGjB;
  if (i0 == k0 || j0 == k0) return;
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int r = t / kGjB, k = t - r * kGjB;
    Cs[k][r] = (k < kb && i0 + r < n) ? A[(i0 + r) * n + k0 + k] : 0.0;
    Rs[r][k] = (r < kb && j0 + k < n) ? A[(k0 + r) * n + j0 + k] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0;
  for (int k = 0; k < kb; ++k) {
    double cv[4], rv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) cv[a] = Cs[k][ty + 16 * a];
#pragma unroll
    for (int b = 0; b < 4; ++b) rv[b] = Rs[k][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += cv[a] * rv[b];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int64_t i = i0 + ty + 16 * a;
    if (i >= n) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t j = j0 + tx + 16 * b;
      if (j < n) A[i * n + j] -= acc[a][b];
    }
  }
}

// C <- -C P^-1 for the rows outside the pivot block (one 64-row strip per
// CTA), and the pivot block <- P^-1 (the CTA of the pivot rows).
__global__ void __launch_bounds__(256) gjb_col(double* __restrict__ A, int64_t n, int64_t k0, int kb,
                                               const double* __restrict__ Pinv) {
  extern __shared__ double gj_smem[];
  double(*Pi)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(gj_smem);
  double(*Cb)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(gj_smem + kGjB * (kGjB + 1));
  const int64_t i0 = int64_t(blockIdx.x) * kGjB;
  if (i0 == k0) {
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
      const int i = t / kb, j = t - i * kb;
      A[(k0 + i) * n + k0 + j] = Pinv[i * kGjB + j];
    }
    return;
  }
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int i = t / kGjB, j = t - i * kGjB;
    Pi[i][j] = (i < kb && j < kb) ? Pinv[i * kGjB + j] : 0.0;
    Cb[i][j] = (i0 + i < n && j < kb) ? A[(i0 + i) * n + k0 + j] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int i = t / kGjB, j = t - i * kGjB;
    if (i0 + i >= n || j >= kb) continue;
    double acc = 0;
    for (int k = 0; k < kb; ++k) acc += Cb[i][k] * Pi[k][j];
    A[(i0 + i) * n + k0 + j] = -acc;
  }
}

dg_status gj_invert_blocked(double* A, int64_t n, cudaStream_t s) {
  DBuf<double> pinv;
  DG_TRY(pinv.alloc(kGjB * kGjB));
  const unsigned nt = unsigned((n + kGjB - 1) / kGjB);
  const int sm1 = int(sizeof(double)) * 2 * kGjB * (kGjB + 1), sm2 = int(sizeof(double)) * 2 * kGjB * (kGjB + 2);
  DG_CUDA(cudaFuncSetAttribute(gjb_row, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1));
  DG_CUDA(cudaFuncSetAttribute(gjb_col, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1));
  DG_CUDA(cudaFuncSetAttribute(gjb_update, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2));
  for (int64_t k0 = 0; k0 < n; k0 += kGjB) {
    const int kb = int(std::min<int64_t>(kGjB, n - k0));
    gjb_pivot<<<1, 256, 0, s>>>(A, n, k0, kb, pinv.p);
    gjb_row<<<nt, 256, sm1, s>>>(A, n, k0, kb, pinv.p);
    gjb_update<<<dim3(nt, nt), 256, sm2, s>>>(A, n, k0, kb);
    gjb_col<<<nt, 256, sm1, s>>>(A, n, k0, kb, pinv.p);
  }
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));  // pinv is freed on return
  return DG_OK;
}

// x = Ainv b with block-diagonal Ainv, one warp per row
__global__ void dense_gemv(const double* __restrict__ A, int64_t N, const uint32_t* __restrict__ row_blk,
                           const int64_t* __restrict__ boff, const int64_t* __restrict__ bn,
                           const int64_t* __restrict__ baoff, const double* __restrict__ b, double* __restrict__ x) {
  const int lane = threadIdx.x & 31;
  for (int64_t row = gtid() >> 5; row < N; row += gstride() >> 5) {
    const uint32_t blk = row_blk[row];
    const int64_t o = boff[blk], n = bn[blk];
    const double* Ar = A + baoff[blk] + (row - o) * n;
    double s = 0;
    for (int64_t j = lane; j < n; j += 32) s += Ar[j] * b[o + j];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (!lane) x[row] = s;
  }
}

// -------------------------------------------------------------- reductions --
constexpr int kRedBlocks = 1184;  // 8 x 148 SMs: enough loads in flight for HBM

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) ws[w] = v;
  __syncthreads();
  v = 0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}
// deterministic second stage: one block sums the partials in a fixed order
__global__ void finish_sum(const double* __restrict__ part, int np, double* __restrict__ out) {
  double v = 0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
  v = block_sum(v);
  if (threadIdx.x == 0) *out = v;
}
// The FP64 vector kernels of the outer CG read 16-byte pairs (the solver's
// vectors are whole allocations, so 16-byte aligned); an odd last element is
// handled by thread 0.
__global__ void dot_partial(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                            double* __restrict__ part) {
  const double2* a2 = reinterpret_cast<const double2*>(a);
  const double2* b2 = reinterpret_cast<const double2*>(b);
  const int64_t n2 = n / 2;
  double v0 = 0, v1 = 0;
  #pragma unroll 2
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    const double2 x = a2[i], y = b2[i];
    v0 = fma(x.x, y.x, v0);
    v1 = fma(x.y, y.y, v1);
  }
  if (gtid() == 0 && (n & 1)) v0 = fma(a[n - 1], b[n - 1], v0);
  const double v = block_sum(v0 + v1);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
// the same for arrays of any alignment (caller-provided vectors)
__global__ void dot_partial_any(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                                double* __restrict__ part) {
  double v0 = 0;
  #pragma unroll 4
  for (int64_t i = gtid(); i < n; i += gstride()) v0 = fma(a[i], b[i], v0);
  const double v = block_sum(v0);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
// x += alpha p; r -= alpha q; partial (r, r); alpha = num / den read on device
__global__ void cg_update(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                          const double* __restrict__ q, int64_t n, const double* __restrict__ num,
                          const double* __restrict__ den, double* __restrict__ part) {
  const double alpha = *num / *den;
  double2* x2 = reinterpret_cast<double2*>(x);
  double2* r2 = reinterpret_cast<double2*>(r);
  const double2* p2 = reinterpret_cast<const double2*>(p);
  const double2* q2 = reinterpret_cast<const double2*>(q);
  const int64_t n2 = n / 2, S = gstride();
  double v0 = 0, v1 = 0;
  constexpr int U = 4;  // steps per thread, all loads first
  for (int64_t i0 = gtid(); i0 < n2; i0 += S * U) {
    double2 xi[U], ri[U], pi[U], qi[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * S;
      if (i < n2) {
        xi[u] = x2[i];
        ri[u] = r2[i];
        pi[u] = p2[i];
        qi[u] = q2[i];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * S;
      if (i >= n2) continue;
      xi[u].x += alpha * pi[u].x;
      xi[u].y += alpha * pi[u].y;
      ri[u].x -= alpha * qi[u].x;
      ri[u].y -= alpha * qi[u].y;
      x2[i] = xi[u];
      r2[i] = ri[u];
      v0 = fma(ri[u].x, ri[u].x, v0);
      v1 = fma(ri[u].y, ri[u].y, v1);
    }
  }
  if (gtid() == 0 && (n & 1)) {
    x[n - 1] += alpha * p[n - 1];
    const double rl = r[n - 1] - alpha * q[n - 1];
    r[n - 1] = rl;
    v0 = fma(rl, rl, v0);
  }
  const double v = block_sum(v0 + v1);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
// p = z + beta p on 16-byte pairs
__device__ __forceinline__ void axpby_pairs(double* __restrict__ p, const double* __restrict__ z, int64_t n,
                                            double beta) {
  double2* p2 = reinterpret_cast<double2*>(p);
  const double2* z2 = reinterpret_cast<const double2*>(z);
  const int64_t n2 = n / 2;
  #pragma unroll 2
  for (int64_t i = gtid(); i < n2; i += gstride()) {
    double2 pi = p2[i];
    const double2 zi = z2[i];
    pi.x = zi.x + beta * pi.x;
    pi.y = zi.y + beta * pi.y;
    p2[i] = pi;
  }
  if (gtid() == 0 && (n & 1)) p[n - 1] = z[n - 1] + beta * p[n - 1];
}
// flexible (Polak-Ribiere) direction: p = z + beta p,
// beta = ((r, z) - (r, z_old)) / (r_old, z_old)
__global__ void cg_direction_flex(double* __restrict__ p, const double* __restrict__ z, int64_t n,
                                  const double* __restrict__ rz, const double* __restrict__ rzo,
                                  const double* __restrict__ den) {
  axpby_pairs(p, z, n, (*rz - *rzo) / *den);
}
// p = z + beta p with beta = num / den
__global__ void cg_direction(double* __restrict__ p, const double* __restrict__ z, int64_t n,
                             const double* __restrict__ num, const double* __restrict__ den) {
  axpby_pairs(p, z, n, *num / *den);
}

}  // namespace

// --------------------------------------------------------------- hierarchy --
struct Level {
  std::unique_ptr<dg_octree> tree;
  std::unique_ptr<dg_da> da;
  std::unique_ptr<dg_mat> A;
  DBuf<double> dinv, x, b, t;
  DBuf<double> acc;   // shared-node sums of the fused sweeps (kept zero between uses)
  // P to this level from level + 1 (CSR over this level's nodes) and R = P^T
  // (CSR over the coarse nodes, entries in fine-node order)
  DBuf<uint32_t> pptr, pcol, rptr, rcol;
  DBuf<double> pval, rval;
  // the weights of P and R as exact 8-bit codes (empty when a weight has
  // none; the transfers then read pval / rval)
  DBuf<uint8_t> pcode, rcode;
  // FP32 inner V-cycle
  DBuf<float> dinv32, x32, b32, t32, pval32, rval32, acc32;
  // learned smoother data (finest level): residual, neighbour stats,
  // 1 / element references, hanging share, mean log2 diagonal
  DBuf<float> sm_r, sm_nsum, sm_nmax, sm_refs, sm_hang;
  float sm_dlogbar = 0.f;
  // coarse_op 1 (levels below the finest): the operator J from the finer
  // level's coefficients = the averaged coefficients with the type-1 elements
  // zeroed (coefJ) plus their children sums (t1); the Jacobi diagonal stays
  // that of the averaged coefficients (the reference's B matrix)
  Type1Set t1;
  DBuf<double> coefJ;
  DBuf<float> coefJ32;
  const double* jcoef() const { return t1.n ? coefJ.p : nullptr; }
  const float* jcoef32() const { return t1.n ? coefJ32.p : nullptr; }
  const Type1Set* jset() const { return t1.n ? &t1 : nullptr; }
};

struct dg_damg {
  dg_damg_config cfg;
  std::vector<Level> lv;
  DBuf<double> Ainv;  // dense inverses of the coarsest operator, one block per mesh
  int64_t nc = 0;
  // block structure of the coarsest level (one block per independent mesh)
  std::vector<int64_t> cb_off, cb_n, cb_aoff;
  DBuf<int64_t> d_cb_off, d_cb_n, d_cb_aoff;
  DBuf<uint32_t> d_crow_blk;
  // batches: mesh offsets of elements / nodes on every level
  int nmesh = 1;
  std::vector<std::vector<int64_t>> mesh_elem_off, mesh_node_off;  // [level][mesh + 1]
  DBuf<uint16_t> d_node_mesh;   // finest-level node -> mesh
  DBuf<double> mesh_part;       // per-mesh squared norms
  // learned post-smoother on the finest level (FP32 inner V-cycle only)
  dg_mlp* mlp = nullptr;
  int mlp_sweeps = 2;
  double mlp_fallback = 0.7;
  bool mlp_active = false;
  DBuf<float> sm_s2;
  // PCG work vectors on the finest level and device scalars
  DBuf<double> r, z, zold, p, q, part, scal;
  DBuf<float> r32, z32;
  cudaStream_t s = nullptr;
  // captured preconditioner, one per post-smoother (0 Jacobi, 1 learned), so
  // that a fallback inside a solve switches graphs instead of capturing again
  cudaGraphExec_t precond_graph[2] = {nullptr, nullptr};
  void drop_graphs() {
    for (cudaGraphExec_t& g : precond_graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  ~dg_damg() {
    drop_graphs();
    if (s) cudaStreamDestroy(s);
  }
};

namespace {

dg_status build_prolongation(Level& F, Level& C, cudaStream_t s) {
  const dg_da* fd = F.da.get();
  const dg_da* cd = C.da.get();
  DG_CHECK(fd->D == cd->D, DG_EINVAL, "levels with different depths");
  const uint32_t top = 1u << (fd->D - 1);
  DBuf<uint32_t> err;
  DG_TRY(err.alloc(1));
  DG_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
  DG_TRY(F.pptr.alloc(fd->N + 1));
  prolong_count<<<grid_for(fd->N, 256), 256, 0, s>>>(fd->nkey.p, fd->N, cd->ekey.p, cd->E, cd->meta.p, top, fd->D,
                                                      F.pptr.p, err.p);
  DG_CUDA(cudaMemsetAsync(F.pptr.p + fd->N, 0, 4, s));
  uint32_t nnz = 0;
  DG_TRY(scan_u32(F.pptr.p, F.pptr.p, fd->N + 1, &nnz, s));
  uint32_t herr = 0;
  DG_CUDA(cudaMemcpyAsync(&herr, err.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  DG_CHECK(!herr, DG_EUNBALANCED, "fine node outside every coarse element");
  DG_TRY(F.pcol.alloc(nnz));
  DG_TRY(F.pval.alloc(nnz));
  prolong_fill<<<grid_for(fd->N, 256), 256, 0, s>>>(fd->nkey.p, fd->N, cd->ekey.p, cd->E, cd->meta.p, cd->nl.p, top,
                                                     fd->D, F.pptr.p, F.pcol.p, F.pval.p);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// R = P^T by coarse rows, entries in fine-node order (a stable sort of the
// entries by their coarse column).
dg_status build_restriction(Level& F, int64_t Nc, cudaStream_t s) {
  const int64_t Nf = F.da->N, nnz = F.pcol.n;
  DBuf<uint64_t> keys, tmp;
  DBuf<uint32_t> frow;
  DG_TRY(keys.alloc(nnz));
  DG_TRY(tmp.alloc(nnz));
  DG_TRY(frow.alloc(nnz));
  DG_TRY(F.rptr.alloc(Nc + 1));
  DG_CUDA(cudaMemsetAsync(F.rptr.p, 0, 4 * (Nc + 1), s));
  ptrans_keys<<<grid_for(Nf, 256), 256, 0, s>>>(F.pptr.p, F.pcol.p, Nf, keys.p, frow.p, F.rptr.p);
  DG_CUDA(cudaGetLastError());
  int bits = 1;
  while ((int64_t(1) << bits) < Nc) ++bits;
  DG_TRY(radix_sort_u64(keys.p, tmp.p, nnz, bits, s, 32));
  uint32_t total = 0;
  DG_TRY(scan_u32(F.rptr.p, F.rptr.p, Nc + 1, &total, s));
  DG_CHECK(int64_t(total) == nnz, DG_EINVAL, "restriction: entry count mismatch");
  DG_TRY(F.rcol.alloc(nnz));
  DG_TRY(F.rval.alloc(nnz));
  ptrans_fill<<<grid_for(nnz, 256), 256, 0, s>>>(keys.p, nnz, frow.p, F.pval.p, F.rcol.p, F.rval.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(s));
  return DG_OK;
}

// The 8-bit weight codes of P and R (kept only when every weight has one).
dg_status build_weight_codes(Level& F, cudaStream_t s) {
  const int64_t nnz = F.pval.n;
  if (!nnz || F.rval.n != nnz) return DG_OK;
  // DG_TRANSFER_CODES=0 keeps the FP64 / FP32 weights (to compare the two forms)
  if (const char* e = getenv("DG_TRANSFER_CODES"))
    if (!strcmp(e, "0")) return DG_OK;
  DBuf<uint32_t> bad;
  DG_TRY(bad.alloc(1));
  DG_CUDA(cudaMemsetAsync(bad.p, 0, 4, s));
  DG_TRY(F.pcode.alloc(nnz));
  DG_TRY(F.rcode.alloc(nnz));
  weight_codes<<<grid_for(nnz, 256), 256, 0, s>>>(F.pval.p, nnz, F.pcode.p, bad.p);
  weight_codes<<<grid_for(nnz, 256), 256, 0, s>>>(F.rval.p, nnz, F.rcode.p, bad.p);
  DG_CUDA(cudaGetLastError());
  uint32_t hbad = 0;
  DG_CUDA(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  if (hbad) {
    F.pcode.reset();
    F.rcode.reset();
  }
  return DG_OK;
}

// rc = R rf and xf += P xc for the scalar hierarchy in FP64 or FP32, by the
// weight codes where the level has them.
template <class T>
void restrict_level(const Level& F, int64_t Nc, const T* rf, T* rc, cudaStream_t s) {
  const unsigned g = grid_for(Nc, 256, 16);
  if (F.rcode.n) {
    restrict_gather_coded<T><<<g, 256, 0, s>>>(F.rptr.p, F.rcol.p, F.rcode.p, Nc, rf, rc);
  } else if constexpr (sizeof(T) == 8) {
    restrict_gather<T><<<g, 256, 0, s>>>(F.rptr.p, F.rcol.p, F.rval.p, Nc, rf, rc);
  } else {
    restrict_gather<T><<<g, 256, 0, s>>>(F.rptr.p, F.rcol.p, F.rval32.p, Nc, rf, rc);
  }
}
template <class T>
void prolong_level(const Level& F, int64_t Nf, const T* xc, T* xf, cudaStream_t s, unsigned g) {
  if (F.pcode.n) {
    prolong_add_coded<T><<<g, 256, 0, s>>>(F.pptr.p, F.pcol.p, F.pcode.p, Nf, xc, xf);
  } else if constexpr (sizeof(T) == 8) {
    prolong_add<T><<<g, 256, 0, s>>>(F.pptr.p, F.pcol.p, F.pval.p, Nf, xc, xf);
  } else {
    prolong_add<T><<<g, 256, 0, s>>>(F.pptr.p, F.pcol.p, F.pval32.p, Nf, xc, xf);
  }
}

dg_status setup_level_vectors(Level& L, cudaStream_t s) {
  const int64_t N = int64_t(L.A->dof) * L.da->N;
  DG_TRY(L.dinv.alloc(N));
  DG_TRY(L.x.alloc(N));
  DG_TRY(L.b.alloc(N));
  DG_TRY(L.t.alloc(N));
  DG_TRY(L.acc.alloc(N));
  DG_CUDA(cudaMemsetAsync(L.acc.p, 0, 8 * N, s));
  if (L.A->kind == 1) DG_TRY(elasticity_diag(L.A.get(), L.dinv.p, s));
  else DG_TRY(lapmass_diag(L.A.get(), L.dinv.p, s));
  invert<<<grid_for(N, 256), 256, 0, s>>>(L.dinv.p, N);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status round_coef_bf16(float* c, int64_t n, cudaStream_t s) {
  to_bf16_values<<<grid_for(n, 256), 256, 0, s>>>(c, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// FP32 copies for the inner V-cycle: smoother diagonal, prolongation weights
// and (optionally BF16-rounded) coefficients.
dg_status setup_level_f32(dg_damg* m, Level& L, cudaStream_t s) {
  const int64_t N = L.da->N;
  DG_TRY(L.dinv32.alloc(N));
  DG_TRY(L.x32.alloc(N));
  DG_TRY(L.b32.alloc(N));
  DG_TRY(L.t32.alloc(N));
  DG_TRY(L.acc32.alloc(N));
  DG_CUDA(cudaMemsetAsync(L.acc32.p, 0, 4 * N, s));
  convert<double, float><<<grid_for(N, 256), 256, 0, s>>>(L.dinv.p, L.dinv32.p, N);
  if (L.pval.n) {
    DG_TRY(L.pval32.alloc(L.pval.n));
    convert<double, float><<<grid_for(L.pval.n, 256), 256, 0, s>>>(L.pval.p, L.pval32.p, L.pval.n);
    DG_TRY(L.rval32.alloc(L.rval.n));
    convert<double, float><<<grid_for(L.rval.n, 256), 256, 0, s>>>(L.rval.p, L.rval32.p, L.rval.n);
  }
  if (L.A->has_coef && m->cfg.inner_prec == DG_PREC_F32_BF16COEF)
    DG_TRY(round_coef_bf16(L.A->coef32.p, 2 * L.da->E, s));
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

__global__ void fill_row_blk(uint32_t* __restrict__ rb, int64_t n0, int64_t n1, uint32_t b) {
  for (int64_t i = n0 + gtid(); i < n1; i += gstride()) rb[i] = b;
}

// The dense inverse of the coarsest operator: up to kMaxCoarseNodes nodes per
// mesh (8.6 GB of FP64 at the limit); one mesh above kGjBlockedFrom nodes is
// inverted by the blocked sweep, smaller or batched meshes one pivot per launch.
constexpr int64_t kMaxCoarseNodes = 32768;
constexpr int64_t kGjBlockedFrom = 1024;
dg_status gj_invert(dg_damg* m, int64_t maxn, int nb);

dg_status setup_coarse(dg_damg* m) {
  Level& L = m->lv.back();
  if (L.A->kind == 1) {
    // dof 3: one mesh, one dense block over its 3 N unknowns
    const int64_t n3 = 3 * L.da->N;
    DG_CHECK(n3 <= kMaxCoarseNodes, DG_EINVAL,
             "coarsest level too large for the dense direct solve (> 32768 unknowns of one mesh)");
    m->cb_off.assign(1, 0);
    m->cb_n.assign(1, n3);
    m->cb_aoff.assign(1, 0);
    m->nc = n3;
    DG_TRY(m->Ainv.alloc(n3 * n3));
    DG_TRY(m->d_cb_off.alloc(1));
    DG_TRY(m->d_cb_n.alloc(1));
    DG_TRY(m->d_cb_aoff.alloc(1));
    DG_TRY(m->d_crow_blk.alloc(n3));
    DG_CUDA(cudaMemcpyAsync(m->d_cb_off.p, m->cb_off.data(), 8, cudaMemcpyHostToDevice, m->s));
    DG_CUDA(cudaMemcpyAsync(m->d_cb_n.p, m->cb_n.data(), 8, cudaMemcpyHostToDevice, m->s));
    DG_CUDA(cudaMemcpyAsync(m->d_cb_aoff.p, m->cb_aoff.data(), 8, cudaMemcpyHostToDevice, m->s));
    DG_CUDA(cudaMemsetAsync(m->d_crow_blk.p, 0, 4 * n3, m->s));
    DG_TRY(elasticity_assemble_dense(L.A.get(), m->Ainv.p, m->s));
    return gj_invert(m, n3, 1);
  }
  const int64_t N = L.da->N;
  const std::vector<int64_t>& noff = m->mesh_node_off.back();
  const int nb = int(noff.size()) - 1;
  m->cb_off.assign(noff.begin(), noff.end() - 1);
  m->cb_n.resize(nb);
  m->cb_aoff.resize(nb);
  int64_t total = 0, maxn = 0;
  for (int b = 0; b < nb; ++b) {
    m->cb_n[b] = noff[b + 1] - noff[b];
    DG_CHECK(m->cb_n[b] <= kMaxCoarseNodes, DG_EINVAL,
             "coarsest level too large for the dense direct solve (> 32768 nodes of one mesh)");
    m->cb_aoff[b] = total;
    total += m->cb_n[b] * m->cb_n[b];
    maxn = m->cb_n[b] > maxn ? m->cb_n[b] : maxn;
  }
  m->nc = N;
  DG_TRY(m->Ainv.alloc(total));
  DG_TRY(m->d_cb_off.alloc(nb));
  DG_TRY(m->d_cb_n.alloc(nb));
  DG_TRY(m->d_cb_aoff.alloc(nb));
  DG_TRY(m->d_crow_blk.alloc(N));
  DG_CUDA(cudaMemcpyAsync(m->d_cb_off.p, m->cb_off.data(), 8 * nb, cudaMemcpyHostToDevice, m->s));
  DG_CUDA(cudaMemcpyAsync(m->d_cb_n.p, m->cb_n.data(), 8 * nb, cudaMemcpyHostToDevice, m->s));
  DG_CUDA(cudaMemcpyAsync(m->d_cb_aoff.p, m->cb_aoff.data(), 8 * nb, cudaMemcpyHostToDevice, m->s));
  for (int b = 0; b < nb; ++b)
    fill_row_blk<<<grid_for(m->cb_n[b], 256), 256, 0, m->s>>>(m->d_crow_blk.p, noff[b], noff[b + 1], uint32_t(b));
  DG_TRY(lapmass_assemble_dense(L.A.get(), m->Ainv.p, total, m->d_crow_blk.p, m->d_cb_off.p, m->d_cb_n.p,
                                m->d_cb_aoff.p, m->s, L.jcoef(), L.jset()));
  return gj_invert(m, maxn, nb);
}

// The dense inverse of the coarsest operator in m->Ainv: the blocked sweep
// for one large block, else one pivot per launch over all blocks.
dg_status gj_invert(dg_damg* m, int64_t maxn, int nb) {
  if (nb == 1 && maxn > kGjBlockedFrom) return gj_invert_blocked(m->Ainv.p, maxn, m->s);
  const int64_t N = m->nc;
  DBuf<double> colk;
  DG_TRY(colk.alloc(N));
  const dim3 g1(grid_for(maxn, 256), unsigned(nb)), g2(grid_for(maxn * maxn, 256), unsigned(nb));
  for (int64_t k = 0; k < maxn; ++k) {
    gj_col<<<g1, 256, 0, m->s>>>(m->Ainv.p, m->d_cb_n.p, m->d_cb_aoff.p, k, colk.p, m->d_cb_off.p);
    gj_row<<<g1, 256, 0, m->s>>>(m->Ainv.p, m->d_cb_n.p, m->d_cb_aoff.p, k, colk.p, m->d_cb_off.p);
    gj_elim<<<g2, 256, 0, m->s>>>(m->Ainv.p, m->d_cb_n.p, m->d_cb_aoff.p, k, colk.p, m->d_cb_off.p);
  }
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(m->s));
  return DG_OK;
}

// Type-1 set and J coefficients of level l (>= 1) from level l - 1.
dg_status setup_type1(dg_damg* m, size_t l) {
  cudaStream_t s = m->s;
  Level& L = m->lv[l];
  Level& F = m->lv[l - 1];
  const int64_t Ec = L.da->E;
  DBuf<uint8_t> flag;
  DBuf<double> child;
  DG_TRY(flag.alloc(Ec));
  DG_TRY(child.alloc(16 * Ec));
  const std::vector<int64_t>& fo = m->mesh_elem_off[l - 1];
  const std::vector<int64_t>& co = m->mesh_elem_off[l];
  for (int i = 0; i < m->nmesh; ++i) {
    const int64_t ef = fo[i + 1] - fo[i], ec = co[i + 1] - co[i];
    type1_detect_kernel<<<grid_for(ec, 256), 256, 0, s>>>(
        F.da->ekey.p + fo[i], ef, F.A->coef.p + fo[i], F.A->coef.p + F.da->E + fo[i], L.da->ekey.p + co[i], ec,
        1e-12, flag.p + co[i], child.p + 16 * co[i]);
  }
  DG_CUDA(cudaGetLastError());
  std::vector<uint8_t> hf(static_cast<size_t>(Ec));
  DG_CUDA(cudaMemcpyAsync(hf.data(), flag.p, Ec, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> ids;
  for (int64_t e = 0; e < Ec; ++e)
    if (hf[size_t(e)]) ids.push_back(uint32_t(e));
  L.t1.n = int64_t(ids.size());
  if (!L.t1.n) return DG_OK;
  const int64_t n = L.t1.n;
  DG_TRY(L.t1.elem.alloc(n));
  DG_CUDA(cudaMemcpyAsync(L.t1.elem.p, ids.data(), 4 * n, cudaMemcpyHostToDevice, s));
  DG_TRY(L.t1.coef.alloc(16 * n));
  gather16<<<grid_for(16 * n, 256), 256, 0, s>>>(child.p, L.t1.elem.p, n, L.t1.coef.p);
  DG_TRY(L.coefJ.alloc(2 * Ec + kCoefPad));
  DG_CUDA(cudaMemcpyAsync(L.coefJ.p, L.A->coef.p, 16 * Ec, cudaMemcpyDeviceToDevice, s));
  zero_elems<<<grid_for(n, 256), 256, 0, s>>>(L.coefJ.p, Ec, L.t1.elem.p, n);
  DG_CUDA(cudaGetLastError());
  if (m->cfg.inner_prec != DG_PREC_F64) {
    DG_TRY(L.coefJ32.alloc(2 * Ec + kCoefPad));
    DG_TRY(convert_f64_to_f32(L.coefJ.p, L.coefJ32.p, 2 * Ec, s));
    DG_TRY(L.t1.coef32.alloc(16 * n));
    DG_TRY(convert_f64_to_f32(L.t1.coef.p, L.t1.coef32.p, 16 * n, s));
    if (m->cfg.inner_prec == DG_PREC_F32_BF16COEF) {
      DG_TRY(round_coef_bf16(L.coefJ32.p, 2 * Ec, s));
      DG_TRY(round_coef_bf16(L.t1.coef32.p, 16 * n, s));
    }
  }
  DG_CUDA(cudaStreamSynchronize(s));  // child is freed on return
  return DG_OK;
}

// dof 3: ElasticityMatMult on every level with that level's boundary nodes
// (assignBoundaryFlags) as its Dirichlet nodes (SetElasticityContexts,
// examples/src/backend/elasticityJac.C:396-480).
dg_status set_elasticity_operators(dg_damg* m) {
  cudaStream_t s = m->s;
  for (size_t l = 0; l < m->lv.size(); ++l) {
    Level& L = m->lv[l];
    auto A = std::make_unique<dg_mat>();
    A->da = L.da.get();
    A->kind = 1;
    A->dof = 3;
    A->mu = m->cfg.mu;
    A->lam = m->cfg.lambda;
    DG_TRY(A->dirichlet.alloc(L.da->N));
    DG_TRY(node_boundary_flags(L.da.get(), A->dirichlet.p, s));
    L.A = std::move(A);
    DG_TRY(setup_level_vectors(L, s));
    L.t1.n = 0;
  }
  m->drop_graphs();
  return setup_coarse(m);
}

dg_status set_operators(dg_damg* m, const double* coef) {
  if (m->cfg.dof == 3) {
    DG_CHECK(!coef, DG_EINVAL, "damg: dof 3 (elasticity) takes no Laplacian-mass coefficients");
    return set_elasticity_operators(m);
  }
  cudaStream_t s = m->s;
  for (size_t l = 0; l < m->lv.size(); ++l) {
    Level& L = m->lv[l];
    auto A = std::make_unique<dg_mat>();
    A->da = L.da.get();
    A->kind = 0;
    A->dof = 1;
    if (coef) {
      A->has_coef = true;
      DG_TRY(A->coef.alloc(2 * L.da->E + kCoefPad));
      if (l == 0) {
        std::vector<double> soa(2 * L.da->E);
        for (int64_t e = 0; e < L.da->E; ++e) {
          soa[e] = coef[2 * e];
          soa[L.da->E + e] = coef[2 * e + 1];
        }
        DG_CUDA(cudaMemcpyAsync(A->coef.p, soa.data(), 16 * L.da->E, cudaMemcpyHostToDevice, s));
        DG_CUDA(cudaStreamSynchronize(s));
      } else {
        Level& F = m->lv[l - 1];
        DBuf<uint32_t> err;
        DG_TRY(err.alloc(1));
        DG_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
        // per mesh: element keys are sorted within each mesh's segment
        const std::vector<int64_t>& fo = m->mesh_elem_off[l - 1];
        const std::vector<int64_t>& co = m->mesh_elem_off[l];
        for (int i = 0; i < m->nmesh; ++i) {
          const int64_t ef = fo[i + 1] - fo[i], ec = co[i + 1] - co[i];
          coarse_coef_kernel<<<grid_for(ec, 256), 256, 0, s>>>(
              F.da->ekey.p + fo[i], ef, F.A->coef.p + fo[i], F.A->coef.p + F.da->E + fo[i], L.da->ekey.p + co[i],
              ec, A->coef.p + co[i], A->coef.p + L.da->E + co[i], err.p);
        }
        uint32_t herr = 0;
        DG_CUDA(cudaMemcpyAsync(&herr, err.p, 4, cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        DG_CHECK(!herr, DG_EINVAL, "coarse element without fine elements");
      }
      DG_TRY(A->coef32.alloc(2 * L.da->E + kCoefPad));
      DG_TRY(convert_f64_to_f32(A->coef.p, A->coef32.p, 2 * L.da->E, s));
    }
    L.A = std::move(A);
    DG_TRY(setup_level_vectors(L, s));
    if (m->cfg.inner_prec != DG_PREC_F64) DG_TRY(setup_level_f32(m, L, s));
    L.t1.n = 0;
    if (coef && l > 0 && m->cfg.coarse_op == 1) DG_TRY(setup_type1(m, l));
  }
  m->drop_graphs();  // operators changed: capture again on the next solve
  return setup_coarse(m);
}

// The level operator y = A x (FP64): Laplacian + mass, or elasticity.
dg_status level_op(const Level& L, const double* x, double* y, cudaStream_t s) {
  if (L.A->kind == 1) return elasticity_apply_f64(L.A.get(), x, y, s);
  return lapmass_apply_f64(L.A.get(), x, y, s);
}

// The dof-3 V(nu_pre, nu_post) cycle: the same Richardson-Jacobi steps as the
// scalar one (zero initial guess, first sweep x = omega D^-1 b), with the
// elasticity operator and the transfers applied per component.
dg_status vcycle3(dg_damg* m, size_t l, const double* b, double* x) {
  cudaStream_t s = m->s;
  Level& L = m->lv[l];
  const int64_t nn = L.da->N, n = 3 * nn;
  const unsigned g = grid_for(n, 256, 16);
  if (l + 1 == m->lv.size()) {
    dense_gemv<<<grid_for(n * 32, 256), 256, 0, s>>>(m->Ainv.p, n, m->d_crow_blk.p, m->d_cb_off.p, m->d_cb_n.p,
                                                     m->d_cb_aoff.p, b, x);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  const double w = m->cfg.omega;
  if (m->cfg.nu_pre > 0) {
    jacobi_first<<<g, 256, 0, s>>>(x, b, L.dinv.p, w, n);
    for (int k = 1; k < m->cfg.nu_pre; ++k) {
      DG_TRY(elasticity_apply_f64(L.A.get(), x, L.t.p, s));
      jacobi_update<<<g, 256, 0, s>>>(x, b, L.dinv.p, L.t.p, w, n);
    }
    DG_TRY(elasticity_apply_f64(L.A.get(), x, L.acc.p, s));
    residual_update<<<g, 256, 0, s>>>(b, L.acc.p, L.t.p, n);
  } else {
    DG_CUDA(cudaMemsetAsync(x, 0, 8 * n, s));
  }
  Level& C = m->lv[l + 1];
  restrict_gather3<<<grid_for(C.da->N, 256, 16), 256, 0, s>>>(L.rptr.p, L.rcol.p, L.rval.p, C.da->N,
                                                             m->cfg.nu_pre > 0 ? (const double*)L.t.p : b, C.b.p);
  DG_TRY(vcycle3(m, l + 1, C.b.p, C.x.p));
  prolong_add3<<<grid_for(nn, 256, 16), 256, 0, s>>>(L.pptr.p, L.pcol.p, L.pval.p, nn, C.x.p, x);
  for (int k = 0; k < m->cfg.nu_post; ++k) {
    DG_TRY(elasticity_apply_f64(L.A.get(), x, L.t.p, s));
    jacobi_update<<<g, 256, 0, s>>>(x, b, L.dinv.p, L.t.p, w, n);
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// z = V(b) on level l (x of level l holds the result)
dg_status vcycle(dg_damg* m, size_t l, const double* b, double* x) {
  if (m->cfg.dof == 3) return vcycle3(m, l, b, x);
  cudaStream_t s = m->s;
  Level& L = m->lv[l];
  const int64_t n = L.da->N;
  const unsigned g = grid_for(n, 256, 16);
  if (l + 1 == m->lv.size()) {
    dense_gemv<<<grid_for(n * 32, 256), 256, 0, s>>>(m->Ainv.p, n, m->d_crow_blk.p, m->d_cb_off.p, m->d_cb_n.p,
                                                     m->d_cb_aoff.p, b, x);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  const double w = m->cfg.omega;
  // pre-smoothing from a zero initial guess; the sweeps after the first and
  // the residual are fused warp-tile operator applications
  if (m->cfg.nu_pre > 0) {
    jacobi_first<<<g, 256, 0, s>>>(x, b, L.dinv.p, w, n);
    for (int k = 1; k < m->cfg.nu_pre; ++k)
      DG_TRY(lapmass_smooth_f64(L.A.get(), x, b, L.dinv.p, w, L.acc.p, s, L.jcoef(), L.jset()));
    DG_TRY(lapmass_residual_f64(L.A.get(), x, b, L.t.p, L.acc.p, s, L.jcoef(), L.jset()));
  } else {
    DG_CUDA(cudaMemsetAsync(x, 0, 8 * n, s));
  }
  Level& C = m->lv[l + 1];
  restrict_level<double>(L, C.da->N, m->cfg.nu_pre > 0 ? (const double*)L.t.p : b, C.b.p, s);
  DG_TRY(vcycle(m, l + 1, C.b.p, C.x.p));
  prolong_level<double>(L, n, C.x.p, x, s, g);
  for (int k = 0; k < m->cfg.nu_post; ++k)
    DG_TRY(lapmass_smooth_f64(L.A.get(), x, b, L.dinv.p, w, L.acc.p, s, L.jcoef(), L.jset()));
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// FP32 V-cycle; the coarsest solve stays FP64 (the dense inverse).
dg_status vcycle32(dg_damg* m, size_t l, const float* b, float* x) {
  cudaStream_t s = m->s;
  Level& L = m->lv[l];
  const int64_t n = L.da->N;
  const unsigned g = grid_for(n, 256, 16);
  if (l + 1 == m->lv.size()) {
    convert<float, double><<<g, 256, 0, s>>>(b, L.b.p, n);
    dense_gemv<<<grid_for(n * 32, 256), 256, 0, s>>>(m->Ainv.p, n, m->d_crow_blk.p, m->d_cb_off.p, m->d_cb_n.p,
                                                     m->d_cb_aoff.p, L.b.p, L.x.p);
    convert<double, float><<<g, 256, 0, s>>>(L.x.p, x, n);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  const float w = float(m->cfg.omega);
  if (m->cfg.nu_pre > 0) {
    jacobi_first<<<g, 256, 0, s>>>(x, b, L.dinv32.p, w, n);
    for (int k = 1; k < m->cfg.nu_pre; ++k)
      DG_TRY(lapmass_smooth_f32(L.A.get(), x, b, L.dinv32.p, w, L.acc32.p, s, L.jcoef32(), L.jset()));
    DG_TRY(lapmass_residual_f32(L.A.get(), x, b, L.t32.p, L.acc32.p, s, L.jcoef32(), L.jset()));
  } else {
    DG_CUDA(cudaMemsetAsync(x, 0, 4 * n, s));
  }
  Level& C = m->lv[l + 1];
  restrict_level<float>(L, C.da->N, m->cfg.nu_pre > 0 ? (const float*)L.t32.p : b, C.b32.p, s);
  DG_TRY(vcycle32(m, l + 1, C.b32.p, C.x32.p));
  prolong_level<float>(L, n, C.x32.p, x, s, g);
  if (l == 0 && m->mlp && m->mlp_active) {
    const float level_feat = 0.f;  // finest level
    for (int k = 0; k < m->mlp_sweeps; ++k) {
      DG_TRY(lapmass_residual_f32(L.A.get(), x, b, L.sm_r.p, L.acc32.p, s));
      DG_TRY(mlp_smooth_step(m->mlp->params.p, L.da.get(), L.sm_r.p, m->sm_s2.p, L.dinv32.p, L.sm_dlogbar,
                             level_feat, L.sm_hang.p, L.sm_refs.p, L.sm_nsum.p, L.sm_nmax.p, x, s));
    }
  } else {
    for (int k = 0; k < m->cfg.nu_post; ++k)
      DG_TRY(lapmass_smooth_f32(L.A.get(), x, b, L.dinv32.p, w, L.acc32.p, s, L.jcoef32(), L.jset()));
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// z = M^-1 r on the finest level: the FP64 V-cycle, or the FP32 one between
// conversions of r and z.
dg_status precond_body(dg_damg* m) {
  if (m->cfg.inner_prec == DG_PREC_F64 || m->cfg.dof == 3) return vcycle(m, 0, m->r.p, m->z.p);
  const int64_t n = m->lv[0].da->N;
  const unsigned g = grid_for(n, 256);
  convert<double, float><<<g, 256, 0, m->s>>>(m->r.p, m->r32.p, n);
  DG_TRY(vcycle32(m, 0, m->r32.p, m->z32.p));
  convert<float, double><<<g, 256, 0, m->s>>>(m->z32.p, m->z.p, n);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// Apply the preconditioner, replaying it from a CUDA graph when enabled (the
// graph is captured on the first application).
dg_status precond(dg_damg* m) {
  if (!m->cfg.use_graph) return precond_body(m);
  cudaGraphExec_t& ge = m->precond_graph[(m->mlp && m->mlp_active) ? 1 : 0];
  if (!ge) {
    // one plain application first: operator autotuning and lazy set-up
    // happen outside the capture
    DG_TRY(precond_body(m));
    cudaGraph_t graph = nullptr;
    DG_CUDA(cudaStreamBeginCapture(m->s, cudaStreamCaptureModeThreadLocal));
    dg_status st = precond_body(m);
    cudaError_t e = cudaStreamEndCapture(m->s, &graph);
    if (st != DG_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    DG_CUDA(e);
    e = cudaGraphInstantiate(&ge, graph, 0);
    cudaGraphDestroy(graph);
    DG_CUDA(e);
  }
  DG_CUDA(cudaGraphLaunch(ge, m->s));
  return DG_OK;
}

// Finest-level node data of the learned smoother (allocated on first use).
dg_status ensure_smoother_data(dg_damg* m) {
  Level& L = m->lv[0];
  if (L.sm_r.n == L.da->N && L.sm_refs.n == L.da->N) return DG_OK;
  const int64_t N = L.da->N;
  DG_TRY(L.sm_r.alloc(N));
  DG_TRY(L.sm_nsum.alloc(N));
  DG_TRY(L.sm_nmax.alloc(N));
  DG_TRY(L.sm_refs.alloc(N));
  DG_TRY(L.sm_hang.alloc(N));
  DG_TRY(m->sm_s2.alloc(1));
  DBuf<float> d32;
  const float* dinv32 = L.dinv32.p;
  if (!dinv32) {
    DG_TRY(d32.alloc(N));
    convert<double, float><<<grid_for(N, 256), 256, 0, m->s>>>(L.dinv.p, d32.p, N);
    dinv32 = d32.p;
  }
  DG_TRY(smoother_node_data(L.da.get(), dinv32, L.sm_refs.p, L.sm_hang.p, &L.sm_dlogbar, m->s));
  return DG_OK;
}

dg_status dot(dg_damg* m, const double* a, const double* b, int64_t n, double* out) {
  dot_partial<<<kRedBlocks, 256, 0, m->s>>>(a, b, n, m->part.p);
  finish_sum<<<1, 256, 0, m->s>>>(m->part.p, kRedBlocks, out);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace

extern "C" {

void dg_damg_default_config(dg_damg_config* c) {
  c->nlevels = 30;
  c->nu_pre = 2;
  c->nu_post = 2;
  c->omega = 2.0 / 3.0;
  c->rtol = 1e-8;
  c->maxit = 200;
  c->inner_prec = DG_PREC_F64;
  c->use_graph = 0;
  c->coarse_op = 0;
  c->dof = 1;
  c->mu = 1.0;
  c->lambda = 1.0;
}

}  // extern "C"

namespace {

// Level hierarchy of one mesh: coarsen + balance (omg.C:1376-1420), a mesh
// and the prolongation per level.
dg_status build_hierarchy(const dg_octree* finest, int nlevels, cudaStream_t s, std::vector<Level>& lv) {
  std::vector<std::unique_ptr<dg_octree>> trees;
  auto t0 = std::make_unique<dg_octree>();
  t0->max_depth = finest->max_depth;
  t0->n = finest->n;
  DG_TRY(t0->keys.alloc(finest->n));
  DG_CUDA(cudaMemcpy(t0->keys.p, finest->keys.p, 8 * finest->n, cudaMemcpyDeviceToDevice));
  trees.push_back(std::move(t0));
  int idx = -1;
  bool repeat = nlevels > 1;
  while (idx < nlevels - 2 && repeat) {
    dg_octree tmp;
    DG_TRY(coarsen_octree(trees.back().get(), &tmp, s));
    auto c = std::make_unique<dg_octree>();
    DG_TRY(balance_octree(&tmp, c.get(), s));
    ++idx;
    if (c->n < 500) repeat = false;
    trees.push_back(std::move(c));
  }
  lv.resize(trees.size());
  for (size_t l = 0; l < trees.size(); ++l) {
    lv[l].tree = std::move(trees[l]);
    lv[l].da = std::make_unique<dg_da>();
    DG_TRY(build_mesh(lv[l].tree.get(), lv[l].da.get(), s));
  }
  for (size_t l = 0; l + 1 < lv.size(); ++l) DG_TRY(build_prolongation(lv[l], lv[l + 1], s));
  return DG_OK;
}

// Coarsen the coarsest level further until the hierarchy has L levels (a
// batch gives every mesh the depth of the deepest one; a mesh coarsened to
// the root stays there, with identity transfers).
dg_status extend_hierarchy(std::vector<Level>& lv, size_t L, cudaStream_t s) {
  while (lv.size() < L) {
    Level& last = lv.back();
    dg_octree tmp;
    DG_TRY(coarsen_octree(last.tree.get(), &tmp, s));
    Level next;
    next.tree = std::make_unique<dg_octree>();
    DG_TRY(balance_octree(&tmp, next.tree.get(), s));
    next.da = std::make_unique<dg_da>();
    DG_TRY(build_mesh(next.tree.get(), next.da.get(), s));
    lv.push_back(std::move(next));
    DG_TRY(build_prolongation(lv[lv.size() - 2], lv.back(), s));
  }
  return DG_OK;
}

dg_status finish_create(dg_damg* m) {
  const int64_t N = int64_t(m->cfg.dof) * m->lv[0].da->N;
  DG_TRY(m->r.alloc(N));
  DG_TRY(m->z.alloc(N));
  DG_TRY(m->p.alloc(N));
  DG_TRY(m->q.alloc(N));
  DG_TRY(m->zold.alloc(N));
  if (m->cfg.inner_prec != DG_PREC_F64) {
    DG_TRY(m->r32.alloc(N));
    DG_TRY(m->z32.alloc(N));
  }
  DG_TRY(m->part.alloc(kRedBlocks));
  DG_TRY(m->scal.alloc(8));
  DG_TRY(m->d_node_mesh.alloc(N));
  DG_TRY(m->mesh_part.alloc(m->nmesh));
  const std::vector<int64_t>& no = m->mesh_node_off[0];
  for (int i = 0; i < m->nmesh; ++i)
    fill_u16<<<grid_for(no[i + 1] - no[i], 256), 256, 0, m->s>>>(m->d_node_mesh.p, no[i], no[i + 1], uint16_t(i));
  DG_CUDA(cudaGetLastError());
  for (size_t l = 0; l + 1 < m->lv.size(); ++l) {
    DG_TRY(build_restriction(m->lv[l], m->lv[l + 1].da->N, m->s));
    DG_TRY(build_weight_codes(m->lv[l], m->s));
  }
  return set_operators(m, nullptr);
}

// Concatenate per-mesh meshes of one level into one mesh (node ids offset).
dg_status concat_das(const std::vector<dg_da*>& in, dg_da* out, cudaStream_t s) {
  out->D = in[0]->D;
  int64_t E = 0, N = 0, P = 0;
  for (dg_da* d : in) {
    DG_CHECK(d->D == out->D, DG_EINVAL, "batched meshes must share maxDepth");
    E += d->E;
    N += d->N;
    P += d->P;
  }
  DG_CHECK(N < (int64_t(1) << 32), DG_EINVAL, "batch too large for 32-bit node ids");
  out->E = E;
  out->N = N;
  out->P = P;
  DG_TRY(out->nl.alloc(8 * E));
  DG_TRY(out->meta.alloc(E));
  DG_TRY(out->ekey.alloc(E));
  DG_TRY(out->nkey.alloc(N));
  int64_t eo = 0, no = 0;
  for (dg_da* d : in) {
    for (int v = 0; v < 8; ++v)
      copy_add_u32<<<grid_for(d->E, 256), 256, 0, s>>>(out->nl.p + int64_t(v) * E + eo, d->nl.p + int64_t(v) * d->E,
                                                        d->E, uint32_t(no));
    DG_CUDA(cudaMemcpyAsync(out->meta.p + eo, d->meta.p, 4 * d->E, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(cudaMemcpyAsync(out->ekey.p + eo, d->ekey.p, 8 * d->E, cudaMemcpyDeviceToDevice, s));
    DG_CUDA(cudaMemcpyAsync(out->nkey.p + no, d->nkey.p, 8 * d->N, cudaMemcpyDeviceToDevice, s));
    eo += d->E;
    no += d->N;
  }
  DG_CUDA(cudaGetLastError());
  // no octet tables: the meshes' parent keys coincide across the batch, so
  // the octet kernels are not offered for a concatenated level
  return build_tiles(out, s);
}

// Concatenate per-mesh prolongations (block diagonal).
dg_status concat_prolong(const std::vector<Level*>& fine, const std::vector<int64_t>& coarse_node_off, Level& out,
                         cudaStream_t s) {
  int64_t rows = 0, nnz = 0;
  for (Level* f : fine) {
    rows += f->da->N;
    nnz += f->pval.n;
  }
  DG_TRY(out.pptr.alloc(rows + 1));
  DG_TRY(out.pcol.alloc(nnz > 0 ? nnz : 1));
  DG_TRY(out.pval.alloc(nnz > 0 ? nnz : 1));
  int64_t ro = 0, zo = 0;
  for (size_t i = 0; i < fine.size(); ++i) {
    Level* f = fine[i];
    const int64_t r = f->da->N, z = f->pval.n;
    copy_add_u32<<<grid_for(r + 1, 256), 256, 0, s>>>(out.pptr.p + ro, f->pptr.p, r + 1, uint32_t(zo));
    if (z) {
      copy_add_u32<<<grid_for(z, 256), 256, 0, s>>>(out.pcol.p + zo, f->pcol.p, z, uint32_t(coarse_node_off[i]));
      DG_CUDA(cudaMemcpyAsync(out.pval.p + zo, f->pval.p, 8 * z, cudaMemcpyDeviceToDevice, s));
    }
    ro += r;
    zo += z;
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace

extern "C" {

dg_status dg_damg_create(const dg_octree* finest, const dg_damg_config* cfg, dg_damg** out) {
  DG_CHECK(finest && out, DG_EINVAL, "damg_create: bad arguments");
  return dg_damg_create_batch(&finest, 1, cfg, out);
}

dg_status dg_damg_create_batch(const dg_octree* const* finest, int count, const dg_damg_config* cfg, dg_damg** out) {
  DG_CHECK(finest && out && count >= 1 && count <= 65535, DG_EINVAL, "damg_create_batch: bad arguments");
  auto m = std::make_unique<dg_damg>();
  if (cfg) m->cfg = *cfg; else dg_damg_default_config(&m->cfg);
  DG_CHECK(m->cfg.nlevels >= 1, DG_EINVAL, "damg_create: nlevels must be >= 1");
  DG_CHECK(m->cfg.dof == 1 || m->cfg.dof == 3, DG_EINVAL, "damg_create: dof must be 1 or 3");
  DG_CHECK(m->cfg.dof == 1 || (count == 1 && m->cfg.inner_prec == DG_PREC_F64 && m->cfg.coarse_op == 0),
           DG_ENOTIMPL, "damg_create: dof 3 (elasticity) is one mesh with the FP64 V-cycle and coarse_op 0");
  DG_CUDA(cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking));
  cudaStream_t s = m->s;
  m->nmesh = count;
  if (count == 1) {
    DG_TRY(build_hierarchy(finest[0], m->cfg.nlevels, s, m->lv));
    for (Level& L : m->lv) {
      m->mesh_elem_off.push_back({0, L.da->E});
      m->mesh_node_off.push_back({0, L.da->N});
    }
  } else {
    // every mesh gets the same number of levels: the largest natural count,
    // the shallower hierarchies coarsened further (so that every coarsest
    // level stays small enough for the dense direct solve)
    std::vector<std::vector<Level>> per(count);
    size_t L = 0;
    for (int i = 0; i < count; ++i) {
      DG_CHECK(finest[i], DG_EINVAL, "damg_create_batch: null octree");
      DG_TRY(build_hierarchy(finest[i], m->cfg.nlevels, s, per[i]));
      L = per[i].size() > L ? per[i].size() : L;
    }
    for (int i = 0; i < count; ++i) DG_TRY(extend_hierarchy(per[i], L, s));
    m->lv.resize(L);
    for (size_t l = 0; l < L; ++l) {
      std::vector<dg_da*> das;
      std::vector<int64_t> eo{0}, no{0};
      for (int i = 0; i < count; ++i) {
        das.push_back(per[i][l].da.get());
        eo.push_back(eo.back() + per[i][l].da->E);
        no.push_back(no.back() + per[i][l].da->N);
      }
      m->lv[l].da = std::make_unique<dg_da>();
      DG_TRY(concat_das(das, m->lv[l].da.get(), s));
      m->mesh_elem_off.push_back(eo);
      m->mesh_node_off.push_back(no);
    }
    for (size_t l = 0; l + 1 < L; ++l) {
      std::vector<Level*> fine;
      for (int i = 0; i < count; ++i) fine.push_back(&per[i][l]);
      DG_TRY(concat_prolong(fine, m->mesh_node_off[l + 1], m->lv[l], s));
    }
    DG_CUDA(cudaStreamSynchronize(s));
  }
  DG_TRY(finish_create(m.get()));
  *out = m.release();
  return DG_OK;
}

int dg_damg_batch_count(const dg_damg* m) { return m ? m->nmesh : 0; }

dg_status dg_damg_batch_offsets(const dg_damg* m, int level, int64_t* elem_off, int64_t* node_off) {
  DG_CHECK(m && level >= 0 && level < int(m->lv.size()), DG_EINVAL, "damg_batch_offsets: bad level");
  for (int i = 0; i <= m->nmesh; ++i) {
    if (elem_off) elem_off[i] = m->mesh_elem_off[level][i];
    if (node_off) node_off[i] = m->mesh_node_off[level][i];
  }
  return DG_OK;
}

dg_status dg_damg_set_lapmass(dg_damg* m, const double* coef) {
  DG_CHECK(m, DG_EINVAL, "damg_set_lapmass: null handle");
  return set_operators(m, coef);
}

dg_status dg_damg_set_tolerances(dg_damg* m, double rtol, int maxit) {
  DG_CHECK(m, DG_EINVAL, "damg_set_tolerances: null handle");
  DG_CHECK(rtol > 0.0 && rtol < 1.0 && maxit > 0, DG_EINVAL, "damg_set_tolerances: rtol in (0,1), maxit > 0");
  m->cfg.rtol = rtol;
  m->cfg.maxit = maxit;
  return DG_OK;
}

int dg_damg_levels(const dg_damg* m) { return m ? int(m->lv.size()) : 0; }

dg_status dg_damg_level_sizes(const dg_damg* m, int64_t* E, int64_t* N) {
  DG_CHECK(m, DG_EINVAL, "damg_level_sizes: null handle");
  for (size_t l = 0; l < m->lv.size(); ++l) {
    if (E) E[l] = m->lv[l].da->E;
    if (N) N[l] = m->lv[l].da->N;
  }
  return DG_OK;
}

dg_da* dg_damg_level_da(dg_damg* m, int level) {
  if (!m || level < 0 || level >= int(m->lv.size())) return nullptr;
  return m->lv[level].da.get();
}

dg_status dg_damg_prolong(dg_damg* m, int level, const double* xc, double* xf, int on_device) {
  DG_CHECK(m && level >= 0 && level + 1 < int(m->lv.size()), DG_EINVAL, "damg_prolong: bad level");
  Level& F = m->lv[level];
  Level& C = m->lv[level + 1];
  const int dof = m->cfg.dof;
  const int64_t nf = dof * F.da->N, nc = dof * C.da->N;
  DBuf<double> dc, df;
  const double* pc = xc;
  double* pf = xf;
  if (!on_device) {
    DG_TRY(dc.alloc(nc));
    DG_TRY(df.alloc(nf));
    DG_CUDA(cudaMemcpy(dc.p, xc, 8 * nc, cudaMemcpyHostToDevice));
    DG_CUDA(cudaMemcpy(df.p, xf, 8 * nf, cudaMemcpyHostToDevice));
    pc = dc.p;
    pf = df.p;
  }
  if (on_device) DG_CUDA(cudaDeviceSynchronize());
  if (dof == 3)
    prolong_add3<<<grid_for(F.da->N, 256), 256, 0, m->s>>>(F.pptr.p, F.pcol.p, F.pval.p, F.da->N, pc, pf);
  else
    prolong_level<double>(F, nf, pc, pf, m->s, grid_for(nf, 256));
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(m->s));
  if (!on_device) DG_CUDA(cudaMemcpy(xf, df.p, 8 * nf, cudaMemcpyDeviceToHost));
  return DG_OK;
}

dg_status dg_damg_restrict(dg_damg* m, int level, const double* rf, double* rc, int on_device) {
  DG_CHECK(m && level >= 0 && level + 1 < int(m->lv.size()), DG_EINVAL, "damg_restrict: bad level");
  Level& F = m->lv[level];
  Level& C = m->lv[level + 1];
  const int dof = m->cfg.dof;
  const int64_t nf = dof * F.da->N, nc = dof * C.da->N;
  DBuf<double> dc, df;
  const double* pf = rf;
  double* pc = rc;
  if (!on_device) {
    DG_TRY(dc.alloc(nc));
    DG_TRY(df.alloc(nf));
    DG_CUDA(cudaMemcpy(df.p, rf, 8 * nf, cudaMemcpyHostToDevice));
    pf = df.p;
    pc = dc.p;
  }
  if (on_device) DG_CUDA(cudaDeviceSynchronize());
  if (dof == 3)
    restrict_gather3<<<grid_for(C.da->N, 256, 16), 256, 0, m->s>>>(F.rptr.p, F.rcol.p, F.rval.p, C.da->N, pf, pc);
  else
    restrict_level<double>(F, nc, pf, pc, m->s);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaStreamSynchronize(m->s));
  if (!on_device) DG_CUDA(cudaMemcpy(rc, dc.p, 8 * nc, cudaMemcpyDeviceToHost));
  return DG_OK;
}

// Preconditioned CG, zero initial guess, stop on ||b - A x||_2 <= rtol ||b||_2.
dg_status dg_damg_solve(dg_damg* m, const double* b, double* x, int on_device, dg_solve_report* rep) {
  DG_CHECK(m && b && x, DG_EINVAL, "damg_solve: bad arguments");
  cudaStream_t s = m->s;
  Level& L = m->lv[0];
  const int64_t n = int64_t(m->cfg.dof) * L.da->N;
  const unsigned g = grid_for(n, 256);
  DBuf<double> db, dx;
  const double* pb = b;
  double* px = x;
  // the caller's device data may come from any stream
  if (on_device) DG_CUDA(cudaDeviceSynchronize());
  // the vector kernels read 16-byte pairs: host data, and device data not
  // 16-byte aligned, go through the solver's own buffers
  const bool staged = !on_device || ((reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(x)) & 15) != 0;
  if (staged) {
    DG_TRY(db.alloc(n));
    DG_TRY(dx.alloc(n));
    DG_CUDA(cudaMemcpyAsync(db.p, b, 8 * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    pb = db.p;
    px = dx.p;
  }
  cudaEvent_t e0, e1;
  DG_CUDA(cudaEventCreate(&e0));
  DG_CUDA(cudaEventCreate(&e1));
  DG_CUDA(cudaEventRecord(e0, s));
  double* sc = m->scal.p;  // [0] bb, [1] rz, [2] pq, [3] rr, [4] rz_new
  DG_CUDA(cudaMemsetAsync(px, 0, 8 * n, s));
  DG_CUDA(cudaMemcpyAsync(m->r.p, pb, 8 * n, cudaMemcpyDeviceToDevice, s));
  DG_TRY(dot(m, pb, pb, n, sc + 0));
  double hb = 0;
  DG_CUDA(cudaMemcpyAsync(&hb, sc + 0, 8, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  const double bnorm = std::sqrt(hb);
  // independent meshes: each must reach the tolerance on its own ||b_i||
  const int nm = m->nmesh;
  std::vector<double> bb(nm, hb), rr(nm);
  auto mesh_norms = [&](const double* v, std::vector<double>& out) -> dg_status {
    DG_CUDA(cudaMemsetAsync(m->mesh_part.p, 0, 8 * nm, s));
    seg_sqnorm<<<kRedBlocks, 256, 8 * nm, s>>>(v, n, m->d_node_mesh.p, nm, m->mesh_part.p);
    DG_CUDA(cudaGetLastError());
    DG_CUDA(cudaMemcpyAsync(out.data(), m->mesh_part.p, 8 * nm, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    return DG_OK;
  };
  if (nm > 1) DG_TRY(mesh_norms(pb, bb));
  int it = 0;
  double rel = bnorm > 0 ? 1.0 : 0.0;
  bool conv = bnorm == 0;
  const bool flexible = m->cfg.inner_prec != DG_PREC_F64;
  int fallbacks = 0;
  double prev_rel = 1.0;
  if (m->mlp) m->mlp_active = true;  // a new solve starts with the learned smoother again
  if (!conv) {
    DG_TRY(precond(m));
    DG_CUDA(cudaMemcpyAsync(m->p.p, m->z.p, 8 * n, cudaMemcpyDeviceToDevice, s));
    DG_TRY(dot(m, m->r.p, m->z.p, n, sc + 1));
    for (it = 1; it <= m->cfg.maxit; ++it) {
      DG_TRY(level_op(L, m->p.p, m->q.p, s));
      DG_TRY(dot(m, m->p.p, m->q.p, n, sc + 2));
      cg_update<<<kRedBlocks, 256, 0, s>>>(px, m->r.p, m->p.p, m->q.p, n, sc + 1, sc + 2, m->part.p);
      finish_sum<<<1, 256, 0, s>>>(m->part.p, kRedBlocks, sc + 3);
      if (nm > 1) {
        DG_TRY(mesh_norms(m->r.p, rr));
        rel = 0;
        for (int i = 0; i < nm; ++i)
          if (bb[i] > 0) rel = std::max(rel, std::sqrt(rr[i] / bb[i]));
      } else {
        double hr = 0;
        DG_CUDA(cudaMemcpyAsync(&hr, sc + 3, 8, cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        rel = std::sqrt(hr) / bnorm;
      }
      if (!(rel == rel)) break;  // NaN: stop and report
      if (rel <= m->cfg.rtol) {
        conv = true;
        break;
      }
      // the FP64 residual judges the learned smoother: when it fails to fall
      // by the set factor, plain damped Jacobi takes over for this solve
      if (m->mlp && m->mlp_active && rel > m->mlp_fallback * prev_rel) {
        m->mlp_active = false;
        ++fallbacks;
      }
      prev_rel = rel;
      if (flexible) DG_CUDA(cudaMemcpyAsync(m->zold.p, m->z.p, 8 * n, cudaMemcpyDeviceToDevice, s));
      DG_TRY(precond(m));
      DG_TRY(dot(m, m->r.p, m->z.p, n, sc + 4));
      if (flexible) {
        DG_TRY(dot(m, m->r.p, m->zold.p, n, sc + 5));
        cg_direction_flex<<<g, 256, 0, s>>>(m->p.p, m->z.p, n, sc + 4, sc + 5, sc + 1);
      } else {
        cg_direction<<<g, 256, 0, s>>>(m->p.p, m->z.p, n, sc + 4, sc + 1);
      }
      DG_CUDA(cudaMemcpyAsync(sc + 1, sc + 4, 8, cudaMemcpyDeviceToDevice, s));
    }
  }
  DG_CUDA(cudaEventRecord(e1, s));
  DG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (staged) {
    DG_CUDA(cudaMemcpyAsync(x, dx.p, 8 * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
  }
  if (rep) {
    rep->iterations = it > m->cfg.maxit ? m->cfg.maxit : it;
    rep->converged = conv ? 1 : 0;
    rep->rel_residual = rel;
    rep->solve_ms = ms;
    rep->smoother_fallbacks = fallbacks;
  }
  DG_TRY(device_wait_status(s));  // an operator kernel gave up waiting: the result is not valid
  return conv ? DG_OK : DG_ENOTCONVERGED;
}

void dg_damg_destroy(dg_damg* m) { delete m; }

}  // extern "C"

// ------------------------------------------------------ multi-RHS solve ---
// R right-hand sides solved together (the batched form with many right-hand
// sides on one mesh): node-major [N][R] blocks, one flexible PCG per
// column in FP64 (its own step lengths, frozen once it has converged) around
// one V-cycle per iteration for all columns -- the operator applications of
// every level are the octet multi-RHS kernel (a warp per parent octant and
// 32 columns), the smoother, residual and transfers elementwise or per row
// over the R columns, the coarsest level the dense inverse times the block.
namespace {

template <class T>
__global__ void mv_jacobi_first(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv, T omega,
                                int64_t n, int R) {
  for (int64_t i = gtid(); i < n; i += gstride()) x[i] = omega * dinv[i / R] * b[i];
}
template <class T>
__global__ void mv_jacobi_update(T* __restrict__ x, const T* __restrict__ b, const T* __restrict__ dinv,
                                 const T* __restrict__ t, T omega, int64_t n, int R) {
  for (int64_t i = gtid(); i < n; i += gstride()) x[i] += omega * dinv[i / R] * (b[i] - t[i]);
}
template <class T>
__global__ void mv_residual(const T* __restrict__ b, const T* __restrict__ t, T* __restrict__ r, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) r[i] = b[i] - t[i];
}
// rc[c][:] = sum_k R[c][k] rf[k][:]  (thread per (row, column): coalesced rows)
template <class T>
__global__ void mv_restrict(const uint32_t* __restrict__ rptr, const uint32_t* __restrict__ rcol,
                            const T* __restrict__ rval, int64_t Nc, int R, const T* __restrict__ rf,
                            T* __restrict__ rc) {
  for (int64_t i = gtid(); i < Nc * R; i += gstride()) {
    const int64_t c = i / R;
    const int j = int(i - c * R);
    T acc = T(0);
    for (uint32_t k = rptr[c]; k < rptr[c + 1]; ++k) acc += rval[k] * rf[int64_t(rcol[k]) * R + j];
    rc[i] = acc;
  }
}
template <class T>
__global__ void mv_prolong_add(const uint32_t* __restrict__ pptr, const uint32_t* __restrict__ pcol,
                               const T* __restrict__ pval, int64_t Nf, int R, const T* __restrict__ xc,
                               T* __restrict__ xf) {
  for (int64_t i = gtid(); i < Nf * R; i += gstride()) {
    const int64_t f = i / R;
    const int j = int(i - f * R);
    T acc = T(0);
    for (uint32_t k = pptr[f]; k < pptr[f + 1]; ++k) acc += pval[k] * xc[int64_t(pcol[k]) * R + j];
    xf[i] += acc;
  }
}
// x = Ainv b for a block of R columns (one dense block: a single mesh)
__global__ void mv_coarse(const double* __restrict__ Ainv, int64_t n, int R, const double* __restrict__ b,
                          double* __restrict__ x) {
  for (int64_t i = gtid(); i < n * R; i += gstride()) {
    const int64_t r = i / R;
    const int j = int(i - r * R);
    const double* a = Ainv + r * n;
    double acc = 0;
    for (int64_t k = 0; k < n; ++k) acc += a[k] * b[k * R + j];
    x[i] = acc;
  }
}
template <class A, class B>
__global__ void mv_convert(const A* __restrict__ a, B* __restrict__ b, int64_t n) {
  for (int64_t i = gtid(); i < n; i += gstride()) b[i] = B(a[i]);
}
// Column sums of a[i][j] b[i][j] over the N rows: per block R partial sums
// (256 / R rows at a time), then one pass over the blocks.
constexpr int kMvDotBlocks = 592;
__global__ void __launch_bounds__(256) mv_dot_partial(const double* __restrict__ a, const double* __restrict__ b,
                                                      int64_t N, int R, double* __restrict__ part) {
  __shared__ double acc[256];
  const int rows = 256 / R, j = int(threadIdx.x) % R, r0 = int(threadIdx.x) / R;
  double v = 0;
  for (int64_t i = int64_t(blockIdx.x) * rows + r0; i < N; i += int64_t(gridDim.x) * rows)
    v += a[i * R + j] * b[i * R + j];
  acc[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < R) {
    double t = 0;
    for (int k = 0; k < rows; ++k) t += acc[k * R + threadIdx.x];
    part[int64_t(blockIdx.x) * R + threadIdx.x] = t;
  }
}
__global__ void mv_dot_finish(const double* __restrict__ part, int nb, int R, double* __restrict__ out) {
  for (int j = threadIdx.x; j < R; j += blockDim.x) {
    double t = 0;
    for (int k = 0; k < nb; ++k) t += part[int64_t(k) * R + j];
    out[j] = t;
  }
}
// per-column PCG steps: y += s a[j] x; p = z + b[j] p
__global__ void mv_axpy(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ a,
                        double sgn, int64_t n, int R) {
  for (int64_t i = gtid(); i < n; i += gstride()) y[i] += sgn * a[i % R] * x[i];
}
__global__ void mv_direction(double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ b,
                             int64_t n, int R) {
  for (int64_t i = gtid(); i < n; i += gstride()) p[i] = z[i] + b[i % R] * p[i];
}
// alpha = rz / pq and the flexible beta = (rz_new - (r, z_old)) / rz, zero for
// converged columns (done[j]); rz <- rz_new
__global__ void mv_alpha(const double* __restrict__ rz, const double* __restrict__ pq,
                         const uint8_t* __restrict__ done, double* __restrict__ alpha, int R) {
  for (int j = threadIdx.x; j < R; j += blockDim.x) alpha[j] = (done[j] || pq[j] == 0) ? 0.0 : rz[j] / pq[j];
}
__global__ void mv_beta(const double* __restrict__ rzn, const double* __restrict__ rzo, double* __restrict__ rz,
                        const uint8_t* __restrict__ done, double* __restrict__ beta, int R, int flexible) {
  for (int j = threadIdx.x; j < R; j += blockDim.x) {
    const double num = flexible ? rzn[j] - rzo[j] : rzn[j];
    beta[j] = (done[j] || rz[j] == 0) ? 0.0 : num / rz[j];
    rz[j] = rzn[j];
  }
}

// Work blocks of every level for one right-hand-side count R.
template <class T>
struct MultiLevels {
  std::vector<DBuf<T>> x, b, t;
};

template <class T>
dg_status vcycle_multi(dg_damg* m, size_t l, const T* b, T* x, int R, MultiLevels<T>& W, DBuf<double>& cb,
                       DBuf<double>& cx) {
  cudaStream_t s = m->s;
  Level& L = m->lv[l];
  const int64_t N = L.da->N, n = N * R;
  const unsigned g = grid_for(n, 256, 16);
  if (l + 1 == m->lv.size()) {
    if constexpr (sizeof(T) == 8) {
      mv_coarse<<<grid_for(n, 256, 16), 256, 0, s>>>(m->Ainv.p, N, R, b, x);
    } else {
      mv_convert<float, double><<<g, 256, 0, s>>>(b, cb.p, n);
      mv_coarse<<<grid_for(n, 256, 16), 256, 0, s>>>(m->Ainv.p, N, R, cb.p, cx.p);
      mv_convert<double, float><<<g, 256, 0, s>>>(cx.p, x, n);
    }
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  }
  const T* dinv;
  const T* coef;
  const T *pval, *rval;
  if constexpr (sizeof(T) == 8) {
    dinv = L.dinv.p;
    coef = L.A->coef.p;
    pval = L.pval.p;
    rval = L.rval.p;
  } else {
    dinv = L.dinv32.p;
    coef = L.A->coef32.p;
    pval = L.pval32.p;
    rval = L.rval32.p;
  }
  const T w = T(m->cfg.omega);
  T* t = W.t[l].p;
  if (m->cfg.nu_pre > 0) {
    mv_jacobi_first<T><<<g, 256, 0, s>>>(x, b, dinv, w, n, R);
    for (int k = 1; k < m->cfg.nu_pre; ++k) {
      DG_TRY(mrhs_octet_apply<T>(L.A.get(), coef, x, t, R, s));
      mv_jacobi_update<T><<<g, 256, 0, s>>>(x, b, dinv, t, w, n, R);
    }
    DG_TRY(mrhs_octet_apply<T>(L.A.get(), coef, x, t, R, s));
    mv_residual<T><<<g, 256, 0, s>>>(b, t, t, n);
  } else {
    DG_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, s));
  }
  Level& C = m->lv[l + 1];
  const int64_t Nc = C.da->N;
  mv_restrict<T><<<grid_for(Nc * R, 256, 16), 256, 0, s>>>(L.rptr.p, L.rcol.p, rval, Nc, R,
                                                           m->cfg.nu_pre > 0 ? (const T*)t : b, W.b[l + 1].p);
  DG_TRY(vcycle_multi<T>(m, l + 1, W.b[l + 1].p, W.x[l + 1].p, R, W, cb, cx));
  mv_prolong_add<T><<<g, 256, 0, s>>>(L.pptr.p, L.pcol.p, pval, N, R, W.x[l + 1].p, x);
  for (int k = 0; k < m->cfg.nu_post; ++k) {
    DG_TRY(mrhs_octet_apply<T>(L.A.get(), coef, x, t, R, s));
    mv_jacobi_update<T><<<g, 256, 0, s>>>(x, b, dinv, t, w, n, R);
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

template <class T>
dg_status alloc_multi_levels(dg_damg* m, int R, MultiLevels<T>& W) {
  const size_t L = m->lv.size();
  W.x.resize(L);
  W.b.resize(L);
  W.t.resize(L);
  for (size_t l = 0; l < L; ++l) {
    const int64_t n = m->lv[l].da->N * int64_t(R);
    DG_TRY(W.x[l].alloc(n));
    DG_TRY(W.b[l].alloc(n));
    DG_TRY(W.t[l].alloc(n));
  }
  return DG_OK;
}

}  // namespace

extern "C" {

dg_status dg_damg_solve_multi(dg_damg* m, const double* B, double* X, int nrhs, int on_device,
                              dg_solve_report* rep) {
  DG_CHECK(m && B && X, DG_EINVAL, "damg_solve_multi: bad arguments");
  const int R = nrhs;
  DG_CHECK(R > 0 && R % 32 == 0 && R <= 256 && 256 % R == 0, DG_EINVAL,
           "damg_solve_multi: nrhs must be 32, 64, 128 or 256");
  DG_CHECK(m->cfg.dof == 1 && m->nmesh == 1 && m->cfg.coarse_op == 0, DG_ENOTIMPL,
           "damg_solve_multi: one mesh, the scalar operator, coarse_op 0");
  DG_CHECK(m->lv.back().da->N <= 32768, DG_EINVAL, "damg_solve_multi: coarsest level too large");
  for (const Level& L : m->lv) DG_CHECK(L.da->octs.n > 0, DG_EINVAL, "damg_solve_multi: mesh without octets");
  cudaStream_t s = m->s;
  const Level& L0 = m->lv[0];
  const int64_t N = L0.da->N, n = N * R;
  const bool f32 = m->cfg.inner_prec != DG_PREC_F64;
  if (on_device) DG_CUDA(cudaDeviceSynchronize());
  DBuf<double> b, x, r, z, zo, p, q, part, sc, cb, cx;
  DBuf<float> r32, z32;
  DBuf<uint8_t> done;
  for (DBuf<double>* v : {&b, &x, &r, &z, &zo, &p, &q}) DG_TRY(v->alloc(n));
  DG_TRY(part.alloc(int64_t(kMvDotBlocks) * R));
  DG_TRY(sc.alloc(8 * int64_t(R)));  // bb, rz, pq, rr, rzn, rzo, alpha, beta
  DG_TRY(done.alloc(R));
  const int64_t nc = m->lv.back().da->N * int64_t(R);
  DG_TRY(cb.alloc(nc));
  DG_TRY(cx.alloc(nc));
  MultiLevels<float> W32;
  MultiLevels<double> W64;
  if (f32) {
    DG_TRY(alloc_multi_levels<float>(m, R, W32));
    DG_TRY(r32.alloc(n));
    DG_TRY(z32.alloc(n));
  } else {
    DG_TRY(alloc_multi_levels<double>(m, R, W64));
  }
  double* bb = sc.p;
  double *rz = sc.p + R, *pq = sc.p + 2 * R, *rr = sc.p + 3 * R, *rzn = sc.p + 4 * R, *rzo = sc.p + 5 * R;
  double *alpha = sc.p + 6 * R, *beta = sc.p + 7 * R;
  DG_CUDA(cudaMemcpyAsync(b.p, B, 8 * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  DG_CUDA(cudaMemsetAsync(done.p, 0, R, s));
  DG_CUDA(cudaStreamSynchronize(s));
  auto dots = [&](const double* u, const double* v, double* out) -> dg_status {
    mv_dot_partial<<<kMvDotBlocks, 256, 0, s>>>(u, v, N, R, part.p);
    mv_dot_finish<<<1, 256, 0, s>>>(part.p, kMvDotBlocks, R, out);
    DG_CUDA(cudaGetLastError());
    return DG_OK;
  };
  const unsigned g = grid_for(n, 256, 16);
  auto precond = [&]() -> dg_status {
    if (f32) {
      mv_convert<double, float><<<g, 256, 0, s>>>(r.p, r32.p, n);
      DG_TRY(vcycle_multi<float>(m, 0, r32.p, z32.p, R, W32, cb, cx));
      mv_convert<float, double><<<g, 256, 0, s>>>(z32.p, z.p, n);
      DG_CUDA(cudaGetLastError());
      return DG_OK;
    }
    return vcycle_multi<double>(m, 0, r.p, z.p, R, W64, cb, cx);
  };
  cudaEvent_t e0, e1;
  DG_CUDA(cudaEventCreate(&e0));
  DG_CUDA(cudaEventCreate(&e1));
  DG_CUDA(cudaEventRecord(e0, s));
  DG_CUDA(cudaMemsetAsync(x.p, 0, 8 * n, s));
  DG_CUDA(cudaMemcpyAsync(r.p, b.p, 8 * n, cudaMemcpyDeviceToDevice, s));
  DG_TRY(dots(b.p, b.p, bb));
  std::vector<double> hbb(R), hrr(R);
  std::vector<uint8_t> hdone(R, 0);
  DG_CUDA(cudaMemcpyAsync(hbb.data(), bb, 8 * R, cudaMemcpyDeviceToHost, s));
  DG_TRY(precond());
  DG_CUDA(cudaMemcpyAsync(p.p, z.p, 8 * n, cudaMemcpyDeviceToDevice, s));
  DG_TRY(dots(r.p, z.p, rz));
  const int flexible = f32 ? 1 : 0;
  int it = 0;
  double worst = 1.0;
  bool conv = false;
  DG_CUDA(cudaStreamSynchronize(s));
  for (int j = 0; j < R; ++j)
    if (hbb[j] == 0) hdone[j] = 1;
  for (it = 1; it <= m->cfg.maxit; ++it) {
    DG_TRY(mrhs_octet_apply<double>(L0.A.get(), L0.A->coef.p, p.p, q.p, R, s));
    DG_TRY(dots(p.p, q.p, pq));
    mv_alpha<<<1, 256, 0, s>>>(rz, pq, done.p, alpha, R);
    mv_axpy<<<g, 256, 0, s>>>(x.p, p.p, alpha, 1.0, n, R);
    mv_axpy<<<g, 256, 0, s>>>(r.p, q.p, alpha, -1.0, n, R);
    DG_TRY(dots(r.p, r.p, rr));
    DG_CUDA(cudaMemcpyAsync(hrr.data(), rr, 8 * R, cudaMemcpyDeviceToHost, s));
    DG_CUDA(cudaStreamSynchronize(s));
    worst = 0;
    bool all = true;
    for (int j = 0; j < R; ++j) {
      const double rel = hbb[j] > 0 ? std::sqrt(hrr[j] / hbb[j]) : 0.0;
      if (!(rel == rel)) worst = rel;
      else worst = std::max(worst, rel);
      if (rel <= m->cfg.rtol) hdone[j] = 1;
      all = all && hdone[j];
    }
    if (!(worst == worst)) break;
    if (all) {
      conv = true;
      break;
    }
    DG_CUDA(cudaMemcpyAsync(done.p, hdone.data(), R, cudaMemcpyHostToDevice, s));
    DG_CUDA(cudaMemcpyAsync(zo.p, z.p, 8 * n, cudaMemcpyDeviceToDevice, s));
    DG_TRY(precond());
    DG_TRY(dots(r.p, z.p, rzn));
    if (flexible) DG_TRY(dots(r.p, zo.p, rzo));
    mv_beta<<<1, 256, 0, s>>>(rzn, rzo, rz, done.p, beta, R, flexible);
    mv_direction<<<g, 256, 0, s>>>(p.p, z.p, beta, n, R);
  }
  DG_CUDA(cudaEventRecord(e1, s));
  DG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DG_CUDA(cudaMemcpyAsync(X, x.p, 8 * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  if (rep) {
    rep->iterations = it > m->cfg.maxit ? m->cfg.maxit : it;
    rep->converged = conv ? 1 : 0;
    rep->rel_residual = worst;
    rep->solve_ms = ms;
    rep->smoother_fallbacks = 0;
  }
  return conv ? DG_OK : DG_ENOTCONVERGED;
}

dg_status dg_vec_dot(const double* x, const double* y, int64_t n, double* result, void* stream) {
  DG_CHECK(result && n >= 0 && (n == 0 || (x && y)), DG_EINVAL, "vec_dot: bad arguments");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  DBuf<double> part;  // one partial sum per reduction block
  DG_TRY(part.alloc(kRedBlocks));
  if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0)
    dot_partial<<<kRedBlocks, 256, 0, s>>>(x, y, n, part.p);
  else
    dot_partial_any<<<kRedBlocks, 256, 0, s>>>(x, y, n, part.p);
  finish_sum<<<1, 256, 0, s>>>(part.p, kRedBlocks, result);
  DG_CUDA(cudaGetLastError());
  // the partials are released when this call returns
  DG_CUDA(cudaStreamSynchronize(s));
  return DG_OK;
}

dg_status dg_damg_set_smoother(dg_damg* m, dg_mlp* mlp, int sweeps, double fallback_ratio) {
  DG_CHECK(m && sweeps >= 1 && fallback_ratio > 0, DG_EINVAL, "damg_set_smoother: bad arguments");
  DG_CHECK(!mlp || m->cfg.dof == 1, DG_ENOTIMPL, "damg_set_smoother: the learned smoother is scalar (dof 1)");
  DG_CHECK(!mlp || m->cfg.inner_prec != DG_PREC_F64, DG_EINVAL,
           "damg_set_smoother: the learned smoother runs in the FP32 inner V-cycle (inner_prec F32)");
  if (mlp) DG_TRY(ensure_smoother_data(m));
  m->mlp = mlp;
  m->mlp_sweeps = sweeps;
  m->mlp_fallback = fallback_ratio;
  m->mlp_active = mlp != nullptr;
  m->drop_graphs();
  return DG_OK;
}

dg_status dg_damg_features(dg_damg* m, const double* r, float* F, float* scale) {
  DG_CHECK(m && r && F, DG_EINVAL, "damg_features: bad arguments");
  DG_CUDA(cudaDeviceSynchronize());
  DG_TRY(ensure_smoother_data(m));
  Level& L = m->lv[0];
  DBuf<float> d32, sc;
  const float* dinv32 = L.dinv32.p;
  if (!dinv32) {
    DG_TRY(d32.alloc(L.da->N));
    convert<double, float><<<grid_for(L.da->N, 256), 256, 0, m->s>>>(L.dinv.p, d32.p, L.da->N);
    dinv32 = d32.p;
  }
  DG_TRY(sc.alloc(1));
  DG_TRY(mlp_features_f64(L.da.get(), r, m->sm_s2.p, dinv32, L.sm_dlogbar, 0.f, L.sm_hang.p, L.sm_refs.p,
                          L.sm_nsum.p, L.sm_nmax.p, F, sc.p, m->s));
  float h = 0;
  DG_CUDA(cudaMemcpyAsync(&h, sc.p, 4, cudaMemcpyDeviceToHost, m->s));
  DG_CUDA(cudaStreamSynchronize(m->s));
  if (scale) *scale = h;
  return DG_OK;
}

dg_status dg_damg_level_apply(dg_damg* m, int level, const double* x, double* y, int on_device) {
  DG_CHECK(m && x && y && level >= 0 && size_t(level) < m->lv.size(), DG_EINVAL, "damg_level_apply: bad arguments");
  Level& L = m->lv[size_t(level)];
  DG_CHECK(L.A, DG_EINVAL, "damg_level_apply: no operator set");
  const int64_t n = int64_t(L.A->dof) * L.da->N;
  const double* xd = x;
  double* yd = y;
  if (!on_device) {
    DG_CUDA(cudaMemcpyAsync(L.x.p, x, 8 * n, cudaMemcpyHostToDevice, m->s));
    xd = L.x.p;
    yd = L.b.p;
  }
  if (L.A->kind == 1) DG_TRY(elasticity_apply_f64(L.A.get(), xd, yd, m->s));
  else DG_TRY(lapmass_apply_j_f64(L.A.get(), L.jcoef(), L.jset(), xd, yd, m->s));
  if (!on_device) DG_CUDA(cudaMemcpyAsync(y, L.b.p, 8 * n, cudaMemcpyDeviceToHost, m->s));
  DG_CUDA(cudaStreamSynchronize(m->s));
  return DG_OK;
}

dg_status dg_damg_transfer_export(dg_damg* m, int level, int which, int64_t* nnz, uint32_t* ptr, uint32_t* col,
                                  double* val) {
  DG_CHECK(m && nnz && level >= 0 && size_t(level) + 1 < m->lv.size() && (which == 0 || which == 1), DG_EINVAL,
           "damg_transfer_export: bad arguments");
  const Level& L = m->lv[size_t(level)];
  const int64_t rows = which == 0 ? L.da->N : m->lv[size_t(level) + 1].da->N;
  const DBuf<uint32_t>& dp = which == 0 ? L.pptr : L.rptr;
  const DBuf<uint32_t>& dc = which == 0 ? L.pcol : L.rcol;
  const DBuf<double>& dv = which == 0 ? L.pval : L.rval;
  uint32_t total = 0;
  DG_CUDA(cudaMemcpy(&total, dp.p + rows, 4, cudaMemcpyDeviceToHost));
  *nnz = total;
  if (ptr) DG_CUDA(cudaMemcpy(ptr, dp.p, 4 * (rows + 1), cudaMemcpyDeviceToHost));
  if (col) DG_CUDA(cudaMemcpy(col, dc.p, 4 * size_t(total), cudaMemcpyDeviceToHost));
  if (val) DG_CUDA(cudaMemcpy(val, dv.p, 8 * size_t(total), cudaMemcpyDeviceToHost));
  return DG_OK;
}

dg_status dg_damg_level_coef(dg_damg* m, int level, double* coef) {
  DG_CHECK(m && coef && level >= 0 && size_t(level) < m->lv.size(), DG_EINVAL, "damg_level_coef: bad arguments");
  const Level& L = m->lv[size_t(level)];
  DG_CHECK(L.A && L.A->kind == 0, DG_EINVAL, "damg_level_coef: no Laplacian-mass operator set");
  const int64_t E = L.da->E;
  std::vector<double> soa(2 * E, 1.0);
  if (L.A->has_coef) DG_CUDA(cudaMemcpy(soa.data(), L.A->coef.p, 16 * E, cudaMemcpyDeviceToHost));
  for (int64_t e = 0; e < E; ++e) {
    coef[2 * e] = soa[e];
    coef[2 * e + 1] = soa[E + e];
  }
  return DG_OK;
}

dg_status dg_damg_coarse_solve(dg_damg* m, const double* b, double* x, void* stream) {
  DG_CHECK(m && b && x && !m->lv.empty(), DG_EINVAL, "damg_coarse_solve: bad arguments");
  DG_CHECK(m->lv.back().A, DG_EINVAL, "damg_coarse_solve: no operator set");
  const int64_t n = int64_t(m->cfg.dof) * m->lv.back().da->N;
  auto s = static_cast<cudaStream_t>(stream);
  dense_gemv<<<grid_for(n * 32, 256), 256, 0, s>>>(m->Ainv.p, n, m->d_crow_blk.p, m->d_cb_off.p, m->d_cb_n.p,
                                                   m->d_cb_aoff.p, b, x);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status dg_damg_vcycle(dg_damg* m, const double* b, double* x) {
  DG_CHECK(m && b && x, DG_EINVAL, "damg_vcycle: bad arguments");
  const int64_t n = int64_t(m->cfg.dof) * m->lv[0].da->N;
  DG_CUDA(cudaDeviceSynchronize());
  DG_CUDA(cudaMemcpyAsync(m->r.p, b, 8 * n, cudaMemcpyDeviceToDevice, m->s));
  DG_TRY(precond_body(m));
  DG_CUDA(cudaMemcpyAsync(x, m->z.p, 8 * n, cudaMemcpyDeviceToDevice, m->s));
  DG_CUDA(cudaStreamSynchronize(m->s));
  return DG_OK;
}

}  // extern "C"
