// Learned post-smoother: a per-node MLP 6 -> 64 -> 64 -> 1 with GELU
// activations, BF16 weights in the forward pass and FP32 accumulation, and
// its training kernels (forward + backward with block-level gradient
// reduction, Adam).  No reference counterpart: the reference smooths with
// damped Jacobi only (bin/options:187-194).
//
// Parameters are one packed FP32 vector (the master copy Adam updates):
//   W1[64][6] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
#include <cuda_bf16.h>

#include "dg_internal.h"

namespace dg {

namespace {

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Parameters as used by the forward pass: BF16-rounded (or exact FP32 when
// `exact` is set, for gradient checks), staged into shared memory.
__device__ __forceinline__ void load_params(const float* __restrict__ p, float* __restrict__ sp, bool exact) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    const float v = p[i];
    sp[i] = exact ? v : __bfloat162float(__float2bfloat16_rn(v));
  }
}

// y = w3 . gelu(W2 gelu(W1 f + b1) + b2) + b3 for one node.
__device__ __forceinline__ float mlp_eval(const float* __restrict__ sp, const float (&f)[kMlpIn]) {
  const float* W1 = sp + kOffW1;
  const float* b1 = sp + kOffB1;
  const float* W2 = sp + kOffW2;
  const float* b2 = sp + kOffB2;
  const float* w3 = sp + kOffW3;
  float a1[kMlpHidden];
#pragma unroll
  for (int k = 0; k < kMlpHidden; ++k) {
    float z = b1[k];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) z = fmaf(W1[k * kMlpIn + i], f[i], z);
    a1[k] = gelu(z);
  }
  float y = sp[kOffB3];
#pragma unroll 4
  for (int j = 0; j < kMlpHidden; ++j) {
    float z = b2[j];
#pragma unroll
    for (int k = 0; k < kMlpHidden; ++k) z = fmaf(W2[j * kMlpHidden + k], a1[k], z);
    y = fmaf(w3[j], gelu(z), y);
  }
  return y;
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ params, const float* __restrict__ F,
                                                          int64_t n, float* __restrict__ out, int exact) {
  __shared__ float sp[kMlpParams];
  load_params(params, sp, exact != 0);
  __syncthreads();
  for (int64_t i = gtid(); i < n; i += gstride()) {
    float f[kMlpIn];
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c) f[c] = F[i * kMlpIn + c];
    out[i] = mlp_eval(sp, f);
  }
}

// Forward + backward of the mean squared error over n nodes; one CTA owns
// kTrainNodes nodes and adds its gradient to grad[] with one atomic per
// parameter.  loss_acc accumulates sum (y - t)^2.
constexpr int kTrainNodes = 64;

__global__ void __launch_bounds__(kTrainNodes) mlp_train_kernel(const float* __restrict__ params,
                                                                const float* __restrict__ F,
                                                                const float* __restrict__ T, int64_t n, float inv_n,
                                                                float* __restrict__ grad, float* __restrict__ loss_acc,
                                                                int exact) {
  extern __shared__ float smem[];
  float* sp = smem;                                   // kMlpParams
  float* A1 = sp + kMlpParams;                        // [node][64] activations of layer 1
  float* G1 = A1 + kTrainNodes * (kMlpHidden + 1);    // gelu'(z1)
  float* D2 = G1 + kTrainNodes * (kMlpHidden + 1);    // gelu'(z2), then dL/dz2
  float* D1 = D2 + kTrainNodes * (kMlpHidden + 1);    // dL/dz1
  float* FS = D1 + kTrainNodes * (kMlpHidden + 1);    // features [node][6]
  float* gsh = FS + kTrainNodes * kMlpIn;             // block gradient of w3, b3
  constexpr int LD = kMlpHidden + 1;
  load_params(params, sp, exact != 0);
  for (int i = threadIdx.x; i < kMlpHidden + 1; i += blockDim.x) gsh[i] = 0.f;
  __syncthreads();
  const float* W1 = sp + kOffW1;
  const float* b1 = sp + kOffB1;
  const float* W2 = sp + kOffW2;
  const float* b2 = sp + kOffB2;
  const float* w3 = sp + kOffW3;
  const int t = threadIdx.x;
  const int64_t node = int64_t(blockIdx.x) * kTrainNodes + t;
  const bool valid = node < n;
  float f[kMlpIn];
#pragma unroll
  for (int c = 0; c < kMlpIn; ++c) {
    f[c] = valid ? F[node * kMlpIn + c] : 0.f;
    FS[t * kMlpIn + c] = f[c];
  }
  // forward
  for (int k = 0; k < kMlpHidden; ++k) {
    float z = b1[k];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) z = fmaf(W1[k * kMlpIn + i], f[i], z);
    A1[t * LD + k] = gelu(z);
    G1[t * LD + k] = gelu_grad(z);
  }
  float y = sp[kOffB3];
  for (int j = 0; j < kMlpHidden; ++j) {
    float z = b2[j];
    for (int k = 0; k < kMlpHidden; ++k) z = fmaf(W2[j * kMlpHidden + k], A1[t * LD + k], z);
    const float a2 = gelu(z);
    D2[t * LD + j] = gelu_grad(z);
    y = fmaf(w3[j], a2, y);
    // w3 gradient needs dy, known only after y: keep a2 in D1 for now
    D1[t * LD + j] = a2;
  }
  const float diff = valid ? (y - T[node]) : 0.f;
  const float dy = 2.f * diff * inv_n;
  if (valid) atomicAdd(loss_acc, diff * diff);
  // output layer: dw3_j = dy a2_j, db3 = dy; dz2_j = dy w3_j gelu'(z2_j)
  for (int j = 0; j < kMlpHidden; ++j) {
    atomicAdd(gsh + j, dy * D1[t * LD + j]);
    D2[t * LD + j] = dy * w3[j] * D2[t * LD + j];
  }
  atomicAdd(gsh + kMlpHidden, dy);
  // dz1_k = gelu'(z1_k) sum_j W2[j][k] dz2_j
  for (int k = 0; k < kMlpHidden; ++k) {
    float s = 0.f;
    for (int j = 0; j < kMlpHidden; ++j) s = fmaf(W2[j * kMlpHidden + k], D2[t * LD + j], s);
    D1[t * LD + k] = s * G1[t * LD + k];
  }
  __syncthreads();
  // block reductions over the nodes of this CTA
  for (int e = t; e < kMlpHidden * kMlpHidden; e += blockDim.x) {  // dW2[j][k] = sum_n dz2_j a1_k
    const int j = e / kMlpHidden, k = e % kMlpHidden;
    float s = 0.f;
    for (int q = 0; q < kTrainNodes; ++q) s = fmaf(D2[q * LD + j], A1[q * LD + k], s);
    atomicAdd(grad + kOffW2 + e, s);
  }
  for (int j = t; j < kMlpHidden; j += blockDim.x) {
    float s2 = 0.f, s1 = 0.f;
    for (int q = 0; q < kTrainNodes; ++q) {
      s2 += D2[q * LD + j];
      s1 += D1[q * LD + j];
    }
    atomicAdd(grad + kOffB2 + j, s2);
    atomicAdd(grad + kOffB1 + j, s1);
    atomicAdd(grad + kOffW3 + j, gsh[j]);
  }
  for (int e = t; e < kMlpHidden * kMlpIn; e += blockDim.x) {  // dW1[k][i] = sum_n dz1_k f_i
    const int k = e / kMlpIn, i = e % kMlpIn;
    float s = 0.f;
    for (int q = 0; q < kTrainNodes; ++q) s = fmaf(D1[q * LD + k], FS[q * kMlpIn + i], s);
    atomicAdd(grad + kOffW1 + e, s);
  }
  if (t == 0) atomicAdd(grad + kOffB3, gsh[kMlpHidden]);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

// ------------------------------------------------------------- smoothing --
// Per-node features of a residual r on one level:
//   f0 = r_i / s,                 s = RMS of r over the level
//   f1 = log2(d_i) - mean log2 d  (d = operator diagonal)
//   f2 = level / (levels - 1)
//   f3 = share of this node's element references that come from hanging vertices
//   f4 = mean residual over the elements around the node / s
//   f5 = max |residual| over the elements around the node / s
template <class R>
__device__ __forceinline__ void node_features(int64_t i, const R* __restrict__ r, float inv_s,
                                              const float* __restrict__ dinv, float dlogbar, float level_feat,
                                              const float* __restrict__ hang, const float* __restrict__ inv_refs,
                                              const float* __restrict__ nsum, const float* __restrict__ nmax,
                                              float (&f)[kMlpIn]) {
  f[0] = float(r[i]) * inv_s;
  f[1] = -log2f(dinv[i]) - dlogbar;
  f[2] = level_feat;
  f[3] = hang[i];
  f[4] = nsum[i] * 0.125f * inv_refs[i] * inv_s;
  f[5] = nmax[i] * inv_s;
}

// Element pass: per node, the sum over incident elements of the element's
// node-residual sum, and the max |r| over them.
template <class R>
__global__ void neighbour_stats_kernel(const uint32_t* __restrict__ nl, int64_t E, const R* __restrict__ r,
                                       float* __restrict__ nsum, float* __restrict__ nmax) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    uint32_t id[8];
    float s = 0.f, m = 0.f;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      id[v] = nl[int64_t(v) * E + e];
      const float rv = float(r[id[v]]);
      s += rv;
      m = fmaxf(m, fabsf(rv));
    }
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      atomicAdd(nsum + id[v], s);
      atomicMax(reinterpret_cast<int*>(nmax) + id[v], __float_as_int(m));  // m >= 0
    }
  }
}

// Element pass: element references per node and how many come from hanging vertices.
__global__ void node_refs_kernel(const uint32_t* __restrict__ nl, const uint32_t* __restrict__ meta, int64_t E,
                                 float* __restrict__ refs, float* __restrict__ hang) {
  for (int64_t e = gtid(); e < E; e += gstride()) {
    const uint32_t mask = meta_mask(meta[e]);
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const uint32_t id = nl[int64_t(v) * E + e];
      atomicAdd(refs + id, 1.f);
      if ((mask >> v) & 1u) atomicAdd(hang + id, 1.f);
    }
  }
}
__global__ void node_refs_finish(float* __restrict__ refs, float* __restrict__ hang, const float* __restrict__ dinv,
                                 int64_t N, float* __restrict__ dlog_sum) {
  float acc = 0.f;
  for (int64_t i = gtid(); i < N; i += gstride()) {
    const float c = refs[i];
    hang[i] = c > 0.f ? hang[i] / c : 0.f;
    refs[i] = c > 0.f ? 1.f / c : 0.f;  // becomes 1 / references
    acc += -log2f(dinv[i]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(dlog_sum, acc);
}

template <class R>
__global__ void sq_sum_kernel(const R* __restrict__ r, int64_t n, float* __restrict__ out) {
  float acc = 0.f;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    const float v = float(r[i]);
    acc = fmaf(v, v, acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Features + MLP + update in one pass, x_i += y_i s / d_i, on the tensor
// cores: each warp evaluates the MLP for 16 nodes at a time with
// mma.sync.m16n8k16 (BF16 inputs, FP32 accumulation) and the tanh form of
// GELU.  Layer 1 is one 16x16 (features padded with zeros) by 16x64
// product, layer 2 a 16x64 by 64x64 one; the accumulator fragments of a layer
// are, lane by lane, the input fragments of the next, so activations never
// leave registers.  Weights are BF16 in shared memory with padded rows (no
// bank conflicts on the B-fragment loads); biases and w3 stay FP32.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// GELU in the tanh form of Hendrycks and Gimpel (2016),
// 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), with the hardware tanh
// approximation: within about 1e-3 of the erf form the network was trained
// with, and a few instructions instead of an erf evaluation per unit.
__device__ __forceinline__ float gelu_fast(float z) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return 0.5f * z * (1.f + t);
}
constexpr int kW1Ld = 24;  // BF16 row stride of W1 (16 padded inputs + 8)
constexpr int kW2Ld = 72;  // BF16 row stride of W2 (64 + 8)

// Feature pair (2 q, 2 q + 1) of node i; pairs 0..2 are the 6 features, 3 is zero padding.
template <class R>
__device__ __forceinline__ float2 feature_pair(int q, int64_t i, int64_t n, const R* __restrict__ r, float inv_s,
                                               const float* __restrict__ dinv, float dlogbar, float level_feat,
                                               const float* __restrict__ hang, const float* __restrict__ inv_refs,
                                               const float* __restrict__ nsum, const float* __restrict__ nmax) {
  if (i >= n || q == 3) return make_float2(0.f, 0.f);
  if (q == 0) return make_float2(float(r[i]) * inv_s, -log2f(dinv[i]) - dlogbar);
  if (q == 1) return make_float2(level_feat, hang[i]);
  return make_float2(nsum[i] * 0.125f * inv_refs[i] * inv_s, nmax[i] * inv_s);
}

__global__ void __launch_bounds__(128) mlp_smooth_tc_kernel(
    const float* __restrict__ params, const float* __restrict__ r, int64_t n, const float* __restrict__ s2,
    const float* __restrict__ dinv, float dlogbar, float level_feat, const float* __restrict__ hang,
    const float* __restrict__ inv_refs, const float* __restrict__ nsum, const float* __restrict__ nmax,
    float* __restrict__ x) {
  __shared__ __align__(16) __nv_bfloat16 sW1[kMlpHidden * kW1Ld];
  __shared__ __align__(16) __nv_bfloat16 sW2[kMlpHidden * kW2Ld];
  __shared__ float sb1[kMlpHidden], sb2[kMlpHidden], sw3[kMlpHidden];
  for (int i = threadIdx.x; i < kMlpHidden * kW1Ld; i += blockDim.x) {
    const int row = i / kW1Ld, col = i % kW1Ld;
    sW1[i] = __float2bfloat16_rn(col < kMlpIn ? params[kOffW1 + row * kMlpIn + col] : 0.f);
  }
  for (int i = threadIdx.x; i < kMlpHidden * kW2Ld; i += blockDim.x) {
    const int row = i / kW2Ld, col = i % kW2Ld;
    sW2[i] = __float2bfloat16_rn(col < kMlpHidden ? params[kOffW2 + row * kMlpHidden + col] : 0.f);
  }
  for (int i = threadIdx.x; i < kMlpHidden; i += blockDim.x) {
    sb1[i] = __bfloat162float(__float2bfloat16_rn(params[kOffB1 + i]));
    sb2[i] = __bfloat162float(__float2bfloat16_rn(params[kOffB2 + i]));
    sw3[i] = __bfloat162float(__float2bfloat16_rn(params[kOffW3 + i]));
  }
  __syncthreads();
  const float b3 = __bfloat162float(__float2bfloat16_rn(params[kOffB3]));
  const float ss = *s2;
  if (!(ss > 0.f)) return;
  const float s = sqrtf(ss / float(n)), inv_s = 1.f / s;
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
  const uint32_t* W1w = reinterpret_cast<const uint32_t*>(sW1);
  const uint32_t* W2w = reinterpret_cast<const uint32_t*>(sW2);
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t base = (blockIdx.x * int64_t(blockDim.x >> 5) + (threadIdx.x >> 5)) * 16; base < n;
       base += warps * 16) {
    const int64_t i0 = base + g, i1 = base + g + 8;
    // layer 1 input fragment: rows g, g + 8 (nodes), columns 2 tq, 2 tq + 1 (features)
    const float2 p0 = feature_pair(tq, i0, n, r, inv_s, dinv, dlogbar, level_feat, hang, inv_refs, nsum, nmax);
    const float2 p1 = feature_pair(tq, i1, n, r, inv_s, dinv, dlogbar, level_feat, hang, inv_refs, nsum, nmax);
    const uint32_t a1[4] = {pack_bf16(p0.x, p0.y), pack_bf16(p1.x, p1.y), 0u, 0u};
    uint32_t a2[4][4];  // layer 2 input fragments, one per 16-wide k-tile
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      const int row = 8 * j + g;
      mma_bf16(d, a1, W1w[(row * kW1Ld + 2 * tq) / 2], W1w[(row * kW1Ld + 2 * tq + 8) / 2]);
      const int c0 = 8 * j + 2 * tq;
      const uint32_t lo = pack_bf16(gelu_fast(d[0] + sb1[c0]), gelu_fast(d[1] + sb1[c0 + 1]));
      const uint32_t hi = pack_bf16(gelu_fast(d[2] + sb1[c0]), gelu_fast(d[3] + sb1[c0 + 1]));
      a2[j >> 1][(j & 1) * 2] = lo;
      a2[j >> 1][(j & 1) * 2 + 1] = hi;
    }
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      const int row = 8 * j + g;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(d, a2[kk], W2w[(row * kW2Ld + 16 * kk + 2 * tq) / 2], W2w[(row * kW2Ld + 16 * kk + 8 + 2 * tq) / 2]);
      const int c0 = 8 * j + 2 * tq;
      y0 = fmaf(sw3[c0], gelu_fast(d[0] + sb2[c0]), fmaf(sw3[c0 + 1], gelu_fast(d[1] + sb2[c0 + 1]), y0));
      y1 = fmaf(sw3[c0], gelu_fast(d[2] + sb2[c0]), fmaf(sw3[c0 + 1], gelu_fast(d[3] + sb2[c0 + 1]), y1));
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    if (tq == 0) {
      if (i0 < n) x[i0] += (y0 + b3) * s * dinv[i0];
      if (i1 < n) x[i1] += (y1 + b3) * s * dinv[i1];
    }
  }
}

template <class R>
__global__ void features_kernel(const R* __restrict__ r, int64_t n, const float* __restrict__ s2,
                                const float* __restrict__ dinv, float dlogbar, float level_feat,
                                const float* __restrict__ hang, const float* __restrict__ inv_refs,
                                const float* __restrict__ nsum, const float* __restrict__ nmax, float* __restrict__ F,
                                float* __restrict__ scale_out) {
  const float ss = *s2;
  const float s = ss > 0.f ? sqrtf(ss / float(n)) : 1.f, inv_s = 1.f / s;
  if (gtid() == 0 && scale_out) *scale_out = s;
  for (int64_t i = gtid(); i < n; i += gstride()) {
    float f[kMlpIn];
    node_features(i, r, inv_s, dinv, dlogbar, level_feat, hang, inv_refs, nsum, nmax, f);
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c) F[i * kMlpIn + c] = f[c];
  }
}

}  // namespace

dg_status smoother_node_data(const dg_da* da, const float* dinv32, float* refs, float* hang, float* dlogbar,
                             cudaStream_t s) {
  DG_CUDA(cudaMemsetAsync(refs, 0, 4 * da->N, s));
  DG_CUDA(cudaMemsetAsync(hang, 0, 4 * da->N, s));
  node_refs_kernel<<<grid_for(da->E, 256), 256, 0, s>>>(da->nl.p, da->meta.p, da->E, refs, hang);
  DBuf<float> acc;
  DG_TRY(acc.alloc(1));
  DG_CUDA(cudaMemsetAsync(acc.p, 0, 4, s));
  node_refs_finish<<<grid_for(da->N, 256), 256, 0, s>>>(refs, hang, dinv32, da->N, acc.p);
  float h = 0.f;
  DG_CUDA(cudaMemcpyAsync(&h, acc.p, 4, cudaMemcpyDeviceToHost, s));
  DG_CUDA(cudaStreamSynchronize(s));
  *dlogbar = h / float(da->N > 0 ? da->N : 1);
  return DG_OK;
}

template <class R>
static dg_status residual_stats(const dg_da* da, const R* r, float* s2, float* nsum, float* nmax, cudaStream_t s) {
  DG_CUDA(cudaMemsetAsync(s2, 0, 4, s));
  DG_CUDA(cudaMemsetAsync(nsum, 0, 4 * da->N, s));
  DG_CUDA(cudaMemsetAsync(nmax, 0, 4 * da->N, s));
  sq_sum_kernel<R><<<grid_for(da->N, 256, 4), 256, 0, s>>>(r, da->N, s2);
  neighbour_stats_kernel<R><<<grid_for(da->E, 256), 256, 0, s>>>(da->nl.p, da->E, r, nsum, nmax);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status mlp_smooth_step(const float* params, const dg_da* da, const float* r, float* s2, const float* dinv32,
                          float dlogbar, float level_feat, const float* hang, const float* inv_refs, float* nsum,
                          float* nmax, float* x, cudaStream_t s) {
  DG_TRY(residual_stats<float>(da, r, s2, nsum, nmax, s));
  mlp_smooth_tc_kernel<<<grid_for((da->N + 3) / 4, 128, 8), 128, 0, s>>>(params, r, da->N, s2, dinv32, dlogbar,
                                                                         level_feat, hang, inv_refs, nsum, nmax, x);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status mlp_features_f64(const dg_da* da, const double* r, float* s2, const float* dinv32, float dlogbar,
                           float level_feat, const float* hang, const float* inv_refs, float* nsum, float* nmax,
                           float* F, float* scale_out, cudaStream_t s) {
  DG_TRY(residual_stats<double>(da, r, s2, nsum, nmax, s));
  features_kernel<double><<<grid_for(da->N, 256), 256, 0, s>>>(r, da->N, s2, dinv32, dlogbar, level_feat, hang,
                                                                inv_refs, nsum, nmax, F, scale_out);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

size_t mlp_train_smem_bytes() {
  return sizeof(float) * (kMlpParams + 4 * kTrainNodes * (kMlpHidden + 1) + kTrainNodes * kMlpIn + kMlpHidden + 1);
}

dg_status mlp_forward(const float* params, const float* F, int64_t n, float* out, bool exact, cudaStream_t s) {
  if (n <= 0) return DG_OK;
  mlp_forward_kernel<<<grid_for(n, 128, 8), 128, 0, s>>>(params, F, n, out, exact ? 1 : 0);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status mlp_gradient(const float* params, const float* F, const float* T, int64_t n, float* grad, float* loss_acc,
                       bool exact, cudaStream_t s) {
  if (n <= 0) return DG_OK;
  static bool attr = false;
  const size_t sm = mlp_train_smem_bytes();
  if (!attr) {
    DG_CUDA(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    attr = true;
  }
  const unsigned blocks = unsigned((n + kTrainNodes - 1) / kTrainNodes);
  mlp_train_kernel<<<blocks, kTrainNodes, sm, s>>>(params, F, T, n, 1.0f / float(n), grad, loss_acc, exact ? 1 : 0);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status mlp_adam(float* p, const float* g, float* m1, float* m2, int step, float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, s>>>(p, g, m1, m2, kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg

// ------------------------------------------------------------------ C ABI --
using namespace dg;

extern "C" {

int dg_mlp_param_count(void) { return kMlpParams; }

dg_status dg_mlp_create(const float* params, dg_mlp** out) {
  DG_CHECK(out, DG_EINVAL, "mlp_create: null output");
  auto* m = new dg_mlp();
  dg_status st = m->params.alloc(kMlpParams);
  if (!st) st = m->grad.alloc(kMlpParams);
  if (!st) st = m->m1.alloc(kMlpParams);
  if (!st) st = m->m2.alloc(kMlpParams);
  if (!st) st = m->loss.alloc(1);
  if (st) {
    delete m;
    return st;
  }
  cudaMemset(m->m1.p, 0, 4 * kMlpParams);
  cudaMemset(m->m2.p, 0, 4 * kMlpParams);
  if (params) {
    if (cudaMemcpy(m->params.p, params, 4 * kMlpParams, cudaMemcpyHostToDevice) != cudaSuccess) {
      delete m;
      set_error(__FILE__, __LINE__, "mlp_create: parameter upload failed");
      return DG_ECUDA;
    }
  } else {
    cudaMemset(m->params.p, 0, 4 * kMlpParams);
  }
  *out = m;
  return DG_OK;
}

dg_status dg_mlp_get_params(const dg_mlp* m, float* host) {
  DG_CHECK(m && host, DG_EINVAL, "mlp_get_params: bad arguments");
  DG_CUDA(cudaMemcpy(host, m->params.p, 4 * kMlpParams, cudaMemcpyDeviceToHost));
  return DG_OK;
}

dg_status dg_mlp_set_params(dg_mlp* m, const float* host) {
  DG_CHECK(m && host, DG_EINVAL, "mlp_set_params: bad arguments");
  DG_CUDA(cudaMemcpy(m->params.p, host, 4 * kMlpParams, cudaMemcpyHostToDevice));
  m->step = 0;
  DG_CUDA(cudaMemset(m->m1.p, 0, 4 * kMlpParams));
  DG_CUDA(cudaMemset(m->m2.p, 0, 4 * kMlpParams));
  return DG_OK;
}

dg_status dg_mlp_forward(dg_mlp* m, const float* F, int64_t n, float* out, int exact_fp32, void* stream) {
  DG_CHECK(m && n >= 0 && (n == 0 || (F && out)), DG_EINVAL, "mlp_forward: bad arguments");
  return mlp_forward(m->params.p, F, n, out, exact_fp32 != 0, reinterpret_cast<cudaStream_t>(stream));
}

dg_status dg_mlp_gradient(dg_mlp* m, const float* F, const float* T, int64_t n, int exact_fp32, float* grad_host,
                          double* loss_host) {
  DG_CHECK(m && F && T && n > 0, DG_EINVAL, "mlp_gradient: bad arguments");
  DG_CUDA(cudaDeviceSynchronize());
  DG_CUDA(cudaMemset(m->grad.p, 0, 4 * kMlpParams));
  DG_CUDA(cudaMemset(m->loss.p, 0, 4));
  DG_TRY(mlp_gradient(m->params.p, F, T, n, m->grad.p, m->loss.p, exact_fp32 != 0, nullptr));
  if (grad_host) DG_CUDA(cudaMemcpy(grad_host, m->grad.p, 4 * kMlpParams, cudaMemcpyDeviceToHost));
  if (loss_host) {
    float l = 0;
    DG_CUDA(cudaMemcpy(&l, m->loss.p, 4, cudaMemcpyDeviceToHost));
    *loss_host = double(l) / double(n);
  }
  return DG_OK;
}

dg_status dg_mlp_train_step(dg_mlp* m, const float* F, const float* T, int64_t n, float lr, double* loss_host) {
  DG_CHECK(m && F && T && n > 0 && lr > 0, DG_EINVAL, "mlp_train_step: bad arguments");
  DG_TRY(dg_mlp_gradient(m, F, T, n, 0, nullptr, loss_host));
  m->step += 1;
  DG_TRY(mlp_adam(m->params.p, m->grad.p, m->m1.p, m->m2.p, m->step, lr, nullptr));
  DG_CUDA(cudaDeviceSynchronize());
  return DG_OK;
}

void dg_mlp_destroy(dg_mlp* m) { delete m; }

}  // extern "C"
