// Multi-right-hand-side operator Y = A X on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory): the scalar Laplacian + mass
// operator (JAC_TYPE2_ELEM_MULT_BLOCK, examples/src/backend/omgNeumann.C:468-488)
// applied to nrhs vectors at once, X and Y node-major [N][nrhs] in FP32.
//
// The contraction is the octet's assembled element matrix times its nodal
// block.  A parent octant with leaf children ("octet", octet.cuh) owns the
// 3 x 3 x 3 lattice of its children's vertices; on that lattice the sum of
// its present children's element operators is the 27 x 27 matrix
//
//   Klat[p][q] = K(d) * sum_c f1_c + M(d) * sum_c f2_c,
//
// the sums over the present children c whose box holds both lattice points,
// d = the number of axes on which p and q differ (|p_a - q_a| <= 1 on every
// axis, else the entry is 0), K(d) = {2/3, 0, -1/6, -1/6} and
// M(d) = {8, 4, 2, 1} / 27 the reference-cube Q1 stiffness and mass entries
// (the Walsh-basis operator of element.cuh written out), f1 = h/2 a_e and
// f2 = h^3/8 b_e the element's scale factors.  For a pair of octets and 64
// right-hand sides one tcgen05.mma chain (M = 128 rows = 2 octets x 64
// right-hand sides, N = 64 = the two octets' 32 lattice columns, K = 32
// lattice points in four steps of 8) computes D[(o, r)][(o', q)] =
// sum_p X_o[p][r] Klat_o'[p][q]; the blocks o = o' are the octets' lattice
// sums (the cross blocks are not read).
//
// Operands in shared memory, both K-major (the lattice index contiguous),
// no swizzle, 8-row x 16-byte core matrices:
//   A (TF32): the two octets' lattice values of X, entry (m = 64 o + r, k = p)
//     at (m / 8) * 1024 + (k / 4) * 128 + (m % 8) * 16 + (k % 4) * 4, copied
//     from the node rows of X by 4-byte cp.async (a warp's copies cover
//     8 right-hand sides x 4 lattice points: 32 distinct banks); the values of
//     hanging lattice points are filled with the mean of their corners (the
//     interpolation T of the hanging-node stencils, handleType2Stencils.C)
//     before the MMA, each thread for its own row m;
//   B (TF32): Klat_0 | Klat_1, entry (k = p, n = 32 o + q) at the same offsets
//     with n in place of m.
// (An MN-major A, which would take X's rows as they are, measured as a
// no-op for kind::tf32 on this hardware: the accumulator was left untouched.)
// The epilogue reads each thread's row of D (32 lattice columns of one octet
// and one right-hand side) with tcgen05.ld, folds the hanging points' sums
// onto their corners (T^T), stages the pair's 2 x 27 lattice rows in shared
// memory and adds them into Y with 16-byte global reductions (4 consecutive
// right-hand sides of one node per lane).
//
// Passes: 1 = TF32 products of the FP32 inputs; 3 = each input split into a
// TF32 high part and its remainder, D = A_hi B_hi + A_lo B_hi + A_hi B_lo
// (FP32-level accuracy).
//
// Pipeline per CTA (128 threads, persistent over pairs): the records of pair
// k + 2 and the X rows of pair k + 1 are copied by cp.async while the
// epilogue of pair k runs; one thread issues the MMAs of a pair and commits
// them to the stage's mbarrier.  Waits on the mbarrier are bounded by a clock
// deadline; past it the kernel records DG_ETIMEOUT, waits (bounded again)
// for the MMAs it issued, frees its tensor memory and returns.
#include <algorithm>
#include <cstring>

#include "dg_internal.h"
#include "octet.cuh"

namespace dg {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcRhs = 64;           // right-hand sides per pass over a pair
constexpr int kTcAbytes = 16384;     // A operand (one of hi / lo)
constexpr int kTcBbytes = 8192;      // B operand (one of hi / lo)
constexpr int kTcRec = kOctRec;      // u32 per octet record: 27 ids, none mask, meta, pad
constexpr int kTcCoef = 16;          // floats per octet: f1[8], f2[8]
constexpr int kTcTmemCols = 128;     // two stages x 64 accumulator columns

__device__ int g_tc_status;  // DG_ETIMEOUT when a bounded wait of this kernel has run out

struct TcMeta {  // one pair: records and coefficients of its two octets
  uint32_t rec[2][kTcRec];
  float coef[2][kTcCoef];
};

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void cp16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp4(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // start >> 4 [0,14), leading byte offset >> 4 [16,30), stride byte offset
  // >> 4 [32,46), version 1 [46,48), base offset 0, no swizzle [61,64)
  return uint64_t((addr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) |
         (uint64_t((sbo >> 4) & 0x3fffu) << 32) | (uint64_t(1) << 46);
}

// kind::tf32 instruction word: F32 accumulator, TF32 A and B, both K-major,
// N = 64, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(64 >> 3) << 17) |
                              (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)) : "memory");
}
// Bounded wait for phase `parity`: false once `limit` clock cycles have
// passed.  A non-blocking test first, then tries that suspend the thread in
// hardware (up to a 0.1 ms hint) until the phase completes, so the wait
// issues few instructions and a limit shorter than one try still ends it.
__device__ __forceinline__ bool bar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_try_suspend(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity), "r"(100000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (true) {
    if (bar_test(bar, parity)) return true;
    if (clock64() - t0 > limit) return false;
    if (bar_try_suspend(bar, parity)) return true;
  }
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Byte offset of entry (row, k) of a K-major operand (A: row = 64 o + r;
// B: row = 32 o + q; k = lattice point p).
__device__ __forceinline__ uint32_t kmaj(int row, int k) {
  return uint32_t((row >> 3) * 1024 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// One of the 343 nonzero lattice pairs of Klat: per axis the coordinate pair
// index in {(0,0),(0,1),(1,0),(1,1),(1,2),(2,1),(2,2)}.
struct KEntry {
  int p, q, d;
  uint32_t cmask;  // children whose box holds both points
};
__device__ __forceinline__ KEntry kentry(int e) {
  const int pa[7] = {0, 0, 1, 1, 1, 2, 2}, qa[7] = {0, 1, 0, 1, 2, 1, 2};
  KEntry k{0, 0, 0, 0xffu};
  int stride = 1;
  for (int a = 0; a < 3; ++a) {
    const int i = e % 7;
    e /= 7;
    k.p += pa[i] * stride;
    k.q += qa[i] * stride;
    k.d += pa[i] != qa[i];
    // child bit on axis a: 0 when both coordinates are <= 1, 1 when both >= 1
    uint32_t keep = 0;
    for (int c = 0; c < 8; ++c) {
      const bool hi = (c >> a) & 1;
      if (hi ? (pa[i] >= 1 && qa[i] >= 1) : (pa[i] <= 1 && qa[i] <= 1)) keep |= 1u << c;
    }
    k.cmask &= keep;
    stride *= 3;
  }
  return k;
}

template <int NP>
struct TcSmem {
  static constexpr int kStage = (NP == 3 ? 2 : 1) * (kTcAbytes + kTcBbytes);
  static constexpr int kMetaOff = 2 * kStage;
  static constexpr int kBarOff = kMetaOff + 3 * int(sizeof(TcMeta));
  static constexpr int kBytes = kBarOff + 64;
};

template <int NP>
__global__ void __launch_bounds__(kTcThreads) mrhs_tc_kernel(int64_t npairs, int ncb, const uint32_t* __restrict__ rec,
                                                             const float* __restrict__ coef, int R,
                                                             const float* __restrict__ X, float* __restrict__ Y,
                                                             long long limit) {
  extern __shared__ __align__(1024) unsigned char sm[];
  using L = TcSmem<NP>;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  TcMeta* meta = reinterpret_cast<TcMeta*>(sm + L::kMetaOff);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::kBarOff);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::kBarOff + 16);
  int* abort_flag = reinterpret_cast<int*>(sm + L::kBarOff + 20);
  const uint32_t sbase = su32(sm);
  auto A_hi = [&](int st) { return sbase + uint32_t(st * L::kStage); };
  auto B_hi = [&](int st) { return sbase + uint32_t(st * L::kStage + kTcAbytes); };
  auto A_lo = [&](int st) { return sbase + uint32_t(st * L::kStage + kTcAbytes + kTcBbytes); };
  auto B_lo = [&](int st) { return sbase + uint32_t(st * L::kStage + 2 * kTcAbytes + kTcBbytes); };

  const int64_t items = npairs * ncb;
  if (int64_t(blockIdx.x) * ((items + gridDim.x - 1) / gridDim.x) >= items) return;

  // operands start at zero: rows 27..31, the zero entries of Klat and the
  // rows of untouched lattice points are never written again
  for (int i = t; i < 2 * L::kStage / 16; i += kTcThreads)
    reinterpret_cast<uint4*>(sm)[i] = make_uint4(0u, 0u, 0u, 0u);
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    bar_init(&bar[0]);
    bar_init(&bar[1]);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // this thread's lattice pairs of Klat
  KEntry ke[3];
  int nke = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int e = t + i * kTcThreads;
    if (e < 343) {
      ke[i] = kentry(e);
      nke = i + 1;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // each CTA works a contiguous range of pairs (neighbours on the curve
  // share nodes, so their reductions meet in L2)
  const int64_t per = (items + gridDim.x - 1) / gridDim.x;
  const int64_t first = int64_t(blockIdx.x) * per, last = first + per < items ? first + per : items;
  auto item_of = [&](int64_t k) { return first + k < last ? first + k : items; };
  // records of local item k into meta slot k % 3
  auto issue_meta = [&](int64_t k) {
    const int64_t it = item_of(k);
    if (it < items && t < 24) {
      const int64_t pair = it / ncb;
      TcMeta& M = meta[k % 3];
      if (t < 16) {
        const int o = t >> 3, c = t & 7;
        cp16(su32(&M.rec[o][4 * c]), rec + (2 * pair + o) * kTcRec + 4 * c);
      } else {
        const int o = (t - 16) >> 2, c = (t - 16) & 3;
        cp16(su32(&M.coef[o][4 * c]), coef + (2 * pair + o) * kTcCoef + 4 * c);
      }
    }
    cp_commit();
  };
  // X rows of local item k into stage st, Klat of its octets into B
  auto gather = [&](int64_t k, int st) {
    const int64_t it = item_of(k);
    const int cb = int(it % ncb);
    const TcMeta& M = meta[k % 3];
    const int pl = lane & 3, rl = lane >> 2;
    for (int task = w; task < 128; task += 4) {  // (octet, group of 4 lattice points, group of 8 columns)
      const int o = task >> 6, p = ((task >> 3) & 7) * 4 + pl, r = (task & 7) * 8 + rl;
      if (p < 27) {
        const uint32_t id = M.rec[o][p];
        if (id != kNoNode) cp4(A_hi(st) + kmaj(64 * o + r, p), X + int64_t(id) * R + cb * kTcRhs + r);
      }
    }
    cp_commit();
    for (int i = 0; i < nke; ++i) {
      const KEntry& e = ke[i];
      const float kd = e.d == 0 ? 2.f / 3.f : e.d == 1 ? 0.f : -1.f / 6.f;
      const float md = e.d == 0 ? 8.f / 27.f : e.d == 1 ? 4.f / 27.f : e.d == 2 ? 2.f / 27.f : 1.f / 27.f;
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        float s1 = 0.f, s2 = 0.f;
        for (uint32_t m = e.cmask; m; m &= m - 1u) {
          const int c = __ffs(m) - 1;
          s1 += M.coef[o][c];
          s2 += M.coef[o][8 + c];
        }
        const float v = kd * s1 + md * s2;
        const uint32_t off = kmaj(32 * o + e.q, e.p);
        if (NP == 3) {
          const float hi = tf32_hi(v);
          asm volatile("st.shared.f32 [%0], %1;" ::"r"(B_hi(st) + off), "f"(hi) : "memory");
          asm volatile("st.shared.f32 [%0], %1;" ::"r"(B_lo(st) + off), "f"(v - hi) : "memory");
        } else {
          asm volatile("st.shared.f32 [%0], %1;" ::"r"(B_hi(st) + off), "f"(v) : "memory");
        }
      }
    }
  };
  // after the values have landed: each thread fills the hanging lattice
  // points of its row m = 64 o + r from their corners (and, for three
  // passes, splits its row into TF32 high parts and remainders)
  auto finish_rows = [&](int64_t k, int st) {
    const TcMeta& M = meta[k % 3];
    const int o = t >> 6;
    const uint32_t none = M.rec[o][27];
    auto ld = [&](uint32_t base, int p) {
      float v;
      asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(base + kmaj(t, p)));
      return v;
    };
    auto st1 = [&](uint32_t base, int p, float v) {
      asm volatile("st.shared.f32 [%0], %1;" ::"r"(base + kmaj(t, p)), "f"(v) : "memory");
    };
    const uint32_t ah = A_hi(st);
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      if (!((none >> p) & 1u)) continue;
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        st1(ah, p, 0.5f * (ld(ah, p - s0) + ld(ah, p + s0)));
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        st1(ah, p, 0.25f * ((ld(ah, p - s0 - s1) + ld(ah, p + s0 - s1)) + (ld(ah, p - s0 + s1) + ld(ah, p + s0 + s1))));
      }
    }
    if (NP == 3) {
#pragma unroll
      for (int p = 0; p < 27; ++p) {
        const float v = ld(ah, p), h = tf32_hi(v);
        st1(ah, p, h);
        st1(A_lo(st), p, v - h);
      }
    }
  };
  auto issue_mma = [&](int st) {
    if (t == 0) {
      tc_fence_after();
      const uint32_t d = tmem + uint32_t(st * 64);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const uint64_t ah = smem_desc(A_hi(st) + s * 256, 128, 1024);
        const uint64_t bh = smem_desc(B_hi(st) + s * 256, 128, 1024);
        tc_mma(d, ah, bh, s > 0 ? 1u : 0u);
        if (NP == 3) {
          tc_mma(d, smem_desc(A_lo(st) + s * 256, 128, 1024), bh, 1u);
          tc_mma(d, ah, smem_desc(B_lo(st) + s * 256, 128, 1024), 1u);
        }
      }
      tc_commit(&bar[st]);
    }
  };
  auto epilogue = [&](int64_t k, int st) {
    const int64_t it = item_of(k);
    const int cb = int(it % ncb);
    const TcMeta& M = meta[k % 3];
    const int o = w >> 1, r = (w & 1) * 32 + lane;
    float v[32];
    tc_fence_after();  // the chain's completion (seen on the mbarrier) before the tensor-memory read
    tc_ld32(tmem + (uint32_t(32 * w) << 16) + uint32_t(st * 64 + 32 * o), v);
    const uint32_t none = M.rec[o][27];
#pragma unroll
    for (int p = 0; p < 27; ++p) {
      if (oct_free(p) == 1) {
        const int s0 = oct_s0(p);
        const float h = ((none >> p) & 1u) ? v[p] * 0.5f : 0.f;
        v[p - s0] += h;
        v[p + s0] += h;
      } else if (oct_free(p) == 2) {
        const int s0 = oct_s0(p), s1 = oct_s1(p);
        const float h = ((none >> p) & 1u) ? v[p] * 0.25f : 0.f;
        v[p - s0 - s1] += h;
        v[p + s0 - s1] += h;
        v[p - s0 + s1] += h;
        v[p + s0 + s1] += h;
      }
    }
    // the lattice sums through the stage's A buffer (its MMA has completed),
    // then out as 16-byte reductions: 4 consecutive right-hand sides of one
    // node per lane
    tc_fence_before();
    const uint32_t sbuf = A_hi(st);
#pragma unroll
    for (int p = 0; p < 27; ++p)
      asm volatile("st.shared.f32 [%0], %1;" ::"r"(sbuf + uint32_t(((o * 27 + p) * kTcRhs + r) * 4)), "f"(v[p])
                   : "memory");
    __syncthreads();
    for (int j = t; j < 2 * 27 * (kTcRhs / 4); j += kTcThreads) {
      const int oo = j / (27 * (kTcRhs / 4)), rem = j % (27 * (kTcRhs / 4)), p = rem / (kTcRhs / 4),
                r4 = rem % (kTcRhs / 4);
      const uint32_t id = M.rec[oo][p];
      if (id == kNoNode) continue;
      float4 a;
      asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
                   : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w)
                   : "r"(sbuf + uint32_t(((oo * 27 + p) * kTcRhs + 4 * r4) * 4)));
      float* dst = Y + int64_t(id) * R + cb * kTcRhs + 4 * r4;
      asm volatile("red.global.add.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(dst), "f"(a.x), "f"(a.y), "f"(a.z), "f"(a.w)
                   : "memory");
    }
    tc_fence_before();
  };

  bool ok = true;
  int64_t pending = -1;  // local item whose MMA chain a timed-out wait left behind
  issue_meta(0);
  issue_meta(1);
  cp_wait<1>();
  __syncthreads();
  gather(0, 0);
  cp_wait<0>();
  __syncthreads();
  finish_rows(0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  issue_mma(0);
  for (int64_t k = 0; item_of(k) < items; ++k) {
    const int st = int(k & 1);
    const bool next = item_of(k + 1) < items;
    issue_meta(k + 2);
    if (next) {
      cp_wait<1>();
      __syncthreads();
      gather(k + 1, st ^ 1);
    }
    if (!bar_wait(&bar[st], uint32_t((k >> 1) & 1), limit)) atomicOr(abort_flag, 1);
    __syncthreads();
    if (*abort_flag) {
      ok = false;
      pending = k;
      break;
    }
    epilogue(k, st);
    if (!next) break;
    cp_wait<0>();
    __syncthreads();
    finish_rows(k + 1, st ^ 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    issue_mma(st ^ 1);
  }
  cp_wait<0>();
  if (!ok) {
    if (t == 0) atomicExch(&g_tc_status, int(DG_ETIMEOUT));
    // the chain of the item that timed out may still run: wait for its
    // commit once more before the tensor memory goes back, bounded by at
    // least about a second whatever limit the caller set
    const long long drain = limit > (1ll << 31) ? limit : (1ll << 31);
    bar_wait(&bar[pending & 1], uint32_t((pending >> 1) & 1), drain);
  }
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
  }
}

// Per octet: f1 = h/2 a_e and f2 = h^3/8 b_e of each present child, 0 for the others.
__global__ void tc_coefs(int64_t n, const uint32_t* __restrict__ ometa, const uint32_t* __restrict__ oelem,
                         const float* __restrict__ ca, const float* __restrict__ cb, float* __restrict__ out) {
  for (int64_t o = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; o <= n; o += int64_t(gridDim.x) * blockDim.x) {
    float* f = out + o * kTcCoef;
    const uint32_t m = o < n ? ometa[o] : 0u;
    const float h = __int_as_float(int(127 + 1 - int(ometa_lev(m))) << 23);
    const float g1 = h * 0.5f, g2 = h * h * h * 0.125f;
    const uint32_t cm = ometa_cmask(m);
    for (int c = 0; c < 8; ++c) {
      float f1 = 0.f, f2 = 0.f;
      if ((cm >> c) & 1u) {
        f1 = g1;
        f2 = g2;
        if (ca) {
          const uint32_t e = oelem[int64_t(c) * n + o];
          f1 *= ca[e];
          f2 *= cb[e];
        }
      }
      f[c] = f1;
      f[8 + c] = f2;
    }
  }
}

}  // namespace

dg_status mrhs_tc_apply(const dg_mat* A, const float* X, float* Y, int R, int passes, cudaStream_t s) {
  dg_da* da = A->da;
  OctetSet& O = da->octs;
  DG_CHECK(A->kind == 0, DG_EINVAL, "mat_mult_multi: scalar operator expected");
  DG_CHECK(R > 0 && R % kTcRhs == 0 && O.n > 0, DG_EINVAL,
           "mat_mult_multi: the tensor-memory form takes nrhs a multiple of 64 on a mesh with octets");
  DG_CHECK(passes == 1 || passes == 3, DG_EINVAL, "mat_mult_multi: passes must be 1 or 3");
  DG_CHECK((reinterpret_cast<uintptr_t>(X) & 15) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0, DG_EINVAL,
           "mat_mult_multi: X and Y must be 16-byte aligned");
  const unsigned pg = unsigned(std::min<int64_t>((O.n + 256) / 256, int64_t(sm_count()) * 8));
  if (!A->tc_coef.p) DG_TRY(A->tc_coef.alloc((O.n + 1) * kTcCoef));
  const float* ca = A->has_coef ? A->coef32.p : nullptr;
  const float* cb = A->has_coef ? A->coef32.p + da->E : nullptr;
  tc_coefs<<<pg, 256, 0, s>>>(O.n, O.meta.p, O.elem.p, ca, cb, A->tc_coef.p);
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaMemsetAsync(Y, 0, sizeof(float) * size_t(da->N) * R, s));
  const int64_t npairs = (O.n + 1) / 2;
  const int ncb = R / kTcRhs;
  const int64_t items = npairs * ncb;
  int per_sm = 0;
  if (passes == 3) {
    constexpr int bytes = TcSmem<3>::kBytes;
    static bool attr3 = false;
    if (!attr3) {
      DG_CUDA(cudaFuncSetAttribute(mrhs_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      DG_CUDA(cudaFuncSetAttribute(mrhs_tc_kernel<3>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)));
      attr3 = true;
    }
    per_sm = std::min(512 / kTcTmemCols, (227 << 10) / (bytes + 1024));
    const unsigned grid = unsigned(std::min<int64_t>(items, int64_t(sm_count()) * per_sm));
    mrhs_tc_kernel<3><<<grid, kTcThreads, bytes, s>>>(npairs, ncb, O.rec.p, A->tc_coef.p, R, X, Y,
                                                       wait_limit());
  } else {
    constexpr int bytes = TcSmem<1>::kBytes;
    static bool attr1 = false;
    if (!attr1) {
      DG_CUDA(cudaFuncSetAttribute(mrhs_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      DG_CUDA(cudaFuncSetAttribute(mrhs_tc_kernel<1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)));
      attr1 = true;
    }
    per_sm = std::min(512 / kTcTmemCols, (227 << 10) / (bytes + 1024));
    const unsigned grid = unsigned(std::min<int64_t>(items, int64_t(sm_count()) * per_sm));
    mrhs_tc_kernel<1><<<grid, kTcThreads, bytes, s>>>(npairs, ncb, O.rec.p, A->tc_coef.p, R, X, Y,
                                                       wait_limit());
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

dg_status mrhs_tc_take_status() {
  int v = 0;
  DG_CUDA(cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int)));
  if (v) {
    const int z = 0;
    DG_CUDA(cudaMemcpyToSymbol(g_tc_status, &z, sizeof(int)));
    DG_CHECK(false, DG_ETIMEOUT, "a bounded wait of the tensor-memory multi-RHS kernel ran out");
  }
  return DG_OK;
}

}  // namespace dg
