// Element arithmetic shared by the operator kernels: the Walsh-basis form
// of the Q1 Laplacian + mass element operator (see matvec.cu's header for
// the derivation).
#pragma once

#include "dg_internal.h"

namespace dg {

// h = 2^-(lev-1) for embedded level lev (omgNeumann.C:470-471).
template <class T>
__device__ __forceinline__ T elem_h(uint32_t lev) {
  return T(__longlong_as_double(int64_t(1023 + 1 - int(lev)) << 52));
}

// In-place 8-point Walsh-Hadamard transform over the vertex bits x=1, y=2, z=4.
template <class T>
__device__ __forceinline__ void wht8(T (&u)[8]) {
#pragma unroll
  for (int B = 1; B < 8; B <<= 1)
#pragma unroll
    for (int v = 0; v < 8; ++v)
      if (!(v & B)) {
        const T a = u[v], b = u[v | B];
        u[v] = a + b;
        u[v | B] = a - b;
      }
}

// u <- (f1 K + f2 M) u on the reference cube, K = K1(x)M1(x)M1 + M1(x)K1(x)M1
// + M1(x)M1(x)K1 and M = M1(x)M1(x)M1.  In the Walsh basis M1 -> diag(1, 1/3)
// and K1 -> diag(0, 1), so a component with n (1,-1) factors is scaled by
// f2 3^-n + f1 n 3^(1-n); the 1/8 of the inverse transform is folded in.
template <class T>
__device__ __forceinline__ void lapmass_ref(T (&u)[8], T f1, T f2) {
  wht8(u);
  const T l0 = f2 * T(0.125);
  const T l1 = (f2 * T(1.0 / 3.0) + f1) * T(0.125);
  const T l2 = (f2 * T(1.0 / 9.0) + f1 * T(2.0 / 3.0)) * T(0.125);
  const T l3 = (f2 * T(1.0 / 27.0) + f1 * T(1.0 / 3.0)) * T(0.125);
  u[0] *= l0;
  u[1] *= l1;
  u[2] *= l1;
  u[4] *= l1;
  u[3] *= l2;
  u[5] *= l2;
  u[6] *= l2;
  u[7] *= l3;
  wht8(u);
}

// r = (f1 K + f2 M) u, u unchanged.
template <class T>
__device__ __forceinline__ void lapmass_ref_to(const T (&u)[8], T f1, T f2, T (&r)[8]) {
#pragma unroll
  for (int v = 0; v < 8; ++v) r[v] = u[v];
  lapmass_ref(r, f1, f2);
}

}  // namespace dg
