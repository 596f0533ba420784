// Device-side element operator in the Hadamard (modal) basis.  See the
// block table in tpo_internal.h.  All loops are over compile-time constants
// so the 24 nodal values stay in registers.
#pragma once

#include "tpo_internal.h"

namespace tpo {

// forward butterfly: nodal (lexicographic corner) -> modal, in place
template <typename T>
__device__ __forceinline__ void modal_forward(T (&v)[8][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int s = 1; s < 8; s <<= 1) {
#pragma unroll
      for (int l = 0; l < 8; ++l) {
        if (!(l & s)) {
          const T a = v[l][c], b = v[l | s][c];
          v[l][c] = a + b;
          v[l | s][c] = b - a;
        }
      }
    }
  }
}

// transpose butterfly: modal -> nodal, in place
template <typename T>
__device__ __forceinline__ void modal_backward(T (&v)[8][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int s = 1; s < 8; s <<= 1) {
#pragma unroll
      for (int l = 0; l < 8; ++l) {
        if (!(l & s)) {
          const T S = v[l][c], D = v[l | s][c];
          v[l][c] = S - D;
          v[l | s][c] = S + D;
        }
      }
    }
  }
}

template <typename T>
__device__ __forceinline__ void blk2(const T (&u)[8][3], T (&o)[8][3], int qa,
                                     int ca, int qb, int cb, const T *k) {
  const T a = u[qa][ca], b = u[qb][cb];
  o[qa][ca] = k[0] * a + k[1] * b;
  o[qb][cb] = k[2] * a + k[3] * b;
}

template <typename T>
__device__ __forceinline__ void blk3(const T (&u)[8][3], T (&o)[8][3], int qa,
                                     int ca, int qb, int cb, int qc, int cc,
                                     const T *k) {
  const T a = u[qa][ca], b = u[qb][cb], d = u[qc][cc];
  o[qa][ca] = k[0] * a + k[1] * b + k[2] * d;
  o[qb][cb] = k[3] * a + k[4] * b + k[5] * d;
  o[qc][cc] = k[6] * a + k[7] * b + k[8] * d;
}

// o = Kh u (modal), o[0][*] = 0 (rigid translations)
template <typename T>
__device__ __forceinline__ void modal_couple(const T (&u)[8][3], T (&o)[8][3],
                                             const Kh<T> &kh) {
  o[0][0] = o[0][1] = o[0][2] = T(0);
  blk3(u, o, 1, 0, 2, 1, 4, 2, kh.v + 0);
  blk2(u, o, 1, 1, 2, 0, kh.v + 9);
  blk2(u, o, 1, 2, 4, 0, kh.v + 13);
  blk2(u, o, 2, 2, 4, 1, kh.v + 17);
  blk2(u, o, 3, 0, 6, 2, kh.v + 21);
  blk2(u, o, 3, 1, 5, 2, kh.v + 25);
  blk2(u, o, 6, 1, 5, 0, kh.v + 29);
  blk3(u, o, 3, 2, 6, 0, 5, 1, kh.v + 33);
  o[7][0] = kh.v[42] * u[7][0];
  o[7][1] = kh.v[43] * u[7][1];
  o[7][2] = kh.v[44] * u[7][2];
}

// v <- Ee * K0 v for one element (nodal, lexicographic corners)
template <typename T>
__device__ __forceinline__ void element_apply(T (&v)[8][3], T Ee,
                                              const Kh<T> &kh) {
  modal_forward(v);
#pragma unroll
  for (int q = 1; q < 8; ++q) {
    v[q][0] *= Ee;
    v[q][1] *= Ee;
    v[q][2] *= Ee;
  }
  T o[8][3];
  modal_couple(v, o, kh);
  modal_backward(o);
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    v[l][0] = o[l][0];
    v[l][1] = o[l][1];
    v[l][2] = o[l][2];
  }
}

// u^T K0 u for one element (nodal input, destroyed)
template <typename T>
__device__ __forceinline__ T element_energy(T (&v)[8][3], const Kh<T> &kh) {
  modal_forward(v);
  T o[8][3];
  modal_couple(v, o, kh);
  T s = T(0);
#pragma unroll
  for (int q = 1; q < 8; ++q) s += v[q][0] * o[q][0] + v[q][1] * o[q][1] + v[q][2] * o[q][2];
  return s;
}

}  // namespace tpo
