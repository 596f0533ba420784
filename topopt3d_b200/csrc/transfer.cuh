// Grid-transfer and dense-solve device helpers shared by the per-level
// kernels (kernels_mg.cu) and the persistent coarse cycle (kernels_coarse.cu).
//
// Prolongation weights (Interpolation.cpp:123-169, row-normalised at
// :330-347): coarse node c sits on fine index 2c; the 1-D weight of c for
// fine f is 1 (f = 2c) or 1/2 (|f - 2c| = 1), normalised by the row sum,
// which is 1 except for an odd last fine node with one coarse neighbour
// (weight 1).  The 3-D weight is the product of the 1-D ones.
//
// The helpers are branch-free over their fixed 27 (restriction) or 8
// (prolongation) taps: invalid taps get weight 0 at a clamped, in-bounds
// index, so all loads can be issued together instead of one dependent load
// after another.
#pragma once

#include <cstdint>

namespace tpo {

__device__ __forceinline__ double pw1t(int f, int c, int Nf) {
  const int d = f - 2 * c;
  if (d < -1 || d > 1) return 0.0;
  if (d == 0) return 1.0;
  return (f + 1 <= Nf - 1) ? 0.5 : 1.0;
}

// sum over the fine nodes f around coarse node (ix,iy,iz) of P(f,I) r_f
template <typename T>
__device__ __forceinline__ void restrict_node(int fx, int fy, int fz, int ix,
                                              int iy, int iz,
                                              const T *__restrict__ rf, T s[3]) {
  int gxs[3], gys[3], gzs[3];
  double wx[3], wy[3], wz[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int gx = 2 * ix + a - 1, gy = 2 * iy + a - 1, gz = 2 * iz + a - 1;
    wx[a] = (gx >= 0 && gx < fx) ? pw1t(gx, ix, fx) : 0.0;
    wy[a] = (gy >= 0 && gy < fy) ? pw1t(gy, iy, fy) : 0.0;
    wz[a] = (gz >= 0 && gz < fz) ? pw1t(gz, iz, fz) : 0.0;
    gxs[a] = min(max(gx, 0), fx - 1);
    gys[a] = min(max(gy, 0), fy - 1);
    gzs[a] = min(max(gz, 0), fz - 1);
  }
  T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const T w = static_cast<T>(wx[a] * wy[b] * wz[c]);
        const int64_t f = ((int64_t)gzs[c] * fy + gys[b]) * fx + gxs[a];
        s0 += w * rf[3 * f];
        s1 += w * rf[3 * f + 1];
        s2 += w * rf[3 * f + 2];
      }
  s[0] = s0;
  s[1] = s1;
  s[2] = s2;
}

// sum over the coarse nodes I around fine node (gx,gy,gz) of P(f,I) x_I
template <typename T>
__device__ __forceinline__ void prolong_node(int fx, int fy, int fz, int cx,
                                             int cy, int cz, int gx, int gy,
                                             int gz, const T *__restrict__ xc,
                                             T s[3]) {
  const int g[3] = {gx, gy, gz}, F[3] = {fx, fy, fz}, Cn[3] = {cx, cy, cz};
  int c0[3], c1[3];
  double w0[3], w1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c0[d] = g[d] >> 1;
    w0[d] = pw1t(g[d], c0[d], F[d]);
    const int c = c0[d] + 1;
    const bool has = (g[d] & 1) && c < Cn[d] && 2 * c <= F[d] - 1;
    w1[d] = has ? pw1t(g[d], c, F[d]) : 0.0;
    c1[d] = min(c, Cn[d] - 1);
  }
  T s0 = T(0), s1 = T(0), s2 = T(0);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ax = k & 1, ay = (k >> 1) & 1, az = k >> 2;
    const T w = static_cast<T>((ax ? w1[0] : w0[0]) * (ay ? w1[1] : w0[1]) *
                               (az ? w1[2] : w0[2]));
    const int64_t I = ((int64_t)(az ? c1[2] : c0[2]) * cy + (ay ? c1[1] : c0[1])) * cx +
                      (ax ? c1[0] : c0[0]);
    s0 += w * xc[3 * I];
    s1 += w * xc[3 * I + 1];
    s2 += w * xc[3 * I + 2];
  }
  s[0] = s0;
  s[1] = s1;
  s[2] = s2;
}

// one row of x = Ainv b by one warp: four independent partial sums so the
// loads of consecutive chunks overlap; result valid in every lane
template <typename T>
__device__ __forceinline__ double gemv_row(const double *__restrict__ a,
                                           const T *__restrict__ b, int64_t n,
                                           int lane) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int64_t k = lane;
  for (; k + 96 < n; k += 128) {
    s0 += a[k] * static_cast<double>(b[k]);
    s1 += a[k + 32] * static_cast<double>(b[k + 32]);
    s2 += a[k + 64] * static_cast<double>(b[k + 64]);
    s3 += a[k + 96] * static_cast<double>(b[k + 96]);
  }
  for (; k < n; k += 32) s0 += a[k] * static_cast<double>(b[k]);
  double s = (s0 + s1) + (s2 + s3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

}  // namespace tpo
