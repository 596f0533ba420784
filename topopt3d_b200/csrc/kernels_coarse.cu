// Persistent coarse-grid V-cycle: every GMG level from `ps` down to the
// coarsest, and the dense coarsest solve, in ONE cooperative kernel.
//
// On the small levels (a few thousand to a few ten thousand nodes) each
// smoothing step, transfer or residual is a microseconds-long latency-bound
// launch; a launch per phase would cost more than the work.  Here the grid
// stays resident (one cooperative launch sized to the co-resident block
// count) and the phases are separated by grid-wide barriers
// (cooperative_groups grid sync, valid because the launch guarantees
// co-residency).  Each phase is a grid-stride loop over nodes.
//
// Per level (Chebyshev degree m, Jacobi): the stencil apply and the
// Chebyshev update of a node are fused into one phase by ping-ponging the
// search direction d (readers use d_k, the phase writes d_{k+1}), so a
// Chebyshev step costs one barrier:
//   pre:  r = D^-1 b, d = r/theta, x = d;  m-1 x [r -= D^-1 A d;
//         d' = c1 d + c2 r; x += d']
//   res = b - A x;  b_c = P^T res;  (recurse);  x += P x_c
//   post: r = D^-1 (b - A x), d = r/theta, x' = x + d;  m-1 x [...]
// The level math is the one of the per-level kernels in kernels_mg.cu.
#include <cooperative_groups.h>

#include "coarse.h"

namespace cg = cooperative_groups;

namespace tpo {

namespace {

__device__ __forceinline__ double pw1c(int f, int c, int Nf) {
  const int d = f - 2 * c;
  if (d < -1 || d > 1) return 0.0;
  if (d == 0) return 1.0;
  return (f + 1 <= Nf - 1) ? 0.5 : 1.0;
}

// y_I = sum_delta A(I, I+delta) u_{I+delta} for one node, branch-free over
// the 27 neighbours (out-of-range neighbours have zero blocks; their index is
// clamped so the load stays in bounds)
template <typename T>
__device__ __forceinline__ void stencil_row(const CoarseLevel<T> &L, int64_t n,
                                            const T *__restrict__ u, T acc[3]) {
  const int nx = L.dims[0], ny = L.dims[1], nz = L.dims[2];
  const int64_t nn = L.nn;
  const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / ((int64_t)nx * ny));
  acc[0] = acc[1] = acc[2] = T(0);
#pragma unroll
  for (int nb = 0; nb < 27; ++nb) {
    const int mi = min(max(i + nb % 3 - 1, 0), nx - 1);
    const int mj = min(max(j + (nb / 3) % 3 - 1, 0), ny - 1);
    const int mk = min(max(k + nb / 9 - 1, 0), nz - 1);
    const int64_t m = ((int64_t)mk * ny + mj) * nx + mi;
    const T u0 = u[3 * m], u1 = u[3 * m + 1], u2 = u[3 * m + 2];
    const T *s = L.S + (int64_t)nb * 9 * nn + n;
    acc[0] += s[0] * u0 + s[nn] * u1 + s[2 * nn] * u2;
    acc[1] += s[3 * nn] * u0 + s[4 * nn] * u1 + s[5 * nn] * u2;
    acc[2] += s[6 * nn] * u0 + s[7 * nn] * u1 + s[8 * nn] * u2;
  }
}

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads)
    k_coarse_cycle(CoarseCycle<T> P) {
  cg::grid_group grid = cg::this_grid();
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;

  // ---------------- down-sweep: pre-smooth, residual, restrict
  for (int l = 0; l < P.nlev; ++l) {
    CoarseLevel<T> &L = P.lev[l];
    const int64_t n3 = 3 * L.nn;
    for (int64_t i = tid; i < n3; i += nthr) {
      const T r = L.dinv[i] * L.b[i];
      const T d = r * L.inv_theta;
      L.r[i] = r;
      L.d0[i] = d;
      L.xpre[i] = d;
    }
    grid.sync();
    T *dc = L.d0, *dn = L.d1;
    for (int k = 1; k < L.deg; ++k) {
      for (int64_t n = tid; n < L.nn; n += nthr) {
        T a[3];
        stencil_row(L, n, dc, a);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int64_t i = 3 * n + c;
          const T r = L.r[i] - L.dinv[i] * a[c];
          const T d = L.c1[k] * dc[i] + L.c2[k] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xpre[i] += d;
        }
      }
      grid.sync();
      T *t = dc; dc = dn; dn = t;
    }
    for (int64_t n = tid; n < L.nn; n += nthr) {
      T a[3];
      stencil_row(L, n, L.xpre, a);
#pragma unroll
      for (int c = 0; c < 3; ++c) L.res[3 * n + c] = L.b[3 * n + c] - a[c];
    }
    grid.sync();
    // b_child = P^T res
    const bool dense_next = (l + 1 == P.nlev);
    T *bc = dense_next ? P.bc : P.lev[l + 1].b;
    const int cx = dense_next ? P.cdims[0] : P.lev[l + 1].dims[0];
    const int cy = dense_next ? P.cdims[1] : P.lev[l + 1].dims[1];
    const int cz = dense_next ? P.cdims[2] : P.lev[l + 1].dims[2];
    const int fx = L.dims[0], fy = L.dims[1], fz = L.dims[2];
    const int64_t nnc = (int64_t)cx * cy * cz;
    for (int64_t I = tid; I < nnc; I += nthr) {
      const int ix = I % cx, iy = (I / cx) % cy, iz = I / ((int64_t)cx * cy);
      T s0 = 0, s1 = 0, s2 = 0;
      for (int az = -1; az <= 1; ++az) {
        const int gz = 2 * iz + az;
        if (gz < 0 || gz >= fz) continue;
        const double wz = pw1c(gz, iz, fz);
        for (int ay = -1; ay <= 1; ++ay) {
          const int gy = 2 * iy + ay;
          if (gy < 0 || gy >= fy) continue;
          const double wy = pw1c(gy, iy, fy);
          for (int ax = -1; ax <= 1; ++ax) {
            const int gx = 2 * ix + ax;
            if (gx < 0 || gx >= fx) continue;
            const T w = static_cast<T>(pw1c(gx, ix, fx) * wy * wz);
            const int64_t f = ((int64_t)gz * fy + gy) * fx + gx;
            s0 += w * L.res[3 * f];
            s1 += w * L.res[3 * f + 1];
            s2 += w * L.res[3 * f + 2];
          }
        }
      }
      bc[3 * I] = s0;
      bc[3 * I + 1] = s1;
      bc[3 * I + 2] = s2;
    }
    grid.sync();
  }

  // ---------------- coarsest: x = Ainv b, a warp per row, FP64 accumulation
  {
    const int lane = threadIdx.x & 31;
    const int64_t warp = tid >> 5, nwarps = nthr >> 5;
    for (int64_t row = warp; row < P.nc; row += nwarps) {
      const double *a = P.Ainv + row * P.nc;
      double s = 0;
      for (int64_t k = lane; k < P.nc; k += 32) s += a[k] * static_cast<double>(P.bc[k]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) P.xc[row] = static_cast<T>(s);
    }
  }
  grid.sync();

  // ---------------- up-sweep: prolong-add, post-smooth
  for (int l = P.nlev - 1; l >= 0; --l) {
    CoarseLevel<T> &L = P.lev[l];
    const bool dense_child = (l + 1 == P.nlev);
    const T *xc = dense_child ? P.xc : P.lev[l + 1].xout;
    const int cx = dense_child ? P.cdims[0] : P.lev[l + 1].dims[0];
    const int cy = dense_child ? P.cdims[1] : P.lev[l + 1].dims[1];
    const int cz = dense_child ? P.cdims[2] : P.lev[l + 1].dims[2];
    const int fx = L.dims[0], fy = L.dims[1], fz = L.dims[2];
    for (int64_t f = tid; f < L.nn; f += nthr) {
      const int gx = f % fx, gy = (f / fx) % fy, gz = f / ((int64_t)fx * fy);
      T s0 = 0, s1 = 0, s2 = 0;
      for (int c2 = gz / 2; 2 * c2 <= gz + 1 && c2 < cz; ++c2) {
        const double wz = pw1c(gz, c2, fz);
        for (int c1 = gy / 2; 2 * c1 <= gy + 1 && c1 < cy; ++c1) {
          const double wy = pw1c(gy, c1, fy);
          for (int c0 = gx / 2; 2 * c0 <= gx + 1 && c0 < cx; ++c0) {
            const T w = static_cast<T>(pw1c(gx, c0, fx) * wy * wz);
            const int64_t I = ((int64_t)c2 * cy + c1) * cx + c0;
            s0 += w * xc[3 * I];
            s1 += w * xc[3 * I + 1];
            s2 += w * xc[3 * I + 2];
          }
        }
      }
      L.xpre[3 * f] += s0;
      L.xpre[3 * f + 1] += s1;
      L.xpre[3 * f + 2] += s2;
    }
    grid.sync();
    for (int64_t n = tid; n < L.nn; n += nthr) {
      T a[3];
      stencil_row(L, n, L.xpre, a);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t i = 3 * n + c;
        const T r = L.dinv[i] * (L.b[i] - a[c]);
        const T d = r * L.inv_theta;
        L.r[i] = r;
        L.d0[i] = d;
        L.xout[i] = L.xpre[i] + d;
      }
    }
    grid.sync();
    T *dc = L.d0, *dn = L.d1;
    for (int k = 1; k < L.deg; ++k) {
      for (int64_t n = tid; n < L.nn; n += nthr) {
        T a[3];
        stencil_row(L, n, dc, a);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int64_t i = 3 * n + c;
          const T r = L.r[i] - L.dinv[i] * a[c];
          const T d = L.c1[k] * dc[i] + L.c2[k] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xout[i] += d;
        }
      }
      grid.sync();
      T *t = dc; dc = dn; dn = t;
    }
  }
}

template <typename T>
int grid_size_for() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!cached[dev]) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coarse_cycle<T>,
                                                  kCoarseThreads, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = std::max(1, std::min(per_sm, 4)) * sms;
  }
  return cached[dev];
}

}  // namespace

template <typename T>
cudaError_t launch_coarse_cycle(const CoarseCycle<T> &P, cudaStream_t s) {
  count_launch();
  const int grid = grid_size_for<T>();
  void *args[] = {const_cast<CoarseCycle<T> *>(&P)};
  return cudaLaunchCooperativeKernel((const void *)k_coarse_cycle<T>, grid,
                                     kCoarseThreads, args, 0, s);
}

template cudaError_t launch_coarse_cycle<double>(const CoarseCycle<double> &,
                                                 cudaStream_t);
template cudaError_t launch_coarse_cycle<float>(const CoarseCycle<float> &,
                                                cudaStream_t);

}  // namespace tpo
