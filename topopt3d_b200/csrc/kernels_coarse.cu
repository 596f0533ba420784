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
#include "transfer.cuh"

namespace cg = cooperative_groups;

namespace tpo {

namespace {

// y_n = sum_delta A(n, n+delta) u_{n+delta} for one node by one warp: lane
// `nb` < 27 loads block nb (9 contiguous values of the node-major copy,
// so the warp reads 243 consecutive values) and the neighbour's u, then the
// three partial sums are reduced across the warp.  Out-of-range neighbours
// have zero blocks; their index is clamped so every load stays in bounds.
// Every lane returns the full sums.
// FROM_B: the input is the Chebyshev start d0 = inv_theta D^-1 b, formed
// on the fly from b and D^-1 instead of being read from u
template <typename T, bool FROM_B = false>
__device__ __forceinline__ void warp_stencil(const CoarseLevel<T> &L, int n,
                                             const T *__restrict__ u, int lane,
                                             T acc[3]) {
  const int nx = L.dims[0], ny = L.dims[1], nz = L.dims[2];
  T p0 = T(0), p1 = T(0), p2 = T(0);
  if (lane < 27) {
    const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
    const int mi = min(max(i + lane % 3 - 1, 0), nx - 1);
    const int mj = min(max(j + (lane / 3) % 3 - 1, 0), ny - 1);
    const int mk = min(max(k + lane / 9 - 1, 0), nz - 1);
    const int m = (mk * ny + mj) * nx + mi;
    const T *s = L.A + (int64_t)n * 243 + lane * 9;
    T u0, u1, u2;
    if (FROM_B) {
      u0 = L.inv_theta * (L.dinv[3 * m] * L.b[3 * m]);
      u1 = L.inv_theta * (L.dinv[3 * m + 1] * L.b[3 * m + 1]);
      u2 = L.inv_theta * (L.dinv[3 * m + 2] * L.b[3 * m + 2]);
    } else {
      u0 = u[3 * m];
      u1 = u[3 * m + 1];
      u2 = u[3 * m + 2];
    }
    p0 = s[0] * u0 + s[1] * u1 + s[2] * u2;
    p1 = s[3] * u0 + s[4] * u1 + s[5] * u2;
    p2 = s[6] * u0 + s[7] * u1 + s[8] * u2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    p0 += __shfl_xor_sync(0xffffffffu, p0, o);
    p1 += __shfl_xor_sync(0xffffffffu, p1, o);
    p2 += __shfl_xor_sync(0xffffffffu, p2, o);
  }
  acc[0] = p0;
  acc[1] = p1;
  acc[2] = p2;
}

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads)
    k_coarse_cycle(CoarseCycle<T> P) {
  cg::grid_group grid = cg::this_grid();
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int gwarp = (int)(tid >> 5), nwarps = (int)(nthr >> 5);

  // ---------------- down-sweep: pre-smooth, residual, restrict
  for (int l = 0; l < P.nlev; ++l) {
    CoarseLevel<T> &L = P.lev[l];
    const int nn = (int)L.nn;
    T *dc = L.d0, *dn = L.d1;
    if (L.deg >= 2) {
      // start (d0 = inv_theta D^-1 b, x = d0) fused with the first step
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil<T, true>(L, n, nullptr, lane, a);
        if (lane < 3) {
          const int64_t i = 3 * (int64_t)n + lane;
          const T di = L.dinv[i];
          const T r0 = di * L.b[i];
          const T d0 = r0 * L.inv_theta;
          const T r = r0 - di * a[lane];
          const T d = L.c1[1] * d0 + L.c2[1] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xpre[i] = d0 + d;
        }
      }
      grid.sync();
      T *t = dc; dc = dn; dn = t;
    } else {
      for (int64_t i = tid; i < 3 * (int64_t)nn; i += nthr)
        L.xpre[i] = L.inv_theta * (L.dinv[i] * L.b[i]);
      grid.sync();
    }
    for (int k = 2; k < L.deg; ++k) {
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil(L, n, dc, lane, a);
        if (lane < 3) {
          const int64_t i = 3 * (int64_t)n + lane;
          const T r = L.r[i] - L.dinv[i] * a[lane];
          const T d = L.c1[k] * dc[i] + L.c2[k] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xpre[i] += d;
        }
      }
      grid.sync();
      T *t = dc; dc = dn; dn = t;
    }
    for (int n = gwarp; n < nn; n += nwarps) {
      T a[3];
      warp_stencil(L, n, L.xpre, lane, a);
      if (lane < 3) L.res[3 * (int64_t)n + lane] = L.b[3 * (int64_t)n + lane] - a[lane];
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
    for (int I = (int)tid; I < (int)nnc; I += (int)nthr) {
      const int ix = I % cx, iy = (I / cx) % cy, iz = I / (cx * cy);
      T s[3];
      restrict_node(fx, fy, fz, ix, iy, iz, L.res, s);
      bc[3 * I] = s[0];
      bc[3 * I + 1] = s[1];
      bc[3 * I + 2] = s[2];
    }
    grid.sync();
  }

  // ---------------- coarsest: x = Ainv b, a warp per row, FP64 accumulation
  for (int row = gwarp; row < (int)P.nc; row += nwarps) {
    const double s = gemv_row(P.Ainv + (int64_t)row * P.nc, P.bc, P.nc, lane);
    if (lane == 0) P.xc[row] = static_cast<T>(s);
  }
  grid.sync();

  // ---------------- up-sweep: prolong-add, post-smooth
  for (int l = P.nlev - 1; l >= 0; --l) {
    CoarseLevel<T> &L = P.lev[l];
    const int nn = (int)L.nn;
    const bool dense_child = (l + 1 == P.nlev);
    const T *xc = dense_child ? P.xc : P.lev[l + 1].xout;
    const int cx = dense_child ? P.cdims[0] : P.lev[l + 1].dims[0];
    const int cy = dense_child ? P.cdims[1] : P.lev[l + 1].dims[1];
    const int cz = dense_child ? P.cdims[2] : P.lev[l + 1].dims[2];
    const int fx = L.dims[0], fy = L.dims[1], fz = L.dims[2];
    for (int f = (int)tid; f < nn; f += (int)nthr) {
      const int gx = f % fx, gy = (f / fx) % fy, gz = f / (fx * fy);
      T s[3];
      prolong_node(fx, fy, fz, cx, cy, cz, gx, gy, gz, xc, s);
      L.xpre[3 * f] += s[0];
      L.xpre[3 * f + 1] += s[1];
      L.xpre[3 * f + 2] += s[2];
    }
    grid.sync();
    for (int n = gwarp; n < nn; n += nwarps) {
      T a[3];
      warp_stencil(L, n, L.xpre, lane, a);
      if (lane < 3) {
        const int64_t i = 3 * (int64_t)n + lane;
        const T r = L.dinv[i] * (L.b[i] - a[lane]);
        const T d = r * L.inv_theta;
        L.r[i] = r;
        L.d0[i] = d;
        L.xout[i] = L.xpre[i] + d;
      }
    }
    grid.sync();
    T *dc = L.d0, *dn = L.d1;
    for (int k = 1; k < L.deg; ++k) {
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil(L, n, dc, lane, a);
        if (lane < 3) {
          const int64_t i = 3 * (int64_t)n + lane;
          const T r = L.r[i] - L.dinv[i] * a[lane];
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
