// Persistent coarse-grid V-cycle: every GMG level from `ps` down to the
// coarsest, and the dense coarsest solve, in ONE cooperative kernel.
//
// On the small levels (a few thousand to a few ten thousand nodes) each
// smoothing step, transfer or residual is a microseconds-long latency-bound
// launch; a launch per phase would cost more than the work.  Here the grid
// stays resident (one cooperative launch sized to the co-resident block
// count) and the phases are separated by grid-wide barriers (grid_barrier
// below, valid because the launch guarantees co-residency).  Each phase is
// a grid-stride loop over nodes.  A block of
// NB right-hand sides rides through the same barriers: the stencil of a
// node is read once for all NB columns.
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
#include "coarse.h"
#include "grid_barrier.cuh"
#include "transfer.cuh"

namespace tpo {

namespace {

// y_n = sum_delta A(n, n+delta) u_{n+delta} for one node by one warp, for
// NB columns: lane `q` < 27 loads block q and the neighbour's u of every
// column.  The node-major copy interleaves the 27 blocks per coefficient
// (A[n*243 + (3r+s)*27 + q]), so each of the 9 loads of the warp reads 27
// consecutive values.  The 3 NB partial sums are then reduced
// across the warp by a reduce-scatter: at each of the first log2(NB)
// butterfly steps a lane keeps half of its columns and sends the other
// half, so that afterwards the lanes of group col = lane / (32 / NB) hold
// column col; the remaining steps complete the sums inside each group.
// Out-of-range neighbours have zero blocks; their index is clamped so every
// load stays in bounds.
// FROM_B: the input is the Chebyshev start d0 = inv_theta D^-1 b, formed
// on the fly from b and D^-1 instead of being read from u
template <typename T, int NB, bool FROM_B = false>
__device__ __forceinline__ void warp_stencil(const CoarseLevel<T> &L, int n,
                                             const T *__restrict__ u, int lane,
                                             T acc[3]) {
  const int nx = L.dims[0], ny = L.dims[1], nz = L.dims[2];
  const int64_t ld = 3 * L.nn;
  T p[NB][3];
#pragma unroll
  for (int c = 0; c < NB; ++c) p[c][0] = p[c][1] = p[c][2] = T(0);
  if (lane < 27) {
    const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
    const int mi = min(max(i + lane % 3 - 1, 0), nx - 1);
    const int mj = min(max(j + (lane / 3) % 3 - 1, 0), ny - 1);
    const int mk = min(max(k + lane / 9 - 1, 0), nz - 1);
    const int m = (mk * ny + mj) * nx + mi;
    const T *s = L.A + (int64_t)n * 243 + lane;
    T a[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) a[q] = s[q * 27];
    T di0 = T(0), di1 = T(0), di2 = T(0);
    if (FROM_B) {
      di0 = L.inv_theta * L.dinv[3 * m];
      di1 = L.inv_theta * L.dinv[3 * m + 1];
      di2 = L.inv_theta * L.dinv[3 * m + 2];
    }
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      T u0, u1, u2;
      if (FROM_B) {
        const T *bc = L.b + c * ld;
        u0 = di0 * bc[3 * m];
        u1 = di1 * bc[3 * m + 1];
        u2 = di2 * bc[3 * m + 2];
      } else {
        const T *uc = u + c * ld;
        u0 = uc[3 * m];
        u1 = uc[3 * m + 1];
        u2 = uc[3 * m + 2];
      }
      p[c][0] = a[0] * u0 + a[1] * u1 + a[2] * u2;
      p[c][1] = a[3] * u0 + a[4] * u1 + a[5] * u2;
      p[c][2] = a[6] * u0 + a[7] * u1 + a[8] * u2;
    }
  }
  // reduce-scatter over the columns
  int o = 16;
#pragma unroll
  for (int half = NB / 2; half >= 1; half /= 2, o >>= 1) {
    const bool upper = (lane & o) != 0;
#pragma unroll
    for (int c = 0; c < half; ++c)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const T send = upper ? p[c][q] : p[c + half][q];
        const T keep = upper ? p[c + half][q] : p[c][q];
        p[c][q] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
  }
  for (; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < 3; ++q) p[0][q] += __shfl_xor_sync(0xffffffffu, p[0][q], o);
  acc[0] = p[0][0];
  acc[1] = p[0][1];
  acc[2] = p[0][2];
}

// lanes per column group after warp_stencil, and the (column, component)
// a lane writes: lanes with comp < 3 write
template <int NB>
struct LaneMap {
  static constexpr int G = 32 / NB;
  int col, comp;
  __device__ explicit LaneMap(int lane) : col(lane / G), comp(lane % G) {}
};

template <typename T>
__device__ __forceinline__ T pick(const T a[3], int q) {
  return q == 0 ? a[0] : (q == 1 ? a[1] : a[2]);
}

// co-resident blocks per SM: 4 for one column (<= 64 registers; measured
// best of 1..6, the small spills cost less than the missing warps), 2 (<= 128
// registers) for wider blocks:
// the phases are latency-bound and need the warps
template <typename T, int NB>
__global__ void __launch_bounds__(kCoarseThreads, NB == 1 ? 4 : 2)
    k_coarse_cycle(CoarseCycle<T> P) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int gwarp = (int)(tid >> 5), nwarps = (int)(nthr >> 5);
  const LaneMap<NB> lm(lane);
  const bool writer = lm.comp < 3;

  // ---------------- down-sweep: pre-smooth, residual, restrict
  for (int l = 0; l < P.nlev; ++l) {
    CoarseLevel<T> &L = P.lev[l];
    const int nn = (int)L.nn;
    const int64_t ld = 3 * L.nn;
    T *dc = L.d0, *dn = L.d1;
    if (L.deg >= 2) {
      // start (d0 = inv_theta D^-1 b, x = d0) fused with the first step
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil<T, NB, true>(L, n, nullptr, lane, a);
        if (writer) {
          const int64_t e = 3 * (int64_t)n + lm.comp;
          const int64_t i = lm.col * ld + e;
          const T di = L.dinv[e];
          const T r0 = di * L.b[i];
          const T d0 = r0 * L.inv_theta;
          const T r = r0 - di * pick(a, lm.comp);
          const T d = L.c1[1] * d0 + L.c2[1] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xpre[i] = d0 + d;
        }
      }
      if (!grid_barrier(P.bar, P.fault)) return;
      T *t = dc; dc = dn; dn = t;
    } else {
      for (int64_t i = tid; i < NB * ld; i += nthr)
        L.xpre[i] = L.inv_theta * (L.dinv[i % ld] * L.b[i]);
      if (!grid_barrier(P.bar, P.fault)) return;
    }
    for (int k = 2; k < L.deg; ++k) {
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil<T, NB>(L, n, dc, lane, a);
        if (writer) {
          const int64_t e = 3 * (int64_t)n + lm.comp;
          const int64_t i = lm.col * ld + e;
          const T r = L.r[i] - L.dinv[e] * pick(a, lm.comp);
          const T d = L.c1[k] * dc[i] + L.c2[k] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xpre[i] += d;
        }
      }
      if (!grid_barrier(P.bar, P.fault)) return;
      T *t = dc; dc = dn; dn = t;
    }
    for (int n = gwarp; n < nn; n += nwarps) {
      T a[3];
      warp_stencil<T, NB>(L, n, L.xpre, lane, a);
      if (writer) {
        const int64_t i = lm.col * ld + 3 * (int64_t)n + lm.comp;
        L.res[i] = L.b[i] - pick(a, lm.comp);
      }
    }
    if (!grid_barrier(P.bar, P.fault)) return;
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
#pragma unroll 1
      for (int c = 0; c < NB; ++c) {
        T s[3];
        restrict_node(fx, fy, fz, ix, iy, iz, L.res + c * ld, s);
        T *o = bc + c * 3 * nnc;
        o[3 * I] = s[0];
        o[3 * I + 1] = s[1];
        o[3 * I + 2] = s[2];
      }
    }
    if (!grid_barrier(P.bar, P.fault)) return;
  }

  // ---------------- coarsest: x = Ainv b, a warp per row, FP64 accumulation
  for (int row = gwarp; row < (int)P.nc && NB == 1; row += nwarps) {
    const double s = gemv_row(P.Ainv + (int64_t)row * P.nc, P.bc, P.nc, lane);
    if (lane == 0) P.xc[row] = static_cast<T>(s);
  }
  for (int row = gwarp; row < (int)P.nc && NB > 1; row += nwarps) {
    const double *a = P.Ainv + (int64_t)row * P.nc;
    double s[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) s[c] = 0.0;
    for (int64_t k = lane; k < P.nc; k += 32) {
      const double av = a[k];
#pragma unroll
      for (int c = 0; c < NB; ++c)
        s[c] += av * static_cast<double>(P.bc[c * P.nc + k]);
    }
#pragma unroll
    for (int c = 0; c < NB; ++c) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_xor_sync(0xffffffffu, s[c], o);
    }
#pragma unroll
    for (int c = 0; c < NB; ++c)
      if (lane == c) P.xc[c * P.nc + row] = static_cast<T>(s[c]);
  }
  if (!grid_barrier(P.bar, P.fault)) return;

  // ---------------- up-sweep: prolong-add, post-smooth
  for (int l = P.nlev - 1; l >= 0; --l) {
    CoarseLevel<T> &L = P.lev[l];
    const int nn = (int)L.nn;
    const int64_t ld = 3 * L.nn;
    const bool dense_child = (l + 1 == P.nlev);
    const T *xc = dense_child ? P.xc : P.lev[l + 1].xout;
    const int cx = dense_child ? P.cdims[0] : P.lev[l + 1].dims[0];
    const int cy = dense_child ? P.cdims[1] : P.lev[l + 1].dims[1];
    const int cz = dense_child ? P.cdims[2] : P.lev[l + 1].dims[2];
    const int64_t ldc = 3 * (int64_t)cx * cy * cz;
    const int fx = L.dims[0], fy = L.dims[1], fz = L.dims[2];
    for (int f = (int)tid; f < nn; f += (int)nthr) {
      const int gx = f % fx, gy = (f / fx) % fy, gz = f / (fx * fy);
#pragma unroll 1
      for (int c = 0; c < NB; ++c) {
        T s[3];
        prolong_node(fx, fy, fz, cx, cy, cz, gx, gy, gz, xc + c * ldc, s);
        T *x = L.xpre + c * ld;
        x[3 * f] += s[0];
        x[3 * f + 1] += s[1];
        x[3 * f + 2] += s[2];
      }
    }
    if (!grid_barrier(P.bar, P.fault)) return;
    for (int n = gwarp; n < nn; n += nwarps) {
      T a[3];
      warp_stencil<T, NB>(L, n, L.xpre, lane, a);
      if (writer) {
        const int64_t e = 3 * (int64_t)n + lm.comp;
        const int64_t i = lm.col * ld + e;
        const T r = L.dinv[e] * (L.b[i] - pick(a, lm.comp));
        const T d = r * L.inv_theta;
        L.r[i] = r;
        L.d0[i] = d;
        L.xout[i] = L.xpre[i] + d;
      }
    }
    if (!grid_barrier(P.bar, P.fault)) return;
    T *dc = L.d0, *dn = L.d1;
    for (int k = 1; k < L.deg; ++k) {
      for (int n = gwarp; n < nn; n += nwarps) {
        T a[3];
        warp_stencil<T, NB>(L, n, dc, lane, a);
        if (writer) {
          const int64_t e = 3 * (int64_t)n + lm.comp;
          const int64_t i = lm.col * ld + e;
          const T r = L.r[i] - L.dinv[e] * pick(a, lm.comp);
          const T d = L.c1[k] * dc[i] + L.c2[k] * r;
          L.r[i] = r;
          dn[i] = d;
          L.xout[i] += d;
        }
      }
      if (!grid_barrier(P.bar, P.fault)) return;
      T *t = dc; dc = dn; dn = t;
    }
  }
}

template <typename T, int NB>
int grid_size_for() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!cached[dev]) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coarse_cycle<T, NB>,
                                                  kCoarseThreads, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = std::max(1, std::min(per_sm, 4)) * sms;
  }
  return cached[dev];
}

template <typename T, int NB>
cudaError_t launch_nb(const CoarseCycle<T> &P, cudaStream_t s) {
  const int grid = grid_size_for<T, NB>();
  void *args[] = {const_cast<CoarseCycle<T> *>(&P)};
  return cudaLaunchCooperativeKernel((const void *)k_coarse_cycle<T, NB>, grid,
                                     kCoarseThreads, args, 0, s);
}

}  // namespace

template <typename T>
cudaError_t launch_coarse_cycle(const CoarseCycle<T> &P, cudaStream_t s) {
  count_launch();
  switch (P.nb) {
    case 1: return launch_nb<T, 1>(P, s);
    case 2: return launch_nb<T, 2>(P, s);
    case 4: return launch_nb<T, 4>(P, s);
    case 8: return launch_nb<T, 8>(P, s);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launch_coarse_cycle<double>(const CoarseCycle<double> &,
                                                 cudaStream_t);
template cudaError_t launch_coarse_cycle<float>(const CoarseCycle<float> &,
                                                cudaStream_t);

}  // namespace tpo
