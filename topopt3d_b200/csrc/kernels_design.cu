// Design-side kernels: the density filter (forward and transpose, matrix
// free), SIMP interpolation, the compliance sensitivity and the OC update.
#include <math_constants.h>

#include "grid_barrier.cuh"
#include "modal.cuh"

namespace tpo {

namespace {

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

// row sums of the raw filter (Filter.cpp:136-147): finv = 1 / sum_j W_ij,
// summed in increasing column order
__global__ void k_filter_rowsum(int nx, int ny, int nz,
                                const FilterTaps *__restrict__ taps,
                                double *finv) {
  const int64_t ne = (int64_t)nx * ny * nz;
  const int nt = taps->n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
    double s = 0;
    for (int t = 0; t < nt; ++t) {
      const int a = i + taps->off[t][0], b = j + taps->off[t][1], c = k + taps->off[t][2];
      if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
      s += taps->w[t];
    }
    finv[e] = 1.0 / s;
  }
}

// rho_i = sum_j (W_ij * finv_i) x_j  (MatMult(P), Material_Interpolation.cpp:35)
__global__ void k_filter_fwd(int nx, int ny, int nz,
                             const FilterTaps *__restrict__ taps,
                             const double *__restrict__ finv,
                             const double *__restrict__ in,
                             double *__restrict__ out) {
  const int64_t ne = (int64_t)nx * ny * nz;
  const int nt = taps->n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
    const double fi = finv[e];
    double s = 0;
    for (int t = 0; t < nt; ++t) {
      const int a = i + taps->off[t][0], b = j + taps->off[t][1], c = k + taps->off[t][2];
      if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
      s += (taps->w[t] * fi) * in[((int64_t)c * ny + b) * nx + a];
    }
    out[e] = s;
  }
}

// out_j = sum_i (W_ij * finv_i) g_i over rows i in increasing order
// (MatMultTranspose(P), Material_Interpolation.cpp:160,180)
__global__ void k_filter_adj(int nx, int ny, int nz,
                             const FilterTaps *__restrict__ taps,
                             const double *__restrict__ finv,
                             const double *__restrict__ in, double uniform,
                             double *__restrict__ out) {
  const int64_t ne = (int64_t)nx * ny * nz;
  const int nt = taps->n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
    double s = 0;
    for (int t = nt - 1; t >= 0; --t) {
      const int a = i - taps->off[t][0], b = j - taps->off[t][1], c = k - taps->off[t][2];
      if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
      const int64_t r = ((int64_t)c * ny + b) * nx + a;
      s += (taps->w[t] * finv[r]) * (in ? in[r] : uniform);
    }
    out[e] = s;
  }
}

// PETSc VecPow special cases (used by MatIntFnc)
__device__ __forceinline__ double vecpow(double v, double p) {
  if (p == 1.0) return v;
  if (p == -1.0) return 1.0 / v;
  if (p == 0.0) return (v == v) ? 1.0 : v;
  if (p == 0.5) return v >= 0 ? sqrt(v) : CUDART_INF;
  if (p == -0.5) return v >= 0 ? 1.0 / sqrt(v) : CUDART_INF;
  if (p == 2.0) return v * v;
  if (p == -2.0) return 1.0 / (v * v);
  return v >= 0 ? pow(v, p) : CUDART_INF;
}

// Material_Interpolation.cpp:40-75 with vdMin <= 0 (y = 1, z = rho)
__global__ void k_simp(int64_t ne, const double *__restrict__ rho, double penal,
                       double eps, double *E, double *dEdz, float *E32,
                       double *Es, double *dEsdz) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const double z = rho[e];
    double d = vecpow(z, penal - 1);
    const double es = d * z;
    d = d * penal;
    dEsdz[e] = d;
    dEdz[e] = d * (1 - eps);
    const double Ee = eps + (1 - eps) * es;
    E[e] = Ee;
    E32[e] = static_cast<float>(Ee);
    Es[e] = es;
  }
}

// dc_e = -dEdz_e * u_e^T K0 u_e (Compliance.cpp:37-46)
__global__ void k_sensitivity(int nelx, int nely, int nelz,
                              const double *__restrict__ U,
                              const double *__restrict__ dEdz, double *dc,
                              const Kh<double> kh) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nelx, j = (e / nelx) % nely, k = e / ((int64_t)nelx * nely);
    double v[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int64_t n = ((int64_t)(k + (l >> 2)) * Ny + (j + ((l >> 1) & 1))) * Nx +
                        (i + (l & 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) v[l][c] = U[3 * n + c];
    }
    dc[e] = -dEdz[e] * element_energy(v, kh);
  }
}

__global__ void k_oc_clip(int64_t n, double *dfdx) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (dfdx[i] > 0) dfdx[i] = 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// one bisection trial of MMA::OCsub (MMA.cpp:139-160): candidate x and
// per-block partial sums of dgdx . (x - xold)
__global__ void k_oc_step(int64_t n, double *x, const double *xold,
                          const double *xmin, const double *xmax,
                          const double *dfdx, const double *dgdx, double move,
                          double lmid, double *part) {
  __shared__ double sh[32];
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double B = pow(-dfdx[i] / dgdx[i] / lmid, 0.5);
    const double xo = xold[i], lo = xmin[i], hi = xmax[i];
    const double step = move * (hi - lo);
    double v = lo + (xo - lo) * B;
    v = fmin(v, xo + step);
    v = fmin(v, hi);
    v = fmax(v, xo - step);
    v = fmax(v, lo);
    x[i] = v;
    s += dgdx[i] * (v - xo);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
}

__global__ void k_sum_parts(int nparts, const double *part, double *out) {
  __shared__ double sh[32];
  double s = 0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) *out = s;
  }
}

// The whole bisection of MMA::OCsub (MMA.cpp:136-161) in one cooperative
// launch of kRedBlocks x 256 threads, with no host round trip per trial.
// Each trial forms the candidate x and the block's partial of
// dgdx . (x - xold) exactly as k_oc_step does on the same grid; after a grid
// barrier every block sums the kRedBlocks partials in k_sum_parts' order,
// so all blocks hold the same total and take the same branch.  The
// partials are double-buffered by trial parity: a block writes the next
// trial's partials only after the next barrier, which every block reaches
// after reading the current ones.
__global__ void __launch_bounds__(256)
    k_oc_bisect(int64_t n, double *x, const double *xold, const double *xmin,
                const double *xmax, const double *dfdx, const double *dgdx,
                double move, double g, double *part, unsigned int *bar,
                double *fault) {
  __shared__ double sh[32];
  __shared__ double total;
  double l1 = 0, l2 = 1e6;
  int trial = 0;
  while (l2 - l1 > 1e-4) {
    const double lmid = 0.5 * (l1 + l2);
    double *pp = part + (trial & 1) * gridDim.x;
    double s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      const double B = pow(-dfdx[i] / dgdx[i] / lmid, 0.5);
      const double xo = xold[i], lo = xmin[i], hi = xmax[i];
      const double step = move * (hi - lo);
      double v = lo + (xo - lo) * B;
      v = fmin(v, xo + step);
      v = fmin(v, hi);
      v = fmax(v, xo - step);
      v = fmax(v, lo);
      x[i] = v;
      s += dgdx[i] * (v - xo);
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      s = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
      s = warp_sum(s);
      if (threadIdx.x == 0) pp[blockIdx.x] = s;
    }
    if (!grid_barrier(bar, fault)) return;
    double t = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += pp[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x < 32) {
      t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
      t = warp_sum(t);
      if (threadIdx.x == 0) total = t;
    }
    __syncthreads();
    if (g + total > 0) l1 = lmid; else l2 = lmid;
    ++trial;
    __syncthreads();
  }
}

// ---- MMA for m >= 2 constraints (MMA::MMAsub, MMA.cpp:185-343, and
// MMA::DualSolve, :353-595).  Every element-wise pass reduces into
// per-block partials over the fixed kRedBlocks grid (m values per block for
// b, m + m(m+1)/2 for the dual gradient and Hessian); the host sums them in
// a fixed order, so the result does not depend on scheduling.

// sum of v over the block into out (thread 0), v a per-thread value
__device__ __forceinline__ double block_total(double v, double *sh) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

// asymptotes (:219-247), move limits alfa/beta (:250-262), p0, q0, P, Q
// (:265-300) and the partials of b (:303-305); then xold2 <- xold1 <- x
// (:307).  P and Q are n x m column-major.
__global__ void __launch_bounds__(256)
    k_mma_prepare(int64_t n, int m, bool fresh, MmaConst k, double *x, double *x1,
                  double *x2, double *low, double *upp, const double *xmin,
                  const double *xmax, const double *dfdx, const double *dgdx,
                  double *alfa, double *beta, double *p0, double *q0, double *P,
                  double *Q, double *part) {
  __shared__ double sh[32];
  double bs[kMmaMaxM];
  for (int j = 0; j < m; ++j) bs[j] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double xi = x[i], span = xmax[i] - xmin[i];
    double lo, up;
    if (fresh) {
      lo = xi - k.asyinit * span;
      up = xi + k.asyinit * span;
    } else {
      const double xa = x1[i], xb = x2[i];
      const double zz = (xi - xa) * (xa - xb);
      const double f = zz > 0 ? k.asyincr : (zz < 0 ? k.asydecr : 1.0);
      lo = xi - f * (xa - low[i]);
      up = xi + f * (upp[i] - xa);
      lo = fmin(fmax(lo, xi - 10 * span), xi - 0.01 * span);
      up = fmax(fmin(up, xi + 10 * span), xi + 0.01 * span);
    }
    alfa[i] = fmax(fmax(lo + k.albefa * (xi - lo), xi - k.move * span), xmin[i]);
    beta[i] = fmin(fmin(up - k.albefa * (up - xi), xi + k.move * span), xmax[i]);
    const double xmami = fmax(up - lo, 1e-5);
    const double ux1 = up - xi, xl1 = xi - lo, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    const double df = dfdx[i];
    double pp = fmax(df, 0.0), qq = fmax(-df, 0.0);
    const double pq0 = 0.001 * (pp + qq) + 0.5 * k.raa0 / xmami;
    p0[i] = (pp + pq0) * ux2;
    q0[i] = (qq + pq0) * xl2;
    for (int j = 0; j < m; ++j) {
      const double dg = dgdx[j * n + i];
      const double Pj = fmax(dg, 0.0) * ux2, Qj = fmax(-dg, 0.0) * xl2;
      P[j * n + i] = Pj;
      Q[j * n + i] = Qj;
      bs[j] += Pj / ux1 + Qj / xl1;
    }
    low[i] = lo;
    upp[i] = up;
    x2[i] = x1[i];
    x1[i] = xi;
  }
  for (int j = 0; j < m; ++j) {
    const double t = block_total(bs[j], sh);
    if (threadIdx.x == 0) part[blockIdx.x * m + j] = t;
  }
}

// x(lambda) (XYZofLam, :432-447) and the partials of the dual gradient sums
// sum_n P_j/ux1 + Q_j/xl1 (DualGrad, :461-474) and of the Hessian sums
// sum_n dhdx_j dLdxx dhdx_k, k >= j (DualHess, :489-515), at lambda
__global__ void __launch_bounds__(256)
    k_mma_dual(int64_t n, int m, MmaLambda lam, const double *alfa, const double *beta,
               const double *low, const double *upp, const double *p0,
               const double *q0, const double *P, const double *Q, double *x,
               double *part) {
  __shared__ double sh[32];
  const int nh = m * (m + 1) / 2, nv = m + nh;
  double acc[kMmaMaxM + kMmaMaxM * (kMmaMaxM + 1) / 2];
  for (int j = 0; j < nv; ++j) acc[j] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double plam = p0[i], qlam = q0[i];
    for (int j = 0; j < m; ++j) {
      plam += P[j * n + i] * lam.v[j];
      qlam += Q[j * n + i] * lam.v[j];
    }
    const double lo = low[i], up = upp[i], al = alfa[i], be = beta[i];
    const double pr = sqrt(plam), qr = sqrt(qlam);
    const double xi = fmax(fmin((pr * lo + qr * up) / (pr + qr), be), al);
    x[i] = xi;
    const double ux1 = up - xi, xl1 = xi - lo;
    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    const double inside = (xi > al && xi < be) ? 1.0 : 0.0;
    const double dL = inside / (2 * plam / (ux2 * ux1) + 2 * qlam / (xl2 * xl1));
    double dh[kMmaMaxM];
    for (int j = 0; j < m; ++j) {
      const double Pj = P[j * n + i], Qj = Q[j * n + i];
      acc[j] += Pj / ux1 + Qj / xl1;
      dh[j] = Pj / ux2 - Qj / xl2;
    }
    int t = m;
    for (int j = 0; j < m; ++j)
      for (int kk = j; kk < m; ++kk) acc[t++] += dh[j] * dL * dh[kk];
  }
  for (int j = 0; j < nv; ++j) {
    const double s = block_total(acc[j], sh);
    if (threadIdx.x == 0) part[blockIdx.x * nv + j] = s;
  }
}

// Change = max |x - xold| / (xmax - xmin) (:309-310)
__global__ void k_max_change(int64_t n, const double *x, const double *xold,
                             const double *xmin, const double *xmax,
                             unsigned long long *out) {
  double mx = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    mx = fmax(mx, fabs((x[i] - xold[i]) / (xmax[i] - xmin[i])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// x < 1e-6 -> 0 (MMA.cpp:166-173), then Change = max |x - xold| / (xmax - xmin)
__global__ void k_oc_finish(int64_t n, double *x, const double *xold,
                            const double *xmin, const double *xmax,
                            unsigned long long *out) {
  double m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v = x[i];
    if (v < 1e-6) {
      v = 0;
      x[i] = 0;
    }
    m = fmax(m, fabs((v - xold[i]) / (xmax[i] - xmin[i])));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace

void launch_filter_rowsum(const Ctx &c, cudaStream_t s) {
  count_launch();
  k_filter_rowsum<<<grid_for(c.ne, 256), 256, 0, s>>>(c.nel[0], c.nel[1],
                                                       c.nel[2], c.taps_d, c.finv);
}

void launch_filter(const Ctx &c, const double *in, double *out, bool transpose,
                   cudaStream_t s) {
  count_launch();
  if (transpose)
    k_filter_adj<<<grid_for(c.ne, 256), 256, 0, s>>>(
        c.nel[0], c.nel[1], c.nel[2], c.taps_d, c.finv, in, 0.0, out);
  else
    k_filter_fwd<<<grid_for(c.ne, 256), 256, 0, s>>>(
        c.nel[0], c.nel[1], c.nel[2], c.taps_d, c.finv, in, out);
}

void launch_filter_adj_uniform(const Ctx &c, double value, double *out,
                               cudaStream_t s) {
  count_launch();
  k_filter_adj<<<grid_for(c.ne, 256), 256, 0, s>>>(
      c.nel[0], c.nel[1], c.nel[2], c.taps_d, c.finv, nullptr, value, out);
}

void launch_simp(const Ctx &c, double penal, double eps, cudaStream_t s) {
  count_launch();
  k_simp<<<grid_for(c.ne, 256), 256, 0, s>>>(c.ne, c.rho, penal, eps, c.E64,
                                              c.dEdz, c.E32, c.Es64, c.dEsdz64);
}

void launch_sensitivity(const Ctx &c, const double *U, double *dc,
                        cudaStream_t s) {
  count_launch();
  k_sensitivity<<<grid_for(c.ne, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                     U, c.dEdz, dc, c.kh64);
}

void launch_oc_clip(int64_t n, double *dfdx, cudaStream_t s) {
  count_launch();
  k_oc_clip<<<grid_for(n, 256), 256, 0, s>>>(n, dfdx);
}

void launch_oc_step(const Ctx &c, int64_t n, double *x, const double *xold,
                    const double *xmin, const double *xmax, const double *dfdx,
                    const double *dgdx, double move, double lmid, double *out,
                    cudaStream_t s) {
  count_launch();
  count_launch();   // k_oc_step + k_sum_parts
  k_oc_step<<<kRedBlocks, 256, 0, s>>>(n, x, xold, xmin, xmax, dfdx, dgdx, move,
                                       lmid, c.part);
  k_sum_parts<<<1, 256, 0, s>>>(kRedBlocks, c.part, out);
}

bool launch_oc_bisect(const Ctx &c, int64_t n, double *x, const double *xold,
                      const double *xmin, const double *xmax, const double *dfdx,
                      const double *dgdx, double move, double g, cudaStream_t s,
                      cudaError_t *err) {
  static int fits[64] = {0};   // 1: kRedBlocks co-resident CTAs fit, -1: not
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!fits[dev]) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oc_bisect, 256, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    fits[dev] = per_sm * sms >= kRedBlocks ? 1 : -1;
  }
  if (fits[dev] < 0) return false;
  count_launch();
  double *part = c.part;   // 2 x kRedBlocks <= kPartCount
  unsigned int *bar = c.gbar;
  double *fault = c.scal + kSlotFault;
  void *args[] = {&n, &x, &xold, &xmin, &xmax, &dfdx, &dgdx, &move, &g, &part, &bar, &fault};
  *err = cudaLaunchCooperativeKernel((const void *)k_oc_bisect, kRedBlocks, 256, args, 0, s);
  return true;
}

void launch_mma_prepare(int64_t n, int m, bool fresh, const MmaConst &k, double *x,
                        double *x1, double *x2, double *low, double *upp,
                        const double *xmin, const double *xmax, const double *dfdx,
                        const double *dgdx, double *alfa, double *beta, double *p0,
                        double *q0, double *P, double *Q, double *part, cudaStream_t s) {
  count_launch();
  k_mma_prepare<<<kRedBlocks, 256, 0, s>>>(n, m, fresh, k, x, x1, x2, low, upp, xmin, xmax,
                                           dfdx, dgdx, alfa, beta, p0, q0, P, Q, part);
}

void launch_mma_dual(int64_t n, int m, const MmaLambda &lam, const double *alfa,
                     const double *beta, const double *low, const double *upp,
                     const double *p0, const double *q0, const double *P, const double *Q,
                     double *x, double *part, cudaStream_t s) {
  count_launch();
  k_mma_dual<<<kRedBlocks, 256, 0, s>>>(n, m, lam, alfa, beta, low, upp, p0, q0, P, Q, x,
                                        part);
}

void launch_max_change(int64_t n, const double *x, const double *xold, const double *xmin,
                       const double *xmax, double *out, cudaStream_t s) {
  count_launch();
  cudaMemsetAsync(out, 0, sizeof(double), s);
  k_max_change<<<grid_for(n, 256), 256, 0, s>>>(n, x, xold, xmin, xmax,
                                                reinterpret_cast<unsigned long long *>(out));
}

void launch_oc_finish(const Ctx &c, int64_t n, double *x, const double *xold,
                      const double *xmin, const double *xmax, double *out,
                      cudaStream_t s) {
  count_launch();
  (void)c;
  cudaMemsetAsync(out, 0, sizeof(double), s);
  k_oc_finish<<<grid_for(n, 256), 256, 0, s>>>(
      n, x, xold, xmin, xmax, reinterpret_cast<unsigned long long *>(out));
}

}  // namespace tpo
