// Design-side kernels: the density filter (forward and transpose, matrix
// free), SIMP interpolation, the compliance sensitivity, the OC update and
// the MMA update.
#include <algorithm>
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

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
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

// ---- MMA for m >= 2 constraints (MMA::MMAsub, MMA.cpp:185-343, with
// MMA::DualSolve, :353-595), the whole update in one cooperative launch.
//
// Phase 0 (MMAsub, :219-307) forms the asymptotes, the move limits
// alfa/beta, p0, q0, P, Q and the partials of b, and shifts xold2 <- xold1
// <- x.  Each later phase evaluates x(lambda) (XYZofLam, :432-447) with the
// partials of the dual gradient sums sum_n P_j/ux1 + Q_j/xl1 (DualGrad,
// :461-474) and of the Hessian sums sum_n dhdx_j dLdxx dhdx_k, k >= j
// (DualHess, :489-515).  After the grid barrier that closes a phase every
// block sums the partials in the same fixed order, and thread 0 of every
// block runs the same scalar Newton logic on the same numbers (residual,
// SearchDir with partial pivoting, SearchDis, the epsilon schedule), so all
// blocks agree on the next lambda without a second barrier.  The partials
// are double-buffered by phase parity (a block writes phase p + 1's only
// after the barrier that every block passes once it has read phase p's).
// Element i is handled by the same thread in every phase, so x, xold1 and
// the scratch need no exchange between threads.  Change (:309-310) is a
// max over blocks by an atomic on the order-preserving bit pattern of
// non-negative doubles.
template <int M>
struct MmaDims {
  static constexpr int NH = M * (M + 1) / 2, NV = M + NH;
};

// all threads: s_tot[j] = sum_b buf[j * G + b], j < CNT, in a fixed order
// (thread t sums b = t, t + 256, ...; then the block reduction of
// mma_store_parts), read past L1 since other blocks wrote buf
template <int CNT>
__device__ __forceinline__ void mma_sum_parts(const double *buf, int G, double *s_tot,
                                              double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double v[CNT];
#pragma unroll
  for (int j = 0; j < CNT; ++j) v[j] = 0.0;
  for (int b = threadIdx.x; b < G; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < CNT; ++j) v[j] += __ldcg(buf + (size_t)j * G + b);
#pragma unroll
  for (int j = 0; j < CNT; ++j) {
    const double t = warp_sum(v[j]);
    if (lane == 0) sh[j * 32 + w] = t;
  }
  __syncthreads();
  for (int j = w; j < CNT; j += nw) {
    double t = lane < nw ? sh[j * 32 + lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) s_tot[j] = t;
  }
  __syncthreads();
}

// all threads: buf[j * G + blockIdx.x] = block sum of v[j], j < cnt
template <int CNT>
__device__ __forceinline__ void mma_store_parts(const double *v, double *buf, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < CNT; ++j) {
    const double t = warp_sum(v[j]);
    if (lane == 0) sh[j * 32 + w] = t;
  }
  __syncthreads();
  for (int j = w; j < CNT; j += nw) {
    double t = lane < nw ? sh[j * 32 + lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) buf[(size_t)j * gridDim.x + blockIdx.x] = t;
  }
}

// x = A^-1 r for the m x m row-major A by Gaussian elimination with
// partial pivoting; false on a zero pivot
template <int M>
__device__ bool mma_solve_small(double (&A)[M * M], double (&r)[M], double (&x)[M]) {
  for (int k = 0; k < M; ++k) {
    int p = k;
    for (int i = k + 1; i < M; ++i)
      if (fabs(A[i * M + k]) > fabs(A[p * M + k])) p = i;
    if (A[p * M + k] == 0.0) return false;
    if (p != k) {
      for (int c = 0; c < M; ++c) {
        const double t = A[k * M + c];
        A[k * M + c] = A[p * M + c];
        A[p * M + c] = t;
      }
      const double t = r[k];
      r[k] = r[p];
      r[p] = t;
    }
    for (int i = k + 1; i < M; ++i) {
      const double f = A[i * M + k] / A[k * M + k];
      for (int c = k; c < M; ++c) A[i * M + c] -= f * A[k * M + c];
      r[i] -= f * r[k];
    }
  }
  for (int k = M - 1; k >= 0; --k) {
    double s = r[k];
    for (int c = k + 1; c < M; ++c) s -= A[k * M + c] * x[c];
    x[k] = s / A[k * M + k];
  }
  return true;
}

template <int M>
__global__ void __launch_bounds__(256) k_mma_solve(MmaSolveArgs a) {
  constexpr int NV = MmaDims<M>::NV;
  __shared__ double sh[NV * 32];
  __shared__ double s_tot[NV];
  __shared__ double s_lam[M];
  __shared__ int s_done;
  const int G = gridDim.x;
  const int64_t n = a.n;
  const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t di = (int64_t)G * blockDim.x;
  int phase = 0;

  // ---- phase 0: MMAsub's element pass (:219-307)
  {
    double bs[M];
#pragma unroll
    for (int j = 0; j < M; ++j) bs[j] = 0.0;
    for (int64_t i = i0; i < n; i += di) {
      const double xi = a.x[i], span = a.xmax[i] - a.xmin[i];
      double lo, up;
      if (a.fresh) {
        lo = xi - a.k.asyinit * span;
        up = xi + a.k.asyinit * span;
      } else {
        const double xa = a.x1[i], xb = a.x2[i];
        const double zz = (xi - xa) * (xa - xb);
        const double f = zz > 0 ? a.k.asyincr : (zz < 0 ? a.k.asydecr : 1.0);
        lo = xi - f * (xa - a.low[i]);
        up = xi + f * (a.upp[i] - xa);
        lo = fmin(fmax(lo, xi - 10 * span), xi - 0.01 * span);
        up = fmax(fmin(up, xi + 10 * span), xi + 0.01 * span);
      }
      a.alfa[i] = fmax(fmax(lo + a.k.albefa * (xi - lo), xi - a.k.move * span), a.xmin[i]);
      a.beta[i] = fmin(fmin(up - a.k.albefa * (up - xi), xi + a.k.move * span), a.xmax[i]);
      const double xmami = fmax(up - lo, 1e-5);
      const double ux1 = up - xi, xl1 = xi - lo, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
      const double df = a.dfdx[i];
      const double pp = fmax(df, 0.0), qq = fmax(-df, 0.0);
      const double pq0 = 0.001 * (pp + qq) + 0.5 * a.k.raa0 / xmami;
      a.p0[i] = (pp + pq0) * ux2;
      a.q0[i] = (qq + pq0) * xl2;
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const double dg = a.dgdx[j * n + i];
        const double Pj = fmax(dg, 0.0) * ux2, Qj = fmax(-dg, 0.0) * xl2;
        a.P[j * n + i] = Pj;
        a.Q[j * n + i] = Qj;
        bs[j] += Pj / ux1 + Qj / xl1;
      }
      a.low[i] = lo;
      a.upp[i] = up;
      a.x2[i] = a.x1[i];
      a.x1[i] = xi;
    }
    double *buf = a.part + (size_t)(phase & 1) * NV * G;
    mma_store_parts<M>(bs, buf, sh);
    if (!grid_barrier(a.bar, a.fault)) return;
    mma_sum_parts<M>(buf, G, s_tot, sh);
    ++phase;
  }

  // ---- DualSolve (:353-405); the scalar state lives in thread 0
  double lam[M], eta[M], b[M];
  double epsi = 1.0;
  int it = 0, steps = 0, status = 0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < M; ++j) {
      b[j] = s_tot[j] - a.g[j];
      lam[j] = 500.0;
      eta[j] = 1.0;
      s_lam[j] = lam[j];
    }
  }
  __syncthreads();
  for (;;) {
    double lr[M], acc[NV];
#pragma unroll
    for (int j = 0; j < M; ++j) lr[j] = s_lam[j];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0.0;
    for (int64_t i = i0; i < n; i += di) {
      double plam = a.p0[i], qlam = a.q0[i];
      double Pj[M], Qj[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        Pj[j] = a.P[j * n + i];
        Qj[j] = a.Q[j * n + i];
        plam += Pj[j] * lr[j];
        qlam += Qj[j] * lr[j];
      }
      const double lo = a.low[i], up = a.upp[i], al = a.alfa[i], be = a.beta[i];
      const double pr = sqrt(plam), qr = sqrt(qlam);
      const double xi = fmax(fmin((pr * lo + qr * up) / (pr + qr), be), al);
      a.x[i] = xi;
      // 1/(U - x) and 1/(x - L) once; the sums and dLdxx from products
      const double iu = 1.0 / (up - xi), il = 1.0 / (xi - lo);
      const double iu2 = iu * iu, il2 = il * il;
      const double inside = (xi > al && xi < be) ? 1.0 : 0.0;
      const double dL = inside / (2 * plam * (iu2 * iu) + 2 * qlam * (il2 * il));
      double dh[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        acc[j] += Pj[j] * iu + Qj[j] * il;
        dh[j] = Pj[j] * iu2 - Qj[j] * il2;
      }
      int t = M;
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int kk = j; kk < M; ++kk) acc[t++] += dh[j] * dL * dh[kk];
    }
    double *buf = a.part + (size_t)(phase & 1) * NV * G;
    mma_store_parts<NV>(acc, buf, sh);
    if (!grid_barrier(a.bar, a.fault)) return;
    mma_sum_parts<NV>(buf, G, s_tot, sh);
    ++phase;
    if (threadIdx.x == 0) {
      // y, z (XYZofLam) and the gradient (DualGrad) at lambda; Set_m's
      // constants a0 = b0 = 1, a = 0, c = 1000, d = 1 (:40-52)
      double Gd[M];
#pragma unroll
      for (int j = 0; j < M; ++j) Gd[j] = s_tot[j] - (b[j] + fmax(lam[j] - 1000.0, 0.0));
      int done = 0;
      for (;;) {
        double rmax = 0.0;    // DualResidual (:417-427), infinity norm
#pragma unroll
        for (int j = 0; j < M; ++j) {
          rmax = fmax(rmax, fabs(Gd[j] + eta[j]));
          rmax = fmax(rmax, fabs(eta[j] * lam[j] - epsi));
        }
        if (rmax > 0.9 * epsi && it < 100) {
          // DualHess (:507-515) and SearchDir (:532-544)
          double A[M * M], r[M], dl[M], de[M];
          int t = M;
#pragma unroll
          for (int j = 0; j < M; ++j)
#pragma unroll
            for (int kk = j; kk < M; ++kk) {
              A[j * M + kk] = A[kk * M + j] = -s_tot[t];
              ++t;
            }
          double tr = 0.0;
#pragma unroll
          for (int j = 0; j < M; ++j) {
            if (lam[j] > 1000.0) A[j * M + j] -= 1.0;
            A[j * M + j] -= eta[j] / lam[j];
            tr += A[j * M + j];
          }
          const double shift = fmin(1e-4 * tr / M, -1e-7);
#pragma unroll
          for (int j = 0; j < M; ++j) {
            A[j * M + j] += shift;
            r[j] = -Gd[j] - epsi / lam[j];
          }
          if (!mma_solve_small<M>(A, r, dl)) {
            status = 1;
            done = 1;
            break;
          }
          double theta = 1.0;   // SearchDis (:559-575)
#pragma unroll
          for (int j = 0; j < M; ++j) {
            de[j] = -eta[j] + epsi / lam[j] - dl[j] * (eta[j] / lam[j]);
            const double r1 = -0.99 * lam[j] / dl[j], r2 = -0.99 * eta[j] / de[j];
            if (r1 >= 0) theta = fmin(theta, r1);
            if (r2 >= 0) theta = fmin(theta, r2);
          }
#pragma unroll
          for (int j = 0; j < M; ++j) {
            lam[j] += theta * dl[j];
            eta[j] += theta * de[j];
          }
          ++it;
          ++steps;
          break;
        }
        epsi *= 0.1;
        it = 0;
        if (!(epsi > a.epsimin)) {
          done = 1;
          break;
        }
      }
      s_done = done;
#pragma unroll
      for (int j = 0; j < M; ++j) s_lam[j] = lam[j];
    }
    __syncthreads();
    if (s_done) break;
  }

  // ---- Change (:309-310)
  double mx = 0.0;
  for (int64_t i = i0; i < n; i += di)
    mx = fmax(mx, fabs((a.x[i] - a.x1[i]) / (a.xmax[i] - a.xmin[i])));
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0)
    atomicMax(reinterpret_cast<unsigned long long *>(a.out),
              (unsigned long long)__double_as_longlong(mx));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out[1] = steps;
    a.out[2] = status;
  }
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

template <int M>
bool launch_mma_solve_m(MmaSolveArgs &a, cudaStream_t s, cudaError_t *err) {
  static int cap[64] = {0}, sms[64] = {0};   // co-resident blocks, SMs, per device
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!cap[dev]) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mma_solve<M>, 256, 0);
    cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
    cap[dev] = per_sm * sms[dev] > 0 ? std::min(per_sm * sms[dev], kRedBlocks) : -1;
  }
  if (cap[dev] < 0) return false;
  // about 4 elements per thread, at least one block per SM: every Newton
  // step ends in a grid barrier and a sum over the blocks' partials, so
  // small meshes run best on few blocks
  const int64_t want = std::max<int64_t>(sms[dev], (a.n + 1023) / 1024);
  const int grid = (int)std::min<int64_t>(want, cap[dev]);
  count_launch();
  *err = cudaMemsetAsync(a.out, 0, sizeof(double), s);
  if (*err != cudaSuccess) return true;
  void *args[] = {&a};
  *err = cudaLaunchCooperativeKernel((const void *)k_mma_solve<M>, grid, 256, args, 0, s);
  return true;
}

bool launch_mma_solve(MmaSolveArgs &a, cudaStream_t s, cudaError_t *err) {
  switch (a.m) {
    case 1: return launch_mma_solve_m<1>(a, s, err);
    case 2: return launch_mma_solve_m<2>(a, s, err);
    case 3: return launch_mma_solve_m<3>(a, s, err);
    case 4: return launch_mma_solve_m<4>(a, s, err);
    case 5: return launch_mma_solve_m<5>(a, s, err);
    case 6: return launch_mma_solve_m<6>(a, s, err);
    case 7: return launch_mma_solve_m<7>(a, s, err);
    case 8: return launch_mma_solve_m<8>(a, s, err);
    default: return false;
  }
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
