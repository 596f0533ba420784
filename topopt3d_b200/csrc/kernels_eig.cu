// Tall-skinny block kernels of the block eigensolver (eigen.cu): the Gram
// blocks of the Rayleigh-Ritz step, the recombination of the basis by the
// Ritz coefficients, and the residual block with its column norms.  The
// reference forms the same products with VecMDot/VecMAXPY over its search
// space (PRINVIT.cpp:319-330).
//
// Every kernel reads each n-row column it needs once per launch; reductions
// over rows go through per-CTA partial sums that a second launch adds in a
// fixed order, so the results do not depend on scheduling.
#include "tpo_internal.h"

namespace tpo {

namespace {

constexpr int kGI = 36;   // Gram super-tile: left columns
constexpr int kGJ = 72;   //                 right columns (A then B images)
constexpr int kGR = 32;   // rows staged per chunk
constexpr int kGramThreads = 256;
constexpr int kGramParts = 296;   // row-chunk CTAs per super-tile

__global__ void __launch_bounds__(kGramThreads)
    k_eig_gram(int64_t n, int m, int k, EigCols cols, double *part) {
  __shared__ __align__(16) double Ls[kGR][kGI];
  __shared__ __align__(16) double Rs[kGR][kGJ];
  const int nsi = (k + kGI - 1) / kGI;
  const int st = blockIdx.y;
  const int i0 = (st % nsi) * kGI, j0 = (st / nsi) * kGJ;
  const int t = threadIdx.x;
  constexpr int kTiles = (kGI / 4) * (kGJ / 4);   // 162 threads hold 4 x 4
  const bool act = t < kTiles;
  const int ig = t / (kGJ / 4), jg = t % (kGJ / 4);
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int64_t r0 = (int64_t)blockIdx.x * kGR; r0 < n; r0 += (int64_t)gridDim.x * kGR) {
    __syncthreads();
    for (int e = t; e < kGR * (kGI + kGJ); e += kGramThreads) {
      const int r = e % kGR, col = e / kGR;   // a warp reads 32 rows of a column
      const int64_t row = r0 + r;
      double v = 0.0;
      if (row < n) {
        if (col < kGI) {
          const int i = i0 + col;
          if (i < k) v = cols.L[i / m][(int64_t)(i % m) * n + row];
        } else {
          const int j = j0 + col - kGI;
          if (j < k)
            v = cols.A[j / m][(int64_t)(j % m) * n + row];
          else if (j < 2 * k)
            v = cols.B[(j - k) / m][(int64_t)((j - k) % m) * n + row];
        }
      }
      if (col < kGI)
        Ls[r][col] = v;
      else
        Rs[r][col - kGI] = v;
    }
    __syncthreads();
    if (act) {
#pragma unroll 4
      for (int r = 0; r < kGR; ++r) {
        const double2 a01 = *reinterpret_cast<const double2 *>(&Ls[r][ig * 4]);
        const double2 a23 = *reinterpret_cast<const double2 *>(&Ls[r][ig * 4 + 2]);
        const double2 b01 = *reinterpret_cast<const double2 *>(&Rs[r][jg * 4]);
        const double2 b23 = *reinterpret_cast<const double2 *>(&Rs[r][jg * 4 + 2]);
        const double av[4] = {a01.x, a01.y, a23.x, a23.y};
        const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
      }
    }
  }
  if (act) {
    double *p = part + ((size_t)st * gridDim.x + blockIdx.x) * (kGI * kGJ);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) p[(ig * 4 + a) * kGJ + jg * 4 + b] = acc[a][b];
  }
}

// H (k x k) and G (k x k), column-major, from the partials in CTA order
__global__ void k_eig_gram_reduce(int k, int nsi, int nst, int nparts, const double *part,
                                  double *H, double *G) {
  const int64_t total = (int64_t)nst * kGI * kGJ;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int st = (int)(q / (kGI * kGJ)), w = (int)(q % (kGI * kGJ));
    const int i = (st % nsi) * kGI + w / kGJ, j = (st / nsi) * kGJ + w % kGJ;
    if (i >= k || j >= 2 * k) continue;
    const double *p = part + (size_t)st * nparts * (kGI * kGJ) + w;
    double s = 0.0;
    for (int c = 0; c < nparts; ++c) s += p[(size_t)c * (kGI * kGJ)];
    if (j < k)
      H[(size_t)j * k + i] = s;
    else
      G[(size_t)(j - k) * k + i] = s;
  }
}

// one thread per (row, image group): out.X[g] = [V_0 .. V_nb-1] C and,
// with P, out.P[g] = [V_1 .. V_nb-1] C(m:, :), C (k x m) column-major
template <int MB>
__global__ void __launch_bounds__(128)
    k_eig_combine(int64_t n, int m, int k, EigCols cols, const double *__restrict__ C,
                  EigOut out, int want_p) {
  __shared__ double Cs[3 * kMaxEigPairs * MB];   // Cs[i * MB + j] = C(i, j)
  for (int e = threadIdx.x; e < k * MB; e += blockDim.x) {
    const int i = e / MB, j = e % MB;
    Cs[e] = j < m ? C[(size_t)j * k + i] : 0.0;
  }
  __syncthreads();
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3 * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(t / n);
    const int64_t row = t - (int64_t)g * n;
    double ax[MB], ap[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) ax[j] = ap[j] = 0.0;
    for (int i = 0; i < k; ++i) {
      const int b = i / m;
      const double *src = g == 0 ? cols.L[b] : (g == 1 ? cols.A[b] : cols.B[b]);
      const double x = src[(int64_t)(i % m) * n + row];
      const double *c = Cs + i * MB;
      if (i < m) {
#pragma unroll
        for (int j = 0; j < MB; ++j) ax[j] = fma(x, c[j], ax[j]);
      } else {
#pragma unroll
        for (int j = 0; j < MB; ++j) {
          ax[j] = fma(x, c[j], ax[j]);
          ap[j] = fma(x, c[j], ap[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MB; ++j) {
      if (j >= m) break;
      out.X[g][(int64_t)j * n + row] = ax[j];
      if (want_p) out.P[g][(int64_t)j * n + row] = ap[j];
    }
  }
}

// R[:, j] = AX[:, j] - theta_j BX[:, j], and per CTA the sums of R[:, j]^2
// (part[cta * 2m + j]) and BX[:, j]^2 (part[cta * 2m + m + j])
constexpr int kNormThreads = 256;
constexpr int kNormParts = 296;

__global__ void __launch_bounds__(kNormThreads)
    k_eig_resid_norms(int64_t n, int m, const double *__restrict__ AX,
                      const double *__restrict__ BX, EigTheta th, double *R, double *part) {
  __shared__ double red[kNormThreads / 32][2 * kMaxEigPairs];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  for (int j = 0; j < m; ++j) {
    double sr = 0.0, sb = 0.0;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
         row += (int64_t)gridDim.x * blockDim.x) {
      const double bx = BX[(int64_t)j * n + row];
      const double r = AX[(int64_t)j * n + row] - th.v[j] * bx;
      R[(int64_t)j * n + row] = r;
      sr = fma(r, r, sr);
      sb = fma(bx, bx, sb);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, o);
      sb += __shfl_down_sync(0xffffffffu, sb, o);
    }
    if (lane == 0) {
      red[warp][j] = sr;
      red[warp][m + j] = sb;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 2 * m; q += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kNormThreads / 32; ++w) s += red[w][q];
    part[(size_t)blockIdx.x * 2 * m + q] = s;
  }
}

// nrm[q] = sqrt(sum over the CTAs of part[cta * 2m + q]), q < 2m
__global__ void k_eig_norms_reduce(int m, int nparts, const double *part, double *nrm) {
  for (int q = threadIdx.x; q < 2 * m; q += blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nparts; ++c) s += part[(size_t)c * 2 * m + q];
    nrm[q] = sqrt(s);
  }
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

size_t eig_gram_scratch(int k) {
  const int nsi = (k + kGI - 1) / kGI, nsj = (2 * k + kGJ - 1) / kGJ;
  const size_t gram = (size_t)nsi * nsj * kGramParts * kGI * kGJ;
  const size_t norms = (size_t)kNormParts * 2 * kMaxEigPairs;
  return gram > norms ? gram : norms;
}

void launch_eig_gram(int64_t n, int m, int nblk, const EigCols &cols, double *part, double *H,
                     double *G, cudaStream_t s) {
  const int k = nblk * m;
  const int nsi = (k + kGI - 1) / kGI, nsj = (2 * k + kGJ - 1) / kGJ;
  count_launch(2);
  k_eig_gram<<<dim3(kGramParts, nsi * nsj), kGramThreads, 0, s>>>(n, m, k, cols, part);
  k_eig_gram_reduce<<<grid_for((int64_t)nsi * nsj * kGI * kGJ, 256), 256, 0, s>>>(
      k, nsi, nsi * nsj, kGramParts, part, H, G);
}

void launch_eig_combine(int64_t n, int m, int nblk, const EigCols &cols, const double *C,
                        const EigOut &out, bool want_p, cudaStream_t s) {
  const int k = nblk * m;
  const int g = grid_for(3 * n, 128);
  count_launch();
  if (m <= 4)
    k_eig_combine<4><<<g, 128, 0, s>>>(n, m, k, cols, C, out, want_p);
  else if (m <= 8)
    k_eig_combine<8><<<g, 128, 0, s>>>(n, m, k, cols, C, out, want_p);
  else if (m <= 12)
    k_eig_combine<12><<<g, 128, 0, s>>>(n, m, k, cols, C, out, want_p);
  else if (m <= 16)
    k_eig_combine<16><<<g, 128, 0, s>>>(n, m, k, cols, C, out, want_p);
  else
    k_eig_combine<32><<<g, 128, 0, s>>>(n, m, k, cols, C, out, want_p);
}

void launch_eig_resid_norms(int64_t n, int m, const double *AX, const double *BX,
                            const EigTheta &th, double *R, double *part, double *nrm,
                            cudaStream_t s) {
  count_launch(2);
  k_eig_resid_norms<<<kNormParts, kNormThreads, 0, s>>>(n, m, AX, BX, th, R, part);
  k_eig_norms_reduce<<<1, 64, 0, s>>>(m, kNormParts, part, nrm);
}

}  // namespace tpo
