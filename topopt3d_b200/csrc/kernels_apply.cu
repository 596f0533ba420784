// Set-up companions of the fine-level operator: the Jacobi diagonal and the
// assembled 27-point stencil used only to form the Galerkin coarse
// operators.  The matrix-free apply itself is in kernels_apply_staged.cu.
#include "modal.cuh"

namespace tpo {

namespace {

// Jacobi diagonal of the fine operator: sum_e E_e K0_ii, identity on fixed
// dofs, non-positive diagonals set to 1 (FEAnalysis.cpp:476-484)
__global__ void k_fine_diag(int nelx, int nely, int nelz,
                            const double *__restrict__ E,
                            const uint8_t *__restrict__ fix,
                            const K0Diag<double> kd, double *dinv64,
                            float *dinv32) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = n % Nx, j = (n / Nx) % Ny, k = n / ((int64_t)Nx * Ny);
    double d[3] = {0, 0, 0};
    for (int bz = 0; bz < 2; ++bz)
      for (int by = 0; by < 2; ++by)
        for (int bx = 0; bx < 2; ++bx) {
          const int ei = i - 1 + bx, ej = j - 1 + by, ek = k - 1 + bz;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
            continue;
          // node n is corner (1-bx, 1-by, 1-bz) of that element
          const int l = (1 - bx) + 2 * (1 - by) + 4 * (1 - bz);
          const double Ee = E[((int64_t)ek * nely + ej) * nelx + ei];
          for (int c = 0; c < 3; ++c) d[c] += Ee * kd.v[3 * l + c];
        }
    const uint8_t f = fix[n];
    for (int c = 0; c < 3; ++c) {
      double v = ((f >> c) & 1) ? 1.0 : d[c];
      if (!(v > 0)) v = 1.0;
      dinv64[3 * n + c] = 1.0 / v;
      dinv32[3 * n + c] = static_cast<float>(1.0 / v);
    }
  }
}

// Fine-level operator assembled as a 27-point 3x3-block stencil (only used
// to form the Galerkin coarse operators).  Block (n, m) sums E_e K0 over the
// elements containing both nodes in increasing element order, as the
// ADD_VALUES assembly does (FEAnalysis.cpp:448-464); fixed rows/columns are
// then zeroed with a unit diagonal.
__global__ void k_fine_stencil(int nelx, int nely, int nelz,
                               const double *__restrict__ E,
                               const uint8_t *__restrict__ fix,
                               const double *__restrict__ K0lex, double *S) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz;
  const int64_t total = nn * 27;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int nb = (int)(t / nn);
    const int64_t n = t - (int64_t)nb * nn;
    const int di = nb % 3 - 1, dj = (nb / 3) % 3 - 1, dk = nb / 9 - 1;
    const int i = n % Nx, j = (n / Nx) % Ny, k = n / ((int64_t)Nx * Ny);
    const int mi = i + di, mj = j + dj, mk = k + dk;
    double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const bool inside = mi >= 0 && mi < Nx && mj >= 0 && mj < Ny && mk >= 0 && mk < Nz;
    if (inside) {
      for (int ek = max(k, mk) - 1; ek <= min(k, mk); ++ek)
        for (int ej = max(j, mj) - 1; ej <= min(j, mj); ++ej)
          for (int ei = max(i, mi) - 1; ei <= min(i, mi); ++ei) {
            if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
              continue;
            const double Ee = E[((int64_t)ek * nely + ej) * nelx + ei];
            const int ln = (i - ei) + 2 * (j - ej) + 4 * (k - ek);
            const int lm = (mi - ei) + 2 * (mj - ej) + 4 * (mk - ek);
            for (int r = 0; r < 3; ++r)
              for (int s = 0; s < 3; ++s)
                blk[3 * r + s] += Ee * K0lex[24 * (3 * ln + r) + 3 * lm + s];
          }
      const int64_t m = (int64_t)mk * Nx * Ny + (int64_t)mj * Nx + mi;
      const uint8_t fn = fix[n], fm = fix[m];
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s)
          if (((fn >> r) & 1) || ((fm >> s) & 1))
            blk[3 * r + s] = (nb == 13 && r == s) ? 1.0 : 0.0;
      if (nb == 13)
        for (int r = 0; r < 3; ++r)
          if (!(blk[4 * r] > 0)) blk[4 * r] = 1.0;
    }
    for (int q = 0; q < 9; ++q) S[(int64_t)(nb * 9 + q) * nn + n] = blk[q];
  }
}

// Identity-row mask of the fine operator: bit c of node n is set when dof
// (n, c) has an identity row and column -- fixed (MatZeroRowsColumns,
// FEAnalysis.cpp:473) or with an assembled diagonal <= 0, which the
// reference replaces by 1 (:476-484).  Such a diagonal means E = 0 on every
// element around the node, so the row and column are zero apart from it.
// A NaN diagonal is left alone: the reference sets it to 1 but keeps the
// NaN off-diagonals, so the solve fails there as here.
__global__ void k_identity_mask(int nelx, int nely, int nelz,
                                const double *__restrict__ E,
                                const uint8_t *__restrict__ fix,
                                const K0Diag<double> kd, uint8_t *idm) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = n % Nx, j = (n / Nx) % Ny, k = n / ((int64_t)Nx * Ny);
    double d[3] = {0, 0, 0};
    for (int bz = 0; bz < 2; ++bz)
      for (int by = 0; by < 2; ++by)
        for (int bx = 0; bx < 2; ++bx) {
          const int ei = i - 1 + bx, ej = j - 1 + by, ek = k - 1 + bz;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
            continue;
          const int l = (1 - bx) + 2 * (1 - by) + 4 * (1 - bz);
          const double Ee = E[((int64_t)ek * nely + ej) * nelx + ei];
          for (int c = 0; c < 3; ++c) d[c] += Ee * kd.v[3 * l + c];
        }
    unsigned m = fix[n];
    for (int c = 0; c < 3; ++c)
      if (d[c] <= 0) m |= 1u << c;
    idm[n] = (uint8_t)m;
  }
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

void launch_fine_diag(const Ctx &c, double *dinv64, float *dinv32,
                      cudaStream_t s) {
  count_launch();
  k_fine_diag<<<grid_for(c.nn, 256), 256, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                   c.E64, c.fix, c.kd64, dinv64,
                                                   dinv32);
}

void launch_identity_mask(const Ctx &c, cudaStream_t s) {
  count_launch();
  k_identity_mask<<<grid_for(c.nn, 256), 256, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                       c.E64, c.fix, c.kd64, c.idm);
}

void launch_fine_stencil(const Ctx &c, double *S, cudaStream_t s) {
  count_launch();
  k_fine_stencil<<<grid_for(c.nn * 27, 256), 256, 0, s>>>(
      c.nel[0], c.nel[1], c.nel[2], c.E64, c.fix, c.K0lex, S);
}
}  // namespace tpo
