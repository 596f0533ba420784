// Stress stiffness Ks for linear buckling (Stability::StressFnc,
// Buckling.cpp:291-361): Ks = sum_e -Es_e ks_e(U) with
//   ks_e = sum_q W_q G_q^T sigtos(D B_q u_e) G_q detJ,
// G_q the displacement-gradient operator (FEAnalysis.cpp:1062-1081) and
// sigtos the 3x3 stress tensor repeated for each displacement component
// (Buckling.cpp:371-414), and the Dirichlet rows/columns zeroed with a zero
// diagonal (Buckling.cpp:29-30).
//
// Because sigtos repeats the same tensor for the three components, ks_e is
// H_e (x) I_3 with the 8x8 scalar matrix
//   H_e[l][m] = detJ sum_q grad N_l(q)^T sigma_q grad N_m(q),
// so Ks is a 27-point SCALAR stencil per node (one weight per neighbour,
// shared by the components): 27 values per node instead of 243.
//
//   k_ks_element  one thread per element: sigma at the 8 Gauss points,
//                 -Es_e H_e (upper triangle, 36 values) to a scratch array
//   k_ks_gather   one thread per node: the 27 stencil weights, summed over
//                 the (up to 8) elements around the node in a fixed order
//   k_ks_apply    y = Ks u for NB columns, fixed components masked on both
//                 sides
#include "tpo_internal.h"

namespace tpo {

namespace {

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

__device__ __forceinline__ int tri(int l, int m) {   // upper-triangle index
  const int a = l < m ? l : m, b = l < m ? m : l;
  return a * 8 - a * (a - 1) / 2 + (b - a);
}

__global__ void k_ks_element(int nelx, int nely, int nelz,
                             const double *__restrict__ U,
                             const double *__restrict__ Es, KsConst kc,
                             double *__restrict__ Hs) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nelx), j = (int)((e / nelx) % nely),
              k = (int)(e / ((int64_t)nelx * nely));
    const int64_t n0 = ((int64_t)k * Ny + j) * Nx + i;
    double u[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int64_t n = n0 + (l & 1) + ((l >> 1) & 1) * Nx + ((l >> 2) & 1) * (int64_t)Nx * Ny;
#pragma unroll
      for (int c = 0; c < 3; ++c) u[l][c] = U[3 * n + c];
    }
    double H[36];
#pragma unroll
    for (int t = 0; t < 36; ++t) H[t] = 0.0;
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      // displacement gradient F[c][a] = d u_c / d x_a
      double F[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
#pragma unroll
          for (int l = 0; l < 8; ++l) s += kc.g[q][a][l] * u[l][c];
          F[c][a] = s;
        }
      // Voigt strain [xx, yy, zz, xy, yz, xz] (engineering shear) and
      // sigma = D eps (RecMesh.cpp:453-462)
      const double exx = F[0][0], eyy = F[1][1], ezz = F[2][2];
      const double gxy = F[0][1] + F[1][0], gyz = F[1][2] + F[2][1],
                   gxz = F[0][2] + F[2][0];
      const double sxx = kc.t1 * exx + kc.t3 * (eyy + ezz);
      const double syy = kc.t1 * eyy + kc.t3 * (exx + ezz);
      const double szz = kc.t1 * ezz + kc.t3 * (exx + eyy);
      const double sxy = kc.t2 * gxy, syz = kc.t2 * gyz, sxz = kc.t2 * gxz;
      const double S[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
      // t[a][m] = sum_b S[a][b] g[b][m]
      double t[3][8];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int m = 0; m < 8; ++m)
          t[a][m] = S[a][0] * kc.g[q][0][m] + S[a][1] * kc.g[q][1][m] +
                    S[a][2] * kc.g[q][2][m];
#pragma unroll
      for (int l = 0; l < 8; ++l)
#pragma unroll
        for (int m = l; m < 8; ++m)
          H[tri(l, m)] += kc.g[q][0][l] * t[0][m] + kc.g[q][1][l] * t[1][m] +
                          kc.g[q][2][l] * t[2][m];
    }
    const double w = -Es[e] * kc.detJ;
#pragma unroll
    for (int t = 0; t < 36; ++t) Hs[(int64_t)t * ne + e] = w * H[t];
  }
}

__global__ void k_ks_gather(int nelx, int nely, int nelz,
                            const double *__restrict__ Hs,
                            double *__restrict__ S) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz, ne = (int64_t)nelx * nely * nelz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % Nx), j = (int)((n / Nx) % Ny), k = (int)(n / ((int64_t)Nx * Ny));
    double acc[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) acc[d] = 0.0;
    // element (i-1+a, j-1+b, k-1+c): node n is its corner (1-a, 1-b, 1-c)
#pragma unroll
    for (int cz = 0; cz < 2; ++cz)
#pragma unroll
      for (int cy = 0; cy < 2; ++cy)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int ei = i - 1 + cx, ej = j - 1 + cy, ek = k - 1 + cz;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
            continue;
          const int64_t e = ((int64_t)ek * nely + ej) * nelx + ei;
          const int ln = (1 - cx) + 2 * (1 - cy) + 4 * (1 - cz);
#pragma unroll
          for (int lm = 0; lm < 8; ++lm) {
            // offset of corner lm from node n
            const int dx = (lm & 1) - (1 - cx), dy = ((lm >> 1) & 1) - (1 - cy),
                      dz = ((lm >> 2) & 1) - (1 - cz);
            const int d = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
            acc[d] += Hs[(int64_t)tri(ln, lm) * ne + e];
          }
        }
#pragma unroll
    for (int d = 0; d < 27; ++d) S[(int64_t)d * nn + n] = acc[d];
  }
}

template <int NB>
__global__ void k_ks_apply(int nx, int ny, int nz, const double *__restrict__ S,
                           const uint8_t *__restrict__ fix,
                           const double *__restrict__ u, double *__restrict__ y,
                           int64_t ld) {
  const int64_t nn = (int64_t)nx * ny * nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / ((int64_t)nx * ny));
    double acc[NB][3];
#pragma unroll
    for (int c = 0; c < NB; ++c) acc[c][0] = acc[c][1] = acc[c][2] = 0.0;
#pragma unroll
    for (int d = 0; d < 27; ++d) {
      const int mi = min(max(i + d % 3 - 1, 0), nx - 1);
      const int mj = min(max(j + (d / 3) % 3 - 1, 0), ny - 1);
      const int mk = min(max(k + d / 9 - 1, 0), nz - 1);
      const int64_t m = ((int64_t)mk * ny + mj) * nx + mi;
      const double w = S[(int64_t)d * nn + n];   // 0 outside the mesh
      const unsigned fm = fix[m];
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        const double *uc = u + c * ld + 3 * m;
#pragma unroll
        for (int q = 0; q < 3; ++q)
          if (!((fm >> q) & 1u)) acc[c][q] += w * uc[q];
      }
    }
    const unsigned fn = fix[n];
#pragma unroll
    for (int c = 0; c < NB; ++c)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        y[c * ld + 3 * n + q] = ((fn >> q) & 1u) ? 0.0 : acc[c][q];
  }
}

// ---- buckling sensitivities (Buckling.cpp:113-272)
//
// With ks_e = H_e (x) I_3, phi^T ks_e(u) phi = detJ sum_q sigma_q(u) : M_q
// where M_q = sum_c grad(phi_c) grad(phi_c)^T at Gauss point q.  This is
// linear in u, so its gradient with respect to u_e (the reference's
// phi^T dKsdu phi, :134-147 and :168-173) is detJ sum_q B_q^T D m_q, m_q the
// Voigt form of M_q with doubled shears.

// M_q of one element for phi (phi[l][c], lexicographic corners) as the
// Voigt vector (Mxx, Myy, Mzz, 2Mxy, 2Myz, 2Mxz)
__device__ __forceinline__ void phi_moment(const KsConst &kc, int q, const double phi[8][3],
                                           double m[6]) {
  double G[3][3];   // G[c][a] = d phi_c / d x_a
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double s = 0.0;
#pragma unroll
      for (int l = 0; l < 8; ++l) s += kc.g[q][a][l] * phi[l][c];
      G[c][a] = s;
    }
  double M[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) M[a][b] = G[0][a] * G[0][b] + G[1][a] * G[1][b] + G[2][a] * G[2][b];
  m[0] = M[0][0];
  m[1] = M[1][1];
  m[2] = M[2][2];
  m[3] = 2.0 * M[0][1];
  m[4] = 2.0 * M[1][2];
  m[5] = 2.0 * M[0][2];
}

// Voigt stress D eps of an engineering-strain Voigt vector
__device__ __forceinline__ void voigt_stress(const KsConst &kc, const double e[6], double s[6]) {
  s[0] = kc.t1 * e[0] + kc.t3 * (e[1] + e[2]);
  s[1] = kc.t1 * e[1] + kc.t3 * (e[0] + e[2]);
  s[2] = kc.t1 * e[2] + kc.t3 * (e[0] + e[1]);
  s[3] = kc.t2 * e[3];
  s[4] = kc.t2 * e[4];
  s[5] = kc.t2 * e[5];
}

// W[(3l + c) * ne + e] = Es_e d(phi^T ks_e phi)/du_{l,c} for one eigenvector
__global__ void k_bk_adj_element(int nelx, int nely, int nelz,
                                 const double *__restrict__ phi,
                                 const double *__restrict__ Es, KsConst kc,
                                 double *__restrict__ W) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nelx), j = (int)((e / nelx) % nely),
              k = (int)(e / ((int64_t)nelx * nely));
    const int64_t n0 = ((int64_t)k * Ny + j) * Nx + i;
    double p[8][3], w[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int64_t n = n0 + (l & 1) + ((l >> 1) & 1) * Nx + ((l >> 2) & 1) * (int64_t)Nx * Ny;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        p[l][c] = phi[3 * n + c];
        w[l][c] = 0.0;
      }
    }
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      double m[6], s[6];
      phi_moment(kc, q, p, m);
      voigt_stress(kc, m, s);
      // B_q^T s
#pragma unroll
      for (int l = 0; l < 8; ++l) {
        const double gx = kc.g[q][0][l], gy = kc.g[q][1][l], gz = kc.g[q][2][l];
        w[l][0] += gx * s[0] + gy * s[3] + gz * s[5];
        w[l][1] += gy * s[1] + gx * s[3] + gz * s[4];
        w[l][2] += gz * s[2] + gy * s[4] + gx * s[5];
      }
    }
    const double sc = Es[e] * kc.detJ;
#pragma unroll
    for (int l = 0; l < 8; ++l)
#pragma unroll
      for (int c = 0; c < 3; ++c) W[(int64_t)(3 * l + c) * ne + e] = sc * w[l][c];
  }
}

// rhs[3n + c] = sum over the (up to 8) elements around node n of their
// W entry for n, in a fixed order; zero at fixed dofs (:186-190)
__global__ void k_bk_adj_gather(int nelx, int nely, int nelz,
                                const double *__restrict__ W,
                                const uint8_t *__restrict__ fix,
                                double *__restrict__ rhs) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz, ne = (int64_t)nelx * nely * nelz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % Nx), j = (int)((n / Nx) % Ny), k = (int)(n / ((int64_t)Nx * Ny));
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int cz = 0; cz < 2; ++cz)
#pragma unroll
      for (int cy = 0; cy < 2; ++cy)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int ei = i - 1 + cx, ej = j - 1 + cy, ek = k - 1 + cz;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
            continue;
          const int64_t e = ((int64_t)ek * nely + ej) * nelx + ei;
          const int ln = (1 - cx) + 2 * (1 - cy) + 4 * (1 - cz);
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[c] += W[(int64_t)(3 * ln + c) * ne + e];
        }
    const unsigned f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) rhs[3 * n + c] = ((f >> c) & 1u) ? 0.0 : acc[c];
  }
}

// per element, over the nev eigenpairs (phi_k, v_k columns of stride ld):
// g_e = scale sum_k a_k (-dEsdz_e phi^T ks_e(U) phi - lam_k dEdz_e phi^T K0 phi
//                        + dEdz_e v^T K0 U)          (:229-265)
__global__ void k_bk_gradient(int nelx, int nely, int nelz,
                              const double *__restrict__ U,
                              const double *__restrict__ phi,
                              const double *__restrict__ v, int64_t ld, int nev,
                              const double *__restrict__ dEdz,
                              const double *__restrict__ dEsdz, KsConst kc,
                              const double *__restrict__ K0, BkCoef coef,
                              double *__restrict__ g) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nelx), j = (int)((e / nelx) % nely),
              k = (int)(e / ((int64_t)nelx * nely));
    const int64_t n0 = ((int64_t)k * Ny + j) * Nx + i;
    int64_t node[8];
    double u[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      node[l] = n0 + (l & 1) + ((l >> 1) & 1) * Nx + ((l >> 2) & 1) * (int64_t)Nx * Ny;
#pragma unroll
      for (int c = 0; c < 3; ++c) u[l][c] = U[3 * node[l] + c];
    }
    // K0 U_e
    double ku[24];
#pragma unroll
    for (int r = 0; r < 24; ++r) {
      double s = 0.0;
#pragma unroll
      for (int l = 0; l < 8; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) s += __ldg(K0 + r * 24 + 3 * l + c) * u[l][c];
      ku[r] = s;
    }
    const double de = dEdz[e], dse = dEsdz[e];
    double acc = 0.0;
#pragma unroll 1
    for (int kk = 0; kk < nev; ++kk) {
      const double *pk = phi + kk * ld, *vk = v + kk * ld;
      double p[8][3];
      double vku = 0.0;
#pragma unroll
      for (int l = 0; l < 8; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          p[l][c] = pk[3 * node[l] + c];
          vku += vk[3 * node[l] + c] * ku[3 * l + c];
        }
      // phi^T ks_e(U) phi = detJ sum_q sigma_q(U) : M_q(phi)
      double pksp = 0.0;
#pragma unroll 1
      for (int q = 0; q < 8; ++q) {
        double F[3][3];   // F[c][a] = d u_c / d x_a
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            double s = 0.0;
#pragma unroll
            for (int l = 0; l < 8; ++l) s += kc.g[q][a][l] * u[l][c];
            F[c][a] = s;
          }
        const double eps[6] = {F[0][0], F[1][1], F[2][2], F[0][1] + F[1][0],
                               F[1][2] + F[2][1], F[0][2] + F[2][0]};
        double sig[6], m[6];
        voigt_stress(kc, eps, sig);
        phi_moment(kc, q, p, m);
        pksp += sig[0] * m[0] + sig[1] * m[1] + sig[2] * m[2] + sig[3] * m[3] +
                sig[4] * m[4] + sig[5] * m[5];
      }
      pksp *= kc.detJ;
      // phi^T K0 phi
      double pkp = 0.0;
#pragma unroll
      for (int r = 0; r < 24; ++r) {
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < 8; ++l)
#pragma unroll
          for (int c = 0; c < 3; ++c) s += __ldg(K0 + r * 24 + 3 * l + c) * p[l][c];
        pkp += p[r / 3][r % 3] * s;
      }
      acc += coef.a[kk] * (-dse * pksp - coef.lam[kk] * de * pkp + de * vku);
    }
    g[e] = coef.scale * acc;
  }
}

// ---- frequency (Dynamic.cpp:18-235)

// Frequency::DiagMassFnc (:181-235) with the fixed-dof zeroing (:42-44):
// m[3n + c] = sum over the elements around n of V_e * scale, scale =
// elemSize * density / (2^3 * 3), plus the point masses mlump; 1e-8 at
// fixed dofs (MatZeroRowsColumns with diagonal 1e-8 after the assembly)
__global__ void k_lumped_mass(int nelx, int nely, int nelz,
                              const double *__restrict__ V, double scale,
                              const uint8_t *__restrict__ fix,
                              const double *__restrict__ mlump,
                              double *__restrict__ m) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int64_t nn = (int64_t)Nx * Ny * Nz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % Nx), j = (int)((n / Nx) % Ny), k = (int)(n / ((int64_t)Nx * Ny));
    double acc = 0.0;
#pragma unroll
    for (int cz = 0; cz < 2; ++cz)
#pragma unroll
      for (int cy = 0; cy < 2; ++cy)
#pragma unroll
        for (int cx = 0; cx < 2; ++cx) {
          const int ei = i - 1 + cx, ej = j - 1 + cy, ek = k - 1 + cz;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= nelx || ej >= nely || ek >= nelz)
            continue;
          acc += V[((int64_t)ek * nely + ej) * nelx + ei] * scale;
        }
    const unsigned f = fix[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      m[3 * n + c] = ((f >> c) & 1u) ? 1e-8 : acc + (mlump ? mlump[3 * n + c] : 0.0);
  }
}

// g_e = scale sum_{k < nterms} a_k (dVdrho_e mscale |phi_e|^2
//                                   - lam_k dEdz_e phi^T K0 phi)   (:127-160)
// with dVdrho = 1 (V = rho, Material_Interpolation.cpp:63-64)
__global__ void k_freq_gradient(int nelx, int nely, int nelz,
                                const double *__restrict__ phi, int64_t ld, int nterms,
                                const double *__restrict__ dEdz,
                                const double *__restrict__ K0, double mscale,
                                BkCoef coef, double *__restrict__ g) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nelx), j = (int)((e / nelx) % nely),
              k = (int)(e / ((int64_t)nelx * nely));
    const int64_t n0 = ((int64_t)k * Ny + j) * Nx + i;
    int64_t node[8];
#pragma unroll
    for (int l = 0; l < 8; ++l)
      node[l] = n0 + (l & 1) + ((l >> 1) & 1) * Nx + ((l >> 2) & 1) * (int64_t)Nx * Ny;
    const double de = dEdz[e];
    double acc = 0.0;
#pragma unroll 1
    for (int kk = 0; kk < nterms; ++kk) {
      const double *pk = phi + kk * ld;
      double p[8][3];
      double pp = 0.0;
#pragma unroll
      for (int l = 0; l < 8; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          p[l][c] = pk[3 * node[l] + c];
          pp += p[l][c] * p[l][c];
        }
      double pkp = 0.0;
#pragma unroll
      for (int r = 0; r < 24; ++r) {
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < 8; ++l)
#pragma unroll
          for (int c = 0; c < 3; ++c) s += __ldg(K0 + r * 24 + 3 * l + c) * p[l][c];
        pkp += p[r / 3][r % 3] * s;
      }
      acc += coef.a[kk] * (mscale * pp - coef.lam[kk] * de * pkp);
    }
    g[e] = coef.scale * acc;
  }
}

template <int NB>
void ks_launch(const Ctx &c, const double *u, double *y) {
  count_launch();
  k_ks_apply<NB><<<grid_for(c.nn, 128), 128, 0, c.stream>>>(
      c.nel[0] + 1, c.nel[1] + 1, c.nel[2] + 1, c.ks_S, c.fix, u, y, 3 * c.nn);
}

}  // namespace

void launch_ks_assemble(const Ctx &c, cudaStream_t s) {
  count_launch(2);
  k_ks_element<<<grid_for(c.ne, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                    c.U, c.Es64, c.ksc, c.ks_H);
  k_ks_gather<<<grid_for(c.nn, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                   c.ks_H, c.ks_S);
}

void launch_bk_adj_rhs(const Ctx &c, const double *phi, double *W, double *rhs,
                       cudaStream_t s) {
  count_launch(2);
  k_bk_adj_element<<<grid_for(c.ne, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2], phi,
                                                        c.Es64, c.ksc, W);
  k_bk_adj_gather<<<grid_for(c.nn, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2], W,
                                                       c.fix, rhs);
}

void launch_bk_gradient(const Ctx &c, const double *phi, const double *v, int64_t ld,
                        int nev, const BkCoef &coef, double *g, cudaStream_t s) {
  count_launch();
  k_bk_gradient<<<grid_for(c.ne, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2], c.U,
                                                     phi, v, ld, nev, c.dEdz, c.dEsdz64,
                                                     c.ksc, c.K0lex, coef, g);
}

void launch_lumped_mass(const Ctx &c, double scale, const double *mlump, double *m,
                        cudaStream_t s) {
  count_launch();
  k_lumped_mass<<<grid_for(c.nn, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2], c.rho,
                                                     scale, c.fix, mlump, m);
}

void launch_freq_gradient(const Ctx &c, const double *phi, int64_t ld, int nterms,
                          double mscale, const BkCoef &coef, double *g, cudaStream_t s) {
  count_launch();
  k_freq_gradient<<<grid_for(c.ne, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2], phi, ld,
                                                       nterms, c.dEdz, c.K0lex, mscale,
                                                       coef, g);
}

void launch_ks_apply(const Ctx &c, const double *u, double *y, int nb) {
  const int64_t ld = 3 * c.nn;
  while (nb > 0) {
    const int w = nb >= 8 ? 8 : nb >= 4 ? 4 : nb >= 2 ? 2 : 1;
    if (w == 8) ks_launch<8>(c, u, y);
    else if (w == 4) ks_launch<4>(c, u, y);
    else if (w == 2) ks_launch<2>(c, u, y);
    else ks_launch<1>(c, u, y);
    u += w * ld;
    y += w * ld;
    nb -= w;
  }
}

}  // namespace tpo
