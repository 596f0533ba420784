// Geometric multigrid kernels: Galerkin coarse operators, stencil operator
// on the coarse levels, trilinear transfers, Chebyshev/Jacobi smoother
// updates and the dense coarsest-level solve.
//
// Level layout (Interpolation.cpp:31-169): a coarse node sits on every even
// fine node index; level l+1 has (N_l + 1) / 2 nodes per dimension,
// numbered lexicographically.  The prolongation weight of coarse node c for
// fine node f is prod_d w_d with w_d = 1 (f_d = 2c_d) or 1/2 (|f_d - 2c_d| =
// 1), each row normalised to sum 1 (Interpolation.cpp:330-347).  The
// normalisation factorises per dimension, so weights are computed on the
// fly from the indices; no interpolation matrix is stored.
//
// Coarse operators are A_{l+1} = P^T A_l P (PCMG Galerkin,
// FEAnalysis.cpp:412), stored as 27-point 3x3-block stencils in SoA form
// S[(nb*9 + 3r + s) * nn + node].
#include <algorithm>

#include "tpo_internal.h"
#include "transfer.cuh"
#include "fused_out.cuh"

namespace tpo {

namespace {

int grid_for(int64_t n, int threads, int64_t cap = 148 * 32) {
  int64_t g = (n + threads - 1) / threads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// normalised 1-D prolongation weight of coarse index c for fine index f
// (fine extent Nf)
__device__ __forceinline__ double pw1(int f, int c, int Nf) {
  const int d = f - 2 * c;
  if (d < -1 || d > 1) return 0.0;
  if (d == 0) return 1.0;
  // odd f: neighbours (f-1)/2 always, (f+1)/2 if f+1 <= Nf-1
  return (f + 1 <= Nf - 1) ? 0.5 : 1.0;
}

// ---- level 1 straight from the element moduli ----------------------------
//
// A_1 = P^T A_0 P with A_0 = M (sum_e E_e K0_e) M + (I - M), M the mask of
// dofs without an identity row (idm).  Every fine element lies inside one
// level-1 coarse element (2x2x2 fine elements) and its 8 nodes interpolate
// from that coarse element's 8 nodes, so
//   A_1 = sum_E sum_{e in E} E_e Q_e^T (M K0 M) Q_e + P^T (I - M) P.
// For a fine element without identity dofs at offset i of a coarse element
// with all 8 corners, Q_e^T K0 Q_e is one of 8 fixed 24x24 matrices (GMi,
// element.cpp); the 3x3 block (ln, lm) of the coarse stencil is then
// sum_i E_{e_i} GMi[i][ln][lm].  Coarse elements whose closed fine box holds
// an identity dof, or that miss a corner (odd element counts), take the
// general path: masked K0 with the interpolation weights of pw1.

// slot[E] >= 0: level-1 coarse element E needs the general path (an
// identity dof in its closed fine box, or a missing corner); slots are
// handed out by an atomic counter (their order does not affect any value)
__global__ void k_coarse_elem_flags(int nelx, int nely, int nelz,
                                    const uint8_t *__restrict__ idm,
                                    int *__restrict__ slot,
                                    int *__restrict__ slot_elem,
                                    unsigned int *__restrict__ count) {
  const int fx = nelx + 1, fy = nely + 1, fz = nelz + 1;
  const int ncx = (nelx + 1) / 2, ncy = (nely + 1) / 2, ncz = (nelz + 1) / 2;
  const int64_t nce = (int64_t)ncx * ncy * ncz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nce;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ex = (int)(t % ncx), ey = (int)((t / ncx) % ncy), ez = (int)(t / ((int64_t)ncx * ncy));
    unsigned any = (2 * ex + 2 > fx - 1) || (2 * ey + 2 > fy - 1) || (2 * ez + 2 > fz - 1);
    for (int z = 2 * ez; z <= min(2 * ez + 2, fz - 1) && !any; ++z)
      for (int y = 2 * ey; y <= min(2 * ey + 2, fy - 1); ++y)
        for (int x = 2 * ex; x <= min(2 * ex + 2, fx - 1); ++x)
          any |= idm[((int64_t)z * fy + y) * fx + x];
    int sl = -1;
    if (any) {
      sl = (int)atomicAdd(count, 1u);
      slot_elem[sl] = (int)t;
    }
    slot[t] = sl;
  }
}

// general path, one thread per (flagged coarse element, ln, lm): the 3x3
// block sum_{fine e in E} E_e sum_{p,q} w(p->ln) w(q->lm) (M K0 M)_pq with
// the interpolation weights of pw1 and the identity-dof masks
__global__ void k_galerkin_general(int nelx, int nely, int nelz, int nslots,
                                   const double *__restrict__ E,
                                   const uint8_t *__restrict__ idm,
                                   const int *__restrict__ slot_elem,
                                   const double *__restrict__ K0lex,
                                   double *__restrict__ G) {
  const int fx = nelx + 1, fy = nely + 1, fz = nelz + 1;
  const int ncx = (nelx + 1) / 2, ncy = (nely + 1) / 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 64 * (int64_t)nslots;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int sl = (int)(t / 64), pr = (int)(t % 64), ln = pr / 8, lm = pr % 8;
    const int ce = slot_elem[sl];
    const int EI = ce % ncx, EJ = (ce / ncx) % ncy, EK = ce / (ncx * ncy);
    // coarse corner coordinates (the far ones may not exist: pw1 gives 0)
    const int ix = EI + (ln & 1), iy = EJ + ((ln >> 1) & 1), iz = EK + ((ln >> 2) & 1);
    const int jx = EI + (lm & 1), jy = EJ + ((lm >> 1) & 1), jz = EK + ((lm >> 2) & 1);
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 8; ++i) {
      const int ex = 2 * EI + (i & 1), ey = 2 * EJ + ((i >> 1) & 1), ez = 2 * EK + ((i >> 2) & 1);
      if (ex >= nelx || ey >= nely || ez >= nelz) continue;
      const double Ee = E[((int64_t)ez * nely + ey) * nelx + ex];
      double wn[8], wm[8];
      unsigned msk[8];
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int gx = ex + (p & 1), gy = ey + ((p >> 1) & 1), gz = ez + ((p >> 2) & 1);
        wn[p] = pw1(gx, ix, fx) * pw1(gy, iy, fy) * pw1(gz, iz, fz);
        wm[p] = pw1(gx, jx, fx) * pw1(gy, jy, fy) * pw1(gz, jz, fz);
        msk[p] = idm[((int64_t)gz * fy + gy) * fx + gx];
      }
      for (int p = 0; p < 8; ++p) {
        if (wn[p] == 0.0) continue;
        for (int q = 0; q < 8; ++q) {
          const double w = Ee * wn[p] * wm[q];
          if (w == 0.0) continue;
          const double *k0 = K0lex + 24 * (3 * p) + 3 * q;
          for (int r = 0; r < 3; ++r) {
            if ((msk[p] >> r) & 1u) continue;
            for (int s2 = 0; s2 < 3; ++s2)
              if (!((msk[q] >> s2) & 1u)) acc[3 * r + s2] += w * k0[24 * r + s2];
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) G[(int64_t)t * 9 + q] = acc[q];
  }
}

// the level-1 stencil: per (coarse node, neighbour) block, the fast-path
// element sums, the general-path blocks of flagged elements and the
// P^T (I - M) P term of the identity dofs
__global__ void k_galerkin_fine(int nelx, int nely, int nelz,
                                const double *__restrict__ E,
                                const uint8_t *__restrict__ idm,
                                const int *__restrict__ slot,
                                const double *__restrict__ G,
                                const double *__restrict__ GMi,
                                double *__restrict__ Sc) {
  const int fx = nelx + 1, fy = nely + 1, fz = nelz + 1;
  const int cx = (fx + 1) / 2, cy = (fy + 1) / 2, cz = (fz + 1) / 2;
  const int ncx = (nelx + 1) / 2, ncy = (nely + 1) / 2, ncz = (nelz + 1) / 2;
  const int64_t nnc = (int64_t)cx * cy * cz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 27 * nnc;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int nb = (int)(t / nnc);
    const int64_t I = t - (int64_t)nb * nnc;
    const int ix = (int)(I % cx), iy = (int)((I / cx) % cy), iz = (int)(I / ((int64_t)cx * cy));
    const int jx = ix + nb % 3 - 1, jy = iy + (nb / 3) % 3 - 1, jz = iz + nb / 9 - 1;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (jx >= 0 && jx < cx && jy >= 0 && jy < cy && jz >= 0 && jz < cz) {
      bool anyflag = false;
      for (int EK = max(iz, jz) - 1; EK <= min(iz, jz); ++EK)
        for (int EJ = max(iy, jy) - 1; EJ <= min(iy, jy); ++EJ)
          for (int EI = max(ix, jx) - 1; EI <= min(ix, jx); ++EI) {
            if (EI < 0 || EJ < 0 || EK < 0 || EI >= ncx || EJ >= ncy || EK >= ncz)
              continue;
            const int ln = (ix - EI) + 2 * (iy - EJ) + 4 * (iz - EK);
            const int lm = (jx - EI) + 2 * (jy - EJ) + 4 * (jz - EK);
            const int sl = slot[((int64_t)EK * ncy + EJ) * ncx + EI];
            if (sl >= 0) {
              anyflag = true;
              const double *g = G + ((int64_t)sl * 64 + ln * 8 + lm) * 9;
#pragma unroll
              for (int q = 0; q < 9; ++q) acc[q] += g[q];
              continue;
            }
            for (int i = 0; i < 8; ++i) {
              const int ex = 2 * EI + (i & 1), ey = 2 * EJ + ((i >> 1) & 1),
                        ez = 2 * EK + ((i >> 2) & 1);
              const double Ee = E[((int64_t)ez * nely + ey) * nelx + ex];
              const double *m = GMi + ((i * 8 + ln) * 8 + lm) * 9;
#pragma unroll
              for (int q = 0; q < 9; ++q) acc[q] += Ee * __ldg(m + q);
            }
          }
      if (anyflag) {
        // P^T (I - M) P: identity dofs in the support of both N and M
        for (int gz = max(2 * iz, 2 * jz) - 1; gz <= min(2 * iz, 2 * jz) + 1; ++gz)
          for (int gy = max(2 * iy, 2 * jy) - 1; gy <= min(2 * iy, 2 * jy) + 1; ++gy)
            for (int gx = max(2 * ix, 2 * jx) - 1; gx <= min(2 * ix, 2 * jx) + 1; ++gx) {
              if (gx < 0 || gy < 0 || gz < 0 || gx >= fx || gy >= fy || gz >= fz) continue;
              const unsigned bits = idm[((int64_t)gz * fy + gy) * fx + gx];
              if (!bits) continue;
              const double w = pw1(gx, ix, fx) * pw1(gy, iy, fy) * pw1(gz, iz, fz) *
                               pw1(gx, jx, fx) * pw1(gy, jy, fy) * pw1(gz, jz, fz);
              for (int c = 0; c < 3; ++c)
                if ((bits >> c) & 1u) acc[4 * c] += w;
            }
      }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) Sc[(int64_t)(nb * 9 + q) * nnc + I] = acc[q];
  }
}

// One dimension of the Galerkin product: P = P_x (x) P_y (x) P_z, so
// P^T A P = P_z^T (P_y^T (P_x^T A P_x) P_y) P_z and each factor keeps a
// 27-point 3x3-block stencil.  Coarsening dimension D of a grid n[3]:
//   A'(O, O+Delta) = sum_{f_D} sum_{g_D = f_D + d_D} w(f_D -> O_D)
//                    w(g_D -> O_D + Delta_D) A(f, f + d),
// with f = O except f_D and d = Delta except d_D: at most 7 (Delta_D = 0)
// or 3 input blocks per output block, instead of up to 343 for the direct
// triple product.  w is the normalised 1-D weight pw1.
template <int D>
__global__ void k_galerkin_dim(int nx, int ny, int nz, const double *__restrict__ Sin,
                               double *__restrict__ Sout) {
  const int n[3] = {nx, ny, nz};
  int m[3] = {nx, ny, nz};
  m[D] = (n[D] + 1) / 2;
  const int64_t nin = (int64_t)nx * ny * nz, nout = (int64_t)m[0] * m[1] * m[2];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 27 * nout;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int nb = (int)(t / nout);
    const int64_t O = t - (int64_t)nb * nout;
    int o[3] = {(int)(O % m[0]), (int)((O / m[0]) % m[1]), (int)(O / ((int64_t)m[0] * m[1]))};
    const int dl[3] = {nb % 3 - 1, (nb / 3) % 3 - 1, nb / 9 - 1};
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool inside = true;
#pragma unroll
    for (int e = 0; e < 3; ++e) inside &= (o[e] + dl[e] >= 0 && o[e] + dl[e] < m[e]);
    if (inside) {
      const int I = o[D], J = o[D] + dl[D];
      for (int fd = 2 * I - 1; fd <= 2 * I + 1; ++fd) {
        if (fd < 0 || fd >= n[D]) continue;
        const double wi = pw1(fd, I, n[D]);
        if (wi == 0.0) continue;
        int f[3] = {o[0], o[1], o[2]};
        f[D] = fd;
        const int64_t fi = ((int64_t)f[2] * ny + f[1]) * nx + f[0];
        for (int dd = -1; dd <= 1; ++dd) {
          const int gd = fd + dd;
          if (gd < 0 || gd >= n[D]) continue;
          const double wj = pw1(gd, J, n[D]);
          if (wj == 0.0) continue;
          int d3[3] = {dl[0], dl[1], dl[2]};
          d3[D] = dd;
          const int fnb = (d3[2] + 1) * 9 + (d3[1] + 1) * 3 + (d3[0] + 1);
          const double w = wi * wj;
          const double *blk = Sin + (int64_t)fnb * 9 * nin + fi;
#pragma unroll
          for (int q = 0; q < 9; ++q) acc[q] += w * blk[q * nin];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) Sout[(int64_t)(nb * 9 + q) * nout + O] = acc[q];
  }
}


// 32 nodes x 9 neighbour rows per CTA: thread (lane, g) takes node
// 32 * block + lane and the three neighbour blocks of row g = (dj, dk),
// i.e. 27 coefficient and 9 u loads, so the loads of a node are spread
// over 9 threads instead of one 324-load chain (the levels this kernel
// serves are small and latency-bound); the 9 partial sums are combined in
// shared memory in a fixed order.  Lanes span consecutive nodes, so each
// coefficient load is coalesced.
constexpr int kStencilRows = 9;
template <typename T, bool RESID>
__global__ void __launch_bounds__(32 * kStencilRows)
    k_apply_stencil(int nx, int ny, int nz, const T *__restrict__ S,
                    const T *__restrict__ u, const T *__restrict__ b,
                    T *__restrict__ y) {
  __shared__ T part[kStencilRows][3][32];
  const int64_t nn = (int64_t)nx * ny * nz;
  const int lane = threadIdx.x, g = threadIdx.y;
  const int dj = g % 3 - 1, dk = g / 3 - 1;
  for (int64_t n0 = (int64_t)blockIdx.x * 32; n0 < nn; n0 += (int64_t)gridDim.x * 32) {
    const int64_t n = n0 + lane;
    T a0 = 0, a1 = 0, a2 = 0;
    if (n < nn) {
      const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / ((int64_t)nx * ny));
      const int mj = j + dj, mk = k + dk;
      if (mj >= 0 && mj < ny && mk >= 0 && mk < nz) {
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int mi = i + di;
          if (mi < 0 || mi >= nx) continue;
          const int nb = g * 3 + di + 1;
          const int64_t m = ((int64_t)mk * ny + mj) * nx + mi;
          const T u0 = u[3 * m], u1 = u[3 * m + 1], u2 = u[3 * m + 2];
          const T *s = S + (int64_t)nb * 9 * nn + n;
          a0 += s[0] * u0 + s[nn] * u1 + s[2 * nn] * u2;
          a1 += s[3 * nn] * u0 + s[4 * nn] * u1 + s[5 * nn] * u2;
          a2 += s[6 * nn] * u0 + s[7 * nn] * u1 + s[8 * nn] * u2;
        }
      }
    }
    part[g][0][lane] = a0;
    part[g][1][lane] = a1;
    part[g][2][lane] = a2;
    __syncthreads();
    if (g < 3 && n < nn) {
      T a = 0;
#pragma unroll
      for (int r = 0; r < kStencilRows; ++r) a += part[r][g][lane];
      if (RESID) a = b[3 * n + g] - a;
      y[3 * n + g] = a;
    }
    __syncthreads();
  }
}

// The FP32 copy of a half-stored stencil is grouped by tiles of 32 nodes:
// coefficient hq (0..125) of node n at ((n / 32) * 126 + hq) * 32 + n % 32,
// so the 126 x 32 values a warp reads for its 32 nodes are one contiguous
// 16,128-byte block that one bulk L2 prefetch covers.  The FP64 copy stays
// coefficient-major, hq * nn + n.
constexpr int kH32Tile = 32;
__host__ __device__ __forceinline__ int64_t h32_index(int hq, int64_t n) {
  return ((n / kH32Tile) * 126 + hq) * kH32Tile + n % kH32Tile;
}
template <typename T>
__device__ __forceinline__ const T *hcoef(const T *H, int hq, int64_t n, int64_t nn);
template <>
__device__ __forceinline__ const double *hcoef(const double *H, int hq, int64_t n,
                                               int64_t nn) {
  return H + hq * nn + n;
}
template <>
__device__ __forceinline__ const float *hcoef(const float *H, int hq, int64_t n, int64_t) {
  return H + h32_index(hq, n);
}
// one bulk prefetch of a 32-node tile of the FP32 stencil into L2
__device__ __forceinline__ void prefetch_h32_tile(const float *H, int64_t n) {
  const float *p = H + (n / kH32Tile) * 126 * kH32Tile;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p),
               "r"(126 * kH32Tile * 4)
               : "memory");
}

// Symmetric half of a Galerkin stencil: A(n, n+d) = A(n+d, n)^T, so only
// the centre block and the 13 forward offsets (nb = 13..26) are stored,
// H[(h*9 + 3r + s) * nn + n] with h = nb - 13.  The apply reads the forward
// blocks of node n and, transposed, the forward blocks that its 13 backward
// neighbours store for it; those were read moments earlier by the
// neighbouring threads, so the second read hits L2 and DRAM traffic is the
// half-size array.
__global__ void k_stencil_to_half(int64_t nn, const double *__restrict__ S,
                                  double *__restrict__ H64,
                                  float *__restrict__ H32) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 126 * nn;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double v = S[117 * nn + t];   // (13*9 + q) * nn + n
    H64[t] = v;
    const int64_t hq = t / nn, n = t - hq * nn;
    H32[h32_index((int)hq, n)] = static_cast<float>(v);
  }
}

// The kernel is bound by the latency of the coefficient loads.  The block
// loop is not unrolled, so a thread needs 32 registers and 16 blocks of 128
// fit on an SM: the 97x49x49 level 1 of 192x96x96 then runs in one wave at
// full occupancy.  Fully unrolled it took 64 registers, half the warps and
// 1.5 waves, and a solve was 1.4% (FP32) / 5.6% (FP64) slower.
template <typename T, int IN, int OUT>
__global__ void __launch_bounds__(128, 16)
    k_apply_stencil_sym1(int nx, int ny, int nz, const T *__restrict__ H,
                         const ApplyArgs<T> args) {
  const int nn = nx * ny * nz;
  // stride between the 9 coefficients of one block
  const int64_t qs = sizeof(T) == 4 ? kH32Tile : (int64_t)nn;
  const int stride = gridDim.x * blockDim.x;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += stride) {
    // FP32: a warp's 32 nodes are one tile of the stencil; the tile this
    // warp takes next goes to L2 in one bulk prefetch
    if (sizeof(T) == 4 && (threadIdx.x & 31) == 0 && n + stride < nn)
      prefetch_h32_tile(reinterpret_cast<const float *>(H), n + stride);
    const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
    T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 1
    for (int h = 0; h < 14; ++h) {
      const int nb = 13 + h;
      const int di = nb % 3 - 1, dj = (nb / 3) % 3 - 1, dk = nb / 9 - 1;
      // forward block A(n, n+d): zero when n+d is outside, index clamped
      {
        const int mi = min(i + di, nx - 1), mj = min(max(j + dj, 0), ny - 1),
                  mk = min(k + dk, nz - 1);
        const int m = (mk * ny + mj) * nx + max(mi, 0);
        const T u0 = sym_in<T, IN>(args, 3 * m), u1 = sym_in<T, IN>(args, 3 * m + 1),
                u2 = sym_in<T, IN>(args, 3 * m + 2);
        const T *s = hcoef(H, h * 9, n, nn);
        a0 += s[0] * u0 + s[qs] * u1 + s[2 * qs] * u2;
        a1 += s[3 * qs] * u0 + s[4 * qs] * u1 + s[5 * qs] * u2;
        a2 += s[6 * qs] * u0 + s[7 * qs] * u1 + s[8 * qs] * u2;
      }
      // backward block A(n, n-d) = A(n-d, n)^T, stored by node n-d
      if (h > 0) {
        const int mi = i - di, mj = j - dj, mk = k - dk;
        const bool in = mi >= 0 && mi < nx && mj >= 0 && mj < ny && mk >= 0 && mk < nz;
        const int m = in ? (mk * ny + mj) * nx + mi : n;
        const T w = in ? T(1) : T(0);
        const T u0 = w * sym_in<T, IN>(args, 3 * m), u1 = w * sym_in<T, IN>(args, 3 * m + 1),
                u2 = w * sym_in<T, IN>(args, 3 * m + 2);
        const T *s = hcoef(H, h * 9, m, nn);
        a0 += s[0] * u0 + s[3 * qs] * u1 + s[6 * qs] * u2;
        a1 += s[qs] * u0 + s[4 * qs] * u1 + s[7 * qs] * u2;
        a2 += s[2 * qs] * u0 + s[5 * qs] * u1 + s[8 * qs] * u2;
      }
    }
    const bool need_u = OUT == OUT_CHEB2 || OUT == OUT_POST0 || OUT == OUT_POST1;
    const T Au[3] = {a0, a1, a2};
#pragma unroll
    for (int c = 0; c < 3; ++c)
      sym_out<T, OUT>(args, 3 * n + c, Au[c], need_u ? sym_in<T, IN>(args, 3 * n + c) : T(0));
  }
}

// NB columns (stride ld) share every coefficient load
template <typename T, bool RESID, int NB>
__global__ void k_apply_stencil_sym(int nx, int ny, int nz,
                                    const T *__restrict__ H,
                                    const T *__restrict__ u,
                                    const T *__restrict__ b, T *__restrict__ y,
                                    int64_t ld) {
  const int nn = nx * ny * nz;
  const int64_t qs = sizeof(T) == 4 ? kH32Tile : (int64_t)nn;
  const int stride = gridDim.x * blockDim.x;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += stride) {
    if (sizeof(T) == 4 && (threadIdx.x & 31) == 0 && n + stride < nn)
      prefetch_h32_tile(reinterpret_cast<const float *>(H), n + stride);
    const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
    T a[NB][3];
#pragma unroll
    for (int col = 0; col < NB; ++col) a[col][0] = a[col][1] = a[col][2] = T(0);
#pragma unroll
    for (int h = 0; h < 14; ++h) {
      const int nb = 13 + h;
      const int di = nb % 3 - 1, dj = (nb / 3) % 3 - 1, dk = nb / 9 - 1;
      // forward block A(n, n+d): zero when n+d is outside, index clamped
      {
        const int mi = min(i + di, nx - 1), mj = min(max(j + dj, 0), ny - 1),
                  mk = min(k + dk, nz - 1);
        const int m = (mk * ny + mj) * nx + max(mi, 0);
        const T *sp = hcoef(H, h * 9, n, nn);
        T c[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) c[q] = sp[q * qs];
#pragma unroll
        for (int col = 0; col < NB; ++col) {
          const T *uc = u + col * ld;
          const T u0 = uc[3 * m], u1 = uc[3 * m + 1], u2 = uc[3 * m + 2];
          a[col][0] += c[0] * u0 + c[1] * u1 + c[2] * u2;
          a[col][1] += c[3] * u0 + c[4] * u1 + c[5] * u2;
          a[col][2] += c[6] * u0 + c[7] * u1 + c[8] * u2;
        }
      }
      // backward block A(n, n-d) = A(n-d, n)^T, stored by node n-d
      if (h > 0) {
        const int mi = i - di, mj = j - dj, mk = k - dk;
        const bool in = mi >= 0 && mi < nx && mj >= 0 && mj < ny && mk >= 0 && mk < nz;
        const int m = in ? (mk * ny + mj) * nx + mi : n;
        const T w = in ? T(1) : T(0);
        const T *sp = hcoef(H, h * 9, m, nn);
        T c[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) c[q] = sp[q * qs];
#pragma unroll
        for (int col = 0; col < NB; ++col) {
          const T *uc = u + col * ld;
          const T u0 = w * uc[3 * m], u1 = w * uc[3 * m + 1], u2 = w * uc[3 * m + 2];
          a[col][0] += c[0] * u0 + c[3] * u1 + c[6] * u2;
          a[col][1] += c[1] * u0 + c[4] * u1 + c[7] * u2;
          a[col][2] += c[2] * u0 + c[5] * u1 + c[8] * u2;
        }
      }
    }
#pragma unroll
    for (int col = 0; col < NB; ++col) {
      T *yc = y + col * ld;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        T v = a[col][q];
        if (RESID) v = b[col * ld + 3 * n + q] - v;
        yc[3 * n + q] = v;
      }
    }
  }
}

__global__ void k_stencil_diag(int64_t nn, const double *__restrict__ S,
                               double *dinv64, float *dinv32) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    for (int c = 0; c < 3; ++c) {
      const double d = S[(int64_t)(13 * 9 + 4 * c) * nn + n];
      dinv64[3 * n + c] = 1.0 / d;
      dinv32[3 * n + c] = static_cast<float>(1.0 / d);
    }
  }
}

// b_c = P^T r_f for nb columns (fine stride 3 nnf, coarse stride 3 nnc)
template <typename T>
__global__ void k_restrict(int fx, int fy, int fz, int cx, int cy, int cz,
                           const T *__restrict__ rf, T *__restrict__ bc,
                           int nb) {
  const int64_t nnc = (int64_t)cx * cy * cz, nnf = (int64_t)fx * fy * fz;
  for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < nnc;
       I += (int64_t)gridDim.x * blockDim.x) {
    const int ix = I % cx, iy = (I / cx) % cy, iz = I / ((int64_t)cx * cy);
    for (int col = 0; col < nb; ++col) {
      T s[3];
      restrict_node(fx, fy, fz, ix, iy, iz, rf + col * 3 * nnf, s);
      T *o = bc + col * 3 * nnc;
      o[3 * I] = s[0];
      o[3 * I + 1] = s[1];
      o[3 * I + 2] = s[2];
    }
  }
}

// x_f += P x_c for nb columns
template <typename T>
__global__ void k_prolong_add(int fx, int fy, int fz, int cx, int cy, int cz,
                              const T *__restrict__ xc, T *__restrict__ xf,
                              int nb) {
  const int64_t nnf = (int64_t)fx * fy * fz, nnc = (int64_t)cx * cy * cz;
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nnf;
       f += (int64_t)gridDim.x * blockDim.x) {
    const int gx = f % fx, gy = (f / fx) % fy, gz = f / ((int64_t)fx * fy);
    for (int col = 0; col < nb; ++col) {
      T s[3];
      prolong_node(fx, fy, fz, cx, cy, cz, gx, gy, gz, xc + col * 3 * nnc, s);
      T *o = xf + col * 3 * nnf;
      o[3 * f] += s[0];
      o[3 * f + 1] += s[1];
      o[3 * f + 2] += s[2];
    }
  }
}

__global__ void k_to_dense(int nx, int ny, int nz, const double *__restrict__ S,
                           double *__restrict__ A) {
  const int64_t nn = (int64_t)nx * ny * nz, n3 = 3 * nn;
  const int64_t total = nn * 27 * 9;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t / nn);
    const int64_t n = t - (int64_t)q * nn;
    const int nb = q / 9, rs = q % 9, r = rs / 3, s = rs % 3;
    const int i = n % nx, j = (n / nx) % ny, k = n / ((int64_t)nx * ny);
    const int mi = i + nb % 3 - 1, mj = j + (nb / 3) % 3 - 1, mk = k + nb / 9 - 1;
    if (mi < 0 || mi >= nx || mj < 0 || mj >= ny || mk < 0 || mk >= nz) continue;
    const int64_t m = ((int64_t)mk * ny + mj) * nx + mi;
    A[(3 * n + r) * n3 + 3 * m + s] = S[t];
  }
}

// x = Ainv b, one warp per row, FP64 accumulation
template <typename T>
__global__ void k_coarse_gemv(int64_t n, const double *__restrict__ A,
                              const T *__restrict__ b, T *__restrict__ x) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const double s = gemv_row(A + row * n, b, n, lane);
    if (lane == 0) x[row] = static_cast<T>(s);
  }
}

// Chebyshev start: r = D^-1 (b or the residual already in r), d = r/theta,
// x (+)= d; column blockIdx.y (stride n), D^-1 shared
template <typename T>
__global__ void k_cheb_init(int64_t n, const T *__restrict__ dinv,
                            const T *__restrict__ b, T *__restrict__ r,
                            T *__restrict__ d, T *__restrict__ x, T inv_theta,
                            bool zero_guess) {
  const int64_t o = blockIdx.y * n;
  if (zero_guess) b += o;
  r += o;
  d += o;
  x += o;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = dinv[i] * (zero_guess ? b[i] : r[i]);
    const T di = ri * inv_theta;
    r[i] = ri;
    d[i] = di;
    x[i] = zero_guess ? di : x[i] + di;
  }
}

// r -= D^-1 A d ; d = c1 d + c2 r ; x += d; column blockIdx.y
template <typename T>
__global__ void k_cheb_step(int64_t n, const T *__restrict__ dinv,
                            const T *__restrict__ Ad, T *__restrict__ r,
                            T *__restrict__ d, T *__restrict__ x, T c1, T c2) {
  const int64_t o = blockIdx.y * n;
  Ad += o;
  r += o;
  d += o;
  x += o;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = r[i] - dinv[i] * Ad[i];
    const T di = c1 * d[i] + c2 * ri;
    r[i] = ri;
    d[i] = di;
    x[i] += di;
  }
}

}  // namespace

template <typename T>
void launch_apply_stencil(const Level &v, const T *S, const T *u, const T *b,
                          T *y, cudaStream_t s) {
  count_launch();
  const int g = grid_for(v.nn, 32);
  const dim3 blk(32, kStencilRows);
  if (b)
    k_apply_stencil<T, true><<<g, blk, 0, s>>>(v.dims[0], v.dims[1], v.dims[2],
                                               S, u, b, y);
  else
    k_apply_stencil<T, false><<<g, blk, 0, s>>>(v.dims[0], v.dims[1], v.dims[2],
                                                S, u, b, y);
}
template void launch_apply_stencil<double>(const Level &, const double *,
                                           const double *, const double *,
                                           double *, cudaStream_t);
template void launch_apply_stencil<float>(const Level &, const float *,
                                          const float *, const float *, float *,
                                          cudaStream_t);

template <typename T, bool RESID, int NB>
void sym_launch(const Level &v, const T *H, const T *u, const T *b, T *y,
                cudaStream_t s) {
  count_launch();
  const int g = grid_for(v.nn, 128);
  if (NB == 1) {
    ApplyArgs<T> a{};
    a.u = u;
    a.b = b;
    a.y = y;
    k_apply_stencil_sym1<T, IN_U, RESID ? OUT_RESID : OUT_Y><<<g, 128, 0, s>>>(
        v.dims[0], v.dims[1], v.dims[2], H, a);
  } else
    k_apply_stencil_sym<T, RESID, NB><<<g, 128, 0, s>>>(
        v.dims[0], v.dims[1], v.dims[2], H, u, b, y, 3 * v.nn);
}



template <typename T, bool RESID>
void sym_dispatch(const Level &v, const T *H, const T *u, const T *b, T *y,
                  cudaStream_t s, int nb) {
  const int64_t ld = 3 * v.nn;
  while (nb > 0) {
    const int w = nb >= 8 ? 8 : nb >= 4 ? 4 : nb >= 2 ? 2 : 1;
    if (w == 8) sym_launch<T, RESID, 8>(v, H, u, b, y, s);
    else if (w == 4) sym_launch<T, RESID, 4>(v, H, u, b, y, s);
    else if (w == 2) sym_launch<T, RESID, 2>(v, H, u, b, y, s);
    else sym_launch<T, RESID, 1>(v, H, u, b, y, s);
    u += w * ld;
    if (b) b += w * ld;
    y += w * ld;
    nb -= w;
  }
}

template <typename T>
void launch_apply_sym_fused(const Level &v, const T *H, int in, int out,
                            const ApplyArgs<T> &a, cudaStream_t s) {
  count_launch();
  const int g = grid_for(v.nn, 128);
  const int nx = v.dims[0], ny = v.dims[1], nz = v.dims[2];
  if (in == IN_CHEB && out == OUT_CHEB2)
    k_apply_stencil_sym1<T, IN_CHEB, OUT_CHEB2><<<g, 128, 0, s>>>(nx, ny, nz, H, a);
  else if (out == OUT_POST0)
    k_apply_stencil_sym1<T, IN_U, OUT_POST0><<<g, 128, 0, s>>>(nx, ny, nz, H, a);
  else if (out == OUT_POST1)
    k_apply_stencil_sym1<T, IN_U, OUT_POST1><<<g, 128, 0, s>>>(nx, ny, nz, H, a);
  else if (out == OUT_RESID)
    k_apply_stencil_sym1<T, IN_U, OUT_RESID><<<g, 128, 0, s>>>(nx, ny, nz, H, a);
  else
    k_apply_stencil_sym1<T, IN_U, OUT_Y><<<g, 128, 0, s>>>(nx, ny, nz, H, a);
}
template void launch_apply_sym_fused<double>(const Level &, const double *, int, int,
                                             const ApplyArgs<double> &, cudaStream_t);
template void launch_apply_sym_fused<float>(const Level &, const float *, int, int,
                                            const ApplyArgs<float> &, cudaStream_t);

template <typename T>
void launch_apply_stencil_sym(const Level &v, const T *H, const T *u,
                              const T *b, T *y, cudaStream_t s, int nb) {
  if (b)
    sym_dispatch<T, true>(v, H, u, b, y, s, nb);
  else
    sym_dispatch<T, false>(v, H, u, b, y, s, nb);
}
template void launch_apply_stencil_sym<double>(const Level &, const double *,
                                               const double *, const double *,
                                               double *, cudaStream_t, int);
template void launch_apply_stencil_sym<float>(const Level &, const float *,
                                              const float *, const float *,
                                              float *, cudaStream_t, int);

void launch_stencil_to_half(int64_t nn, const double *S, double *H64,
                            float *H32, cudaStream_t s) {
  count_launch();
  k_stencil_to_half<<<grid_for(126 * nn, 256), 256, 0, s>>>(nn, S, H64, H32);
}

int launch_galerkin_fine(Ctx &c, double *Sc, cudaStream_t s) {
  const int64_t nce = (int64_t)((c.nel[0] + 1) / 2) * ((c.nel[1] + 1) / 2) *
                      ((c.nel[2] + 1) / 2);
  count_launch(1);
  if (cudaMemsetAsync(c.gk_count, 0, sizeof(unsigned int), s) != cudaSuccess) return TPO_E_CUDA;
  k_coarse_elem_flags<<<grid_for(nce, 128), 128, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                          c.idm, c.gk_slot, c.gk_elem,
                                                          c.gk_count);
  unsigned int nslots = 0;
  if (cudaMemcpyAsync(&nslots, c.gk_count, sizeof(unsigned int), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return TPO_E_CUDA;
  if ((size_t)nslots * 576 > c.gk_cap) {
    if (c.gk_G) cudaFree(c.gk_G);
    c.gk_G = nullptr;
    c.gk_cap = 0;
    const size_t cap = std::max<size_t>((size_t)nslots * 576, 576);
    if (cudaMalloc(&c.gk_G, sizeof(double) * cap) != cudaSuccess) return TPO_E_CUDA;
    c.gk_cap = cap;
  }
  if (nslots) {
    count_launch();
    k_galerkin_general<<<grid_for(64 * (int64_t)nslots, 128, 1 << 20), 128, 0, s>>>(
        c.nel[0], c.nel[1], c.nel[2], (int)nslots, c.E64, c.idm, c.gk_elem, c.K0lex,
        c.gk_G);
  }
  count_launch();
  k_galerkin_fine<<<grid_for(27 * c.lev[1].nn, 128, 1 << 20), 128, 0, s>>>(
      c.nel[0], c.nel[1], c.nel[2], c.E64, c.idm, c.gk_slot, c.gk_G, c.GMi, Sc);
  // the tensor-core form of the FP32 level-1 operator (kernels_l1tc.cu)
  return l1tc_prepare(c, Sc, (int)nslots, s);
}

void launch_galerkin_dims(const Level &fine, const double *Sf, double *Sc,
                          double *tmp, cudaStream_t s) {
  const int fx = fine.dims[0], fy = fine.dims[1], fz = fine.dims[2];
  const int cx = (fx + 1) / 2, cy = (fy + 1) / 2;
  const int64_t n1 = (int64_t)cx * fy * fz, n2 = (int64_t)cx * cy * fz;
  double *t1 = tmp, *t2 = tmp + 243 * n1;
  count_launch(3);
  k_galerkin_dim<0><<<grid_for(27 * n1, 128, 1 << 20), 128, 0, s>>>(fx, fy, fz, Sf, t1);
  k_galerkin_dim<1><<<grid_for(27 * n2, 128, 1 << 20), 128, 0, s>>>(cx, fy, fz, t1, t2);
  const int64_t n3 = n2 / fz * ((fz + 1) / 2);
  k_galerkin_dim<2><<<grid_for(27 * n3, 128, 1 << 20), 128, 0, s>>>(cx, cy, fz, t2, Sc);
}

size_t galerkin_dims_scratch(const Level &fine) {
  const int fx = fine.dims[0], fy = fine.dims[1], fz = fine.dims[2];
  const int cx = (fx + 1) / 2, cy = (fy + 1) / 2;
  return 243 * ((size_t)cx * fy * fz + (size_t)cx * cy * fz);
}


void launch_stencil_diag(const Level &v, const double *S, double *dinv64,
                         float *dinv32, cudaStream_t s) {
  count_launch();
  k_stencil_diag<<<grid_for(v.nn, 256), 256, 0, s>>>(v.nn, S, dinv64, dinv32);
}

template <typename T>
void launch_restrict(const Level &fine, const Level &coarse, const T *rf,
                     T *bc, cudaStream_t s, int nb) {
  count_launch();
  k_restrict<T><<<grid_for(coarse.nn, 128), 128, 0, s>>>(
      fine.dims[0], fine.dims[1], fine.dims[2], coarse.dims[0], coarse.dims[1],
      coarse.dims[2], rf, bc, nb);
}
template void launch_restrict<double>(const Level &, const Level &,
                                      const double *, double *, cudaStream_t,
                                      int);
template void launch_restrict<float>(const Level &, const Level &,
                                     const float *, float *, cudaStream_t, int);

template <typename T>
void launch_prolong_add(const Level &fine, const Level &coarse, const T *xc,
                        T *xf, cudaStream_t s, int nb) {
  count_launch();
  k_prolong_add<T><<<grid_for(fine.nn, 128), 128, 0, s>>>(
      fine.dims[0], fine.dims[1], fine.dims[2], coarse.dims[0], coarse.dims[1],
      coarse.dims[2], xc, xf, nb);
}
template void launch_prolong_add<double>(const Level &, const Level &,
                                         const double *, double *,
                                         cudaStream_t, int);
template void launch_prolong_add<float>(const Level &, const Level &,
                                        const float *, float *, cudaStream_t,
                                        int);

void launch_to_dense(const Level &v, const double *S, double *A,
                     cudaStream_t s) {
  count_launch();
  const int64_t n3 = 3 * v.nn;
  cudaMemsetAsync(A, 0, sizeof(double) * n3 * n3, s);
  k_to_dense<<<grid_for(v.nn * 243, 256), 256, 0, s>>>(v.dims[0], v.dims[1],
                                                       v.dims[2], S, A);
}

namespace {
__global__ void k_soa_to_aos(int64_t nn, const double *__restrict__ S,
                             double *__restrict__ A64, float *__restrict__ A32) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn * 243;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = t / 243;
    const int w = (int)(t - n * 243);   // (3r+s)*27 + nb
    const int q = (w % 27) * 9 + w / 27;
    const double v = S[(int64_t)q * nn + n];
    A64[t] = v;
    A32[t] = static_cast<float>(v);
  }
}
}  // namespace

void launch_soa_to_aos(int64_t nn, const double *S, double *A64, float *A32,
                       cudaStream_t s) {
  count_launch();
  k_soa_to_aos<<<grid_for(nn * 243, 256), 256, 0, s>>>(nn, S, A64, A32);
}

template <typename T>
void launch_coarse_gemv(int64_t n, const double *Ainv, const T *b, T *x,
                        cudaStream_t s, int nb) {
  const int64_t warps = n;
  const int threads = 256;
  int64_t blocks = (warps * 32 + threads - 1) / threads;
  if (blocks > 148 * 8) blocks = 148 * 8;
  for (int col = 0; col < nb; ++col) {
    count_launch();
    k_coarse_gemv<T><<<(int)blocks, threads, 0, s>>>(n, Ainv, b + col * n,
                                                     x + col * n);
  }
}
template void launch_coarse_gemv<double>(int64_t, const double *,
                                         const double *, double *,
                                         cudaStream_t, int);
template void launch_coarse_gemv<float>(int64_t, const double *, const float *,
                                        float *, cudaStream_t, int);

static dim3 col_grid(int64_t n, int nb) {
  int g = grid_for(n, 256);
  if (nb > 1) g = std::max(148, g / nb);
  return dim3(g, nb);
}

template <typename T>
void launch_cheb_init(int64_t n, const T *dinv, const T *b, T *r, T *d, T *x,
                      double inv_theta, bool zero_guess, cudaStream_t s,
                      int nb) {
  count_launch();
  k_cheb_init<T><<<col_grid(n, nb), 256, 0, s>>>(
      n, dinv, b, r, d, x, static_cast<T>(inv_theta), zero_guess);
}
template void launch_cheb_init<double>(int64_t, const double *, const double *,
                                       double *, double *, double *, double,
                                       bool, cudaStream_t, int);
template void launch_cheb_init<float>(int64_t, const float *, const float *,
                                      float *, float *, float *, double, bool,
                                      cudaStream_t, int);

template <typename T>
void launch_cheb_step(int64_t n, const T *dinv, const T *Ad, T *r, T *d, T *x,
                      double c1, double c2, cudaStream_t s, int nb) {
  count_launch();
  k_cheb_step<T><<<col_grid(n, nb), 256, 0, s>>>(
      n, dinv, Ad, r, d, x, static_cast<T>(c1), static_cast<T>(c2));
}
template void launch_cheb_step<double>(int64_t, const double *, const double *,
                                       double *, double *, double *, double,
                                       double, cudaStream_t, int);
template void launch_cheb_step<float>(int64_t, const float *, const float *,
                                      float *, float *, float *, double, double,
                                      cudaStream_t, int);

}  // namespace tpo
