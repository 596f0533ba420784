// Fine-level matrix-free stiffness operator and its set-up companions.
//
// apply: y = M K(rho) M u + (1 - M) u, K = sum_e E_e K0 (FEAnalysis.cpp:
// 443-468) with the Dirichlet rows/columns replaced by identity
// (MatZeroRowsColumns, :473).  M is the per-node fixed-component mask.
//
// Layout in HBM: u, y interleaved per node (dof 3n+c, reference order);
// E per element in reference element order; fix as one byte per node.
//
// Kernel structure: a CTA owns a TX x TY column of elements and marches up
// the z axis one element layer at a time.  Each step stages the next node
// plane of u (with a one-node halo) in shared memory with row-contiguous,
// coalesced loads, every thread applies E_e K0 to its element in the modal
// basis (~210 FP ops instead of the dense 1152), and the element results
// are gathered per node with warp shuffles along x and one shared-memory
// exchange along y -- no atomics.  Threads on
// the low x/y edge of the tile only supply halo elements, so a CTA owns
// (TX-1) x (TY-1) output node columns.  The contribution of the element
// layer below each node plane is carried in registers between steps.
#include "modal.cuh"

namespace tpo {

namespace {

constexpr int kTX = 32;
constexpr int kTY = 8;

template <typename T, bool RESID>
__global__ void __launch_bounds__(kTX *kTY)
    k_apply_fine(int nelx, int nely, int nelz, int zchunk,
                 const T *__restrict__ E, const uint8_t *__restrict__ fix,
                 const T *__restrict__ u, const T *__restrict__ b,
                 T *__restrict__ y, const Kh<T> kh) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  __shared__ T su[2][3][kTY + 1][kTX + 1];
  __shared__ T sy[6][kTY][kTX];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
  const int X0 = blockIdx.x * (kTX - 1) - 1, Y0 = blockIdx.y * (kTY - 1) - 1;
  const int zs = blockIdx.z * zchunk;
  const int ze = min(zs + zchunk, Nz);
  const int ex = X0 + tx, ey = Y0 + ty;
  const bool exy = ex >= 0 && ex < nelx && ey >= 0 && ey < nely;
  const bool owner = tx >= 1 && ty >= 1 && ex < Nx && ey < Ny;
  const int64_t plane = (int64_t)Nx * Ny;

  auto load_plane = [&](int z, int buf) {
    for (int k = tid; k < 3 * (kTX + 1) * (kTY + 1); k += kTX * kTY) {
      const int row = k / (3 * (kTX + 1));
      const int rem = k - row * 3 * (kTX + 1);
      const int xi = rem / 3, c = rem - 3 * xi;
      const int gx = X0 + xi, gy = Y0 + row;
      T v = T(0);
      if (z >= 0 && z < Nz && gx >= 0 && gx < Nx && gy >= 0 && gy < Ny) {
        const int64_t n = z * plane + (int64_t)gy * Nx + gx;
        if (!((__ldg(fix + n) >> c) & 1)) v = __ldg(u + 3 * n + c);
      }
      su[buf][c][row][xi] = v;
    }
  };

  T acc[3] = {T(0), T(0), T(0)};
  load_plane(zs - 1, (zs - 1) & 1);
  for (int ez = zs - 1; ez < ze; ++ez) {
    load_plane(ez + 1, (ez + 1) & 1);
    __syncthreads();
    T v[8][3];
    const int pb = ez & 1, pt = (ez + 1) & 1;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int bx = l & 1, by = (l >> 1) & 1, p = (l >> 2) ? pt : pb;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[l][c] = su[p][c][ty + by][tx + bx];
    }
    const bool ev = exy && ez >= 0 && ez < nelz;
    const T Ee = ev ? __ldg(E + ((int64_t)ez * nely + ey) * nelx + ex) : T(0);
    element_apply(v, Ee, kh);
    // Gather per node (tx, ty) = corner 0/4 of its own element, corner 1/5 of
    // the -x element, 2/6 of the -y element, 3/7 of the -x-y element.  A warp
    // is one tile row, so the -x contributions move by shuffle; each thread
    // pre-sums (own 2/6 + left neighbour's 3/7) for the row above and passes
    // it through shared memory.  Lane 0 receives its own value from the
    // shuffle; lane-0 results only reach non-owner threads.
    T bot[3], top[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T l3 = __shfl_up_sync(0xffffffffu, v[3][c], 1);
      const T l7 = __shfl_up_sync(0xffffffffu, v[7][c], 1);
      const T l1 = __shfl_up_sync(0xffffffffu, v[1][c], 1);
      const T l5 = __shfl_up_sync(0xffffffffu, v[5][c], 1);
      sy[c][ty][tx] = v[2][c] + l3;
      sy[3 + c][ty][tx] = v[6][c] + l7;
      bot[c] = v[0][c] + l1;
      top[c] = v[4][c] + l5;
    }
    __syncthreads();
    if (owner) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bot[c] += sy[c][ty - 1][tx];
        top[c] += sy[3 + c][ty - 1][tx];
      }
      if (ez >= zs) {
        const int64_t n = ez * plane + (int64_t)ey * Nx + ex;
        const uint8_t f = __ldg(fix + n);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T val = acc[c] + bot[c];
          if ((f >> c) & 1) val = __ldg(u + 3 * n + c);
          if (RESID) val = __ldg(b + 3 * n + c) - val;
          y[3 * n + c] = val;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = top[c];
    }
  }
}

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

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

template <typename T>
void launch_apply_fine(const Ctx &c, const T *E, const T *u, const T *b, T *y,
                       cudaStream_t s) {
  count_launch();
  const int Nx = c.nel[0] + 1, Ny = c.nel[1] + 1, Nz = c.nel[2] + 1;
  dim3 block(kTX, kTY);
  const int gx = (Nx + kTX - 2) / (kTX - 1), gy = (Ny + kTY - 2) / (kTY - 1);
  // z chunks: enough CTAs for ~4 per SM, each marching >= 8 planes
  int chunks = (4 * 148 + gx * gy - 1) / (gx * gy);
  if (chunks > (Nz + 7) / 8) chunks = (Nz + 7) / 8;
  if (chunks < 1) chunks = 1;
  const int zchunk = (Nz + chunks - 1) / chunks;
  dim3 grid(gx, gy, (Nz + zchunk - 1) / zchunk);
  const Kh<T> &kh = *reinterpret_cast<const Kh<T> *>(
      sizeof(T) == 8 ? (const void *)&c.kh64 : (const void *)&c.kh32);
  if (b)
    k_apply_fine<T, true><<<grid, block, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                 zchunk, E, c.fix, u, b, y, kh);
  else
    k_apply_fine<T, false><<<grid, block, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                  zchunk, E, c.fix, u, b, y, kh);
}

template void launch_apply_fine<double>(const Ctx &, const double *,
                                        const double *, const double *,
                                        double *, cudaStream_t);
template void launch_apply_fine<float>(const Ctx &, const float *,
                                       const float *, const float *, float *,
                                       cudaStream_t);

void launch_fine_diag(const Ctx &c, double *dinv64, float *dinv32,
                      cudaStream_t s) {
  count_launch();
  k_fine_diag<<<grid_for(c.nn, 256), 256, 0, s>>>(c.nel[0], c.nel[1], c.nel[2],
                                                   c.E64, c.fix, c.kd64, dinv64,
                                                   dinv32);
}

void launch_fine_stencil(const Ctx &c, double *S, cudaStream_t s) {
  count_launch();
  k_fine_stencil<<<grid_for(c.nn * 27, 256), 256, 0, s>>>(
      c.nel[0], c.nel[1], c.nel[2], c.E64, c.fix, c.K0lex, S);
}
}  // namespace tpo
