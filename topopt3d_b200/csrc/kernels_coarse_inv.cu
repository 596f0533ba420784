// Dense inverse of the coarsest-level operator, in place, by blocked
// symmetric sweeps (Gauss-Jordan elimination without pivoting).
//
// The coarsest operator is symmetric positive definite (the Galerkin
// product of the clamped fine operator; the reference factorises it with a
// direct solver, FEAnalysis.cpp:555-573), so every pivot block -- a Schur
// complement -- is SPD and no pivoting is needed.  The V-cycle applies the
// explicit inverse as one bandwidth-parallel matrix-vector product.
//
// The sweep of block K (P = A_KK^-1, F = the column block A_{.K}, G = F P):
//   A_KK <- -P;  A_iK <- G_i;  A_Kj <- G_j^T;  A_ij <- A_ij - G_i F_j^T
// keeps the matrix symmetric, so only the tiles on or below the diagonal
// are updated (the row block K left of the diagonal holds G^T); after every
// block has been swept the matrix is -A^-1, and a last pass negates it and
// fills the upper triangle.  A sweep is two launches: F and G for every row
// block (k_sw_fg), and the rank-64 update of the lower tiles on 64 x 64
// tiles with FP64 tensor-core MMAs (k_sw_update), one CTA of which then
// inverts the next
// diagonal block by scalar Gauss-Jordan with a 4 x 4 block of it in each
// thread's registers (sweep_diag; k_sw_diag for the first block).
#include "tpo_internal.h"

namespace tpo {

namespace {

constexpr int kGB = 64;    // block size (rows / columns of a pivot block)
constexpr int kGT = 256;   // threads per CTA: 16 x 16, 4 x 4 outputs each
#ifndef TPO_SW_MINB
#define TPO_SW_MINB 3
#endif

// D (8 x 8) += A (8 x 4) B (4 x 8) in FP64 on the tensor cores.  Fragments
// (PTX ISA, mma.m8n8k4 .f64): lane = 4 g + q holds A[g][q], B[q][g] and
// D[g][2q], D[g][2q + 1].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// 8-byte asynchronous copy global -> shared; src_bytes 0 fills zeros (the
// source address must still be valid)
__device__ __forceinline__ void cp_async8(double *dst, const double *src, int src_bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// tile_gemm's operands in dynamic shared memory, the whole depth at once:
// Xs[k][i] and, by layout, Ys[k][j] (YT) or Ys[j][k]; rows padded to 68
// doubles so a warp's fragment reads fall on distinct bank pairs
constexpr int kLd = kGB + 4;
constexpr size_t kGemmSmem = 2 * sizeof(double) * kGB * kLd;

// C (M x N, column-major, ldc) = (ACC ? C : 0) + s X Y for M, N <= 64 and a
// depth Kd <= kGB, with X[i][k] = X[k * ldx + i] and Y[k][j] = Y[k * ldy + j]
// (YT) or Y[j * ldy + k].  The operands are staged with asynchronous copies
// and, with ACC, the thread's part of C is read while they are in flight;
// every read of X and Y happens before the first write of C.  8 warps, each
// a 16 x 32 block of the 64 x 64 tile as 2 x 4 tensor-core tiles of 8 x 8.
template <bool ACC, bool YT>
__device__ __forceinline__ void tile_gemm(double *smem, int M, int N, int Kd,
                                          const double *X, int ldx, const double *Y,
                                          int ldy, double *C, int ldc, double s) {
  double *Xs = smem, *Ys = smem + kGB * kLd;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int r0 = (w >> 1) * 16, c0 = (w & 1) * 32;
  __syncthreads();   // the buffers are free (a previous use has finished)
#pragma unroll 4
  for (int e8 = 0; e8 < kGB * kGB / kGT; ++e8) {
    const int e = t + e8 * kGT;
    {
      const int i = e % kGB, k = e / kGB;
      const bool ok = i < M && k < Kd;
      cp_async8(Xs + k * kLd + i, ok ? X + (int64_t)k * ldx + i : X, ok ? 8 : 0);
    }
    if (YT) {
      const int j = e % kGB, k = e / kGB;
      const bool ok = j < N && k < Kd;
      cp_async8(Ys + k * kLd + j, ok ? Y + (int64_t)k * ldy + j : Y, ok ? 8 : 0);
    } else {
      const int k = e % kGB, j = e / kGB;
      const bool ok = j < N && k < Kd;
      cp_async8(Ys + j * kLd + k, ok ? Y + (int64_t)j * ldy + k : Y, ok ? 8 : 0);
    }
  }
  double cv[2][4][2];
  if (ACC) {
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int i = r0 + a * 8 + g, j = c0 + b * 8 + 2 * q + h;
          cv[a][b][h] = (i < M && j < N) ? C[(int64_t)j * ldc + i] : 0.0;
        }
  }
  double acc[2][4][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  cp_async_wait_all();
  __syncthreads();
#pragma unroll 4
  for (int k0 = 0; k0 < kGB; k0 += 4) {
    double av[2], bv[4];
#pragma unroll
    for (int a = 0; a < 2; ++a) av[a] = Xs[(k0 + q) * kLd + r0 + a * 8 + g];
#pragma unroll
    for (int b = 0; b < 4; ++b)
      bv[b] = YT ? Ys[(k0 + q) * kLd + c0 + b * 8 + g] : Ys[(c0 + b * 8 + g) * kLd + k0 + q];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) dmma(acc[a][b], av[a], bv[b]);
  }
  __syncthreads();   // C may alias an operand
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int i = r0 + a * 8 + g;
    if (i >= M) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = c0 + b * 8 + 2 * q + h;
        if (j >= N) continue;
        C[(int64_t)j * ldc + i] = ACC ? fma(s, acc[a][b][h], cv[a][b][h]) : s * acc[a][b][h];
      }
  }
}

// P = A_KK^-1 of the bs x bs diagonal block at (K0, K0) by scalar
// Gauss-Jordan; thread (tx, ty) keeps rows 4tx.. and columns 4ty.. in
// registers, and each step broadcasts the pivot row and column through
// shared memory (double-buffered, one barrier per step).  P goes to the
// workspace (ld kGB) and -P to A.  A pivot that is not positive records
// its global index + 1 in *info (the first one wins).
__device__ __forceinline__ void sweep_diag(int n, double *A, int K0, int bs, double *P,
                                           int *info) {
  __shared__ double rowk[2][kGB], colk[2][kGB];
  const int t = threadIdx.x, tx = t % 16, ty = t / 16;
  const int r0 = tx * 4, c0 = ty * 4;
  double m[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = r0 + a, cc = c0 + b;
      // identity outside the block, so the padding never pivots on zero
      m[a][b] = (r < bs && cc < bs) ? A[(int64_t)(K0 + cc) * n + K0 + r]
                                    : (r == cc ? 1.0 : 0.0);
    }
#pragma unroll 4
  for (int k = 0; k < kGB; ++k) {
    const int buf = k & 1;
    // publish the pivot row (owners: rows 4tx..4tx+3 hold k) and column
    // (the row/column index is selected with unrolled compares so m stays
    // in registers)
    if ((k >> 2) == tx) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (a == (k & 3)) {
#pragma unroll
          for (int b = 0; b < 4; ++b) rowk[buf][c0 + b] = m[a][b];
        }
    }
    if ((k >> 2) == ty) {
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (b == (k & 3)) {
#pragma unroll
          for (int a = 0; a < 4; ++a) colk[buf][r0 + a] = m[a][b];
        }
    }
    __syncthreads();
    const double p = rowk[buf][k];
    const bool ok = p > 0.0 && p < INFINITY;
    if (!ok && t == 0 && k < bs) atomicCAS(info, 0, K0 + k + 1);
    const double ip = ok ? 1.0 / p : 0.0;
    double rk[4], ck[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) rk[b] = rowk[buf][c0 + b] * ip;
#pragma unroll
    for (int a = 0; a < 4; ++a) ck[a] = colk[buf][r0 + a];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int r = r0 + a, cc = c0 + b;
        double v = fma(-ck[a], rk[b], m[a][b]);   // generic entry
        if (r == k) v = rk[b];                     // pivot row: a / p
        if (cc == k) v = (r == k) ? ip : -ck[a] * ip;   // pivot column
        m[a][b] = v;
      }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = r0 + a, cc = c0 + b;
      if (r < bs && cc < bs) {
        P[cc * kGB + r] = m[a][b];
        A[(int64_t)(K0 + cc) * n + K0 + r] = -m[a][b];
      }
    }
}

__global__ void __launch_bounds__(kGT) k_sw_diag(int n, double *A, int K0, int bs,
                                                  double *P, int *info) {
  sweep_diag(n, A, K0, bs, P, info);
}

// CTA I (I != K): F_I = the rows of tile I of the column block K (below the
// diagonal: tile (I, K); above: the transposed tile (K, I) of the row
// block), and G_I = F_I P; both n x bs, column-major
__global__ void __launch_bounds__(kGT, 3) k_sw_fg(int n, const double *A, int K0, int bs,
                                               const double *P, double *F, double *G) {
  const int I = blockIdx.x, i0 = I * kGB;
  if (i0 == K0) return;
  const int rows = min(kGB, n - i0);
  // 16 independent copies per thread, unrolled so the loads overlap
  if (i0 > K0) {
#pragma unroll
    for (int q = 0; q < kGB * kGB / kGT; ++q) {
      const int e = threadIdx.x + q * kGT, i = e % kGB, k = e / kGB;
      if (i < rows && k < bs) F[(int64_t)k * n + i0 + i] = A[(int64_t)(K0 + k) * n + i0 + i];
    }
  } else {
    // A(K0 + k, i0 + i): k fastest for coalesced reads
#pragma unroll
    for (int q = 0; q < kGB * kGB / kGT; ++q) {
      const int e = threadIdx.x + q * kGT, k = e % kGB, i = e / kGB;
      if (i < rows && k < bs) F[(int64_t)k * n + i0 + i] = A[(int64_t)(i0 + i) * n + K0 + k];
    }
  }
  __syncthreads();
  extern __shared__ __align__(16) double gemm_smem[];
  // G_I (rows x bs) = F_I (rows x bs) P (bs x bs); P[k][j] = P[j * kGB + k]
  tile_gemm<false, false>(gemm_smem, rows, bs, bs, F + i0, n, P, kGB, G + i0, n, 1.0);
}

// lower tile (I, J), I >= J: the column block gets G_I, the row block left
// of the diagonal G_J^T, every other tile A_IJ - G_I F_J^T.  The CTA of the
// next diagonal tile (K+1, K+1) runs as block (0, 0), the first one
// dispatched, and after its update inverts that block for the next sweep
// (P and -P as k_sw_diag), so the diagonal inversion overlaps the rest of
// the update instead of running alone between sweeps.
__global__ void __launch_bounds__(kGT, TPO_SW_MINB) k_sw_update(int n, double *A, int K0, int bs,
                                                    const double *F, const double *G,
                                                    double *P, int *info) {
  int I = blockIdx.x, J = blockIdx.y;
  const int Kn = K0 / kGB + 1;   // the next diagonal tile
  const bool look = Kn * kGB < n;
  if (look) {
    if (I == 0 && J == 0) I = J = Kn;
    else if (I == Kn && J == Kn) I = J = 0;
  }
  if (J > I) return;
  const int i0 = I * kGB, j0 = J * kGB;
  const int M = min(kGB, n - i0), N = min(kGB, n - j0);
  if (i0 == K0 && j0 == K0) return;   // the diagonal block: swept already
  if (j0 == K0) {                      // A(i0 + i, K0 + k) = G(i0 + i, k)
    for (int e = threadIdx.x; e < M * bs; e += kGT) {
      const int i = e % M, k = e / M;
      A[(int64_t)(K0 + k) * n + i0 + i] = G[(int64_t)k * n + i0 + i];
    }
    return;
  }
  if (i0 == K0) {                      // A(K0 + k, j0 + j) = G(j0 + j, k)
    for (int e = threadIdx.x; e < N * bs; e += kGT) {
      const int k = e % bs, j = e / bs;
      A[(int64_t)(j0 + j) * n + K0 + k] = G[(int64_t)k * n + j0 + j];
    }
    return;
  }
  extern __shared__ __align__(16) double gemm_smem[];
  // Y[k][j] = F(j0 + j, k) = F[k * n + j0 + j]
  tile_gemm<true, true>(gemm_smem, M, N, bs, G + i0, n, F + j0, n, A + (int64_t)j0 * n + i0,
                        n, -1.0);
  if (look && I == Kn && J == Kn) {
    __syncthreads();   // the tile's update is visible to the whole CTA
    sweep_diag(n, A, i0, M, P, info);
  }
}

// A <- -A on the lower triangle, mirrored into the upper one
__global__ void k_sw_final(int n, double *A) {
  const int I = blockIdx.x, J = blockIdx.y;
  if (J > I) return;
  const int i0 = I * kGB, j0 = J * kGB;
  const int M = min(kGB, n - i0), N = min(kGB, n - j0);
  for (int e = threadIdx.x; e < M * N; e += blockDim.x) {
    const int i = e % M, j = e / M;
    const int gi = i0 + i, gj = j0 + j;
    if (gi < gj) continue;   // diagonal tiles: the lower half writes both
    const double v = -A[(int64_t)gj * n + gi];
    A[(int64_t)gj * n + gi] = v;
    if (gi != gj) A[(int64_t)gi * n + gj] = v;
  }
}

}  // namespace

size_t coarse_inverse_work(int64_t n) { return 2 * (size_t)n * kGB + kGB * kGB; }

void launch_coarse_inverse(int64_t n64, double *A, double *work, int *info, cudaStream_t s) {
  const int n = (int)n64;
  const int nt = (n + kGB - 1) / kGB;
  double *P = work, *F = work + kGB * kGB, *G = F + (size_t)n * kGB;
  static unsigned long long attr_set = 0;   // bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (!((attr_set >> (dev & 63)) & 1ull)) {
    cudaFuncSetAttribute(k_sw_fg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    cudaFuncSetAttribute(k_sw_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kGemmSmem);
    attr_set |= 1ull << (dev & 63);
  }
  cudaMemsetAsync(info, 0, sizeof(int), s);
  count_launch();
  k_sw_diag<<<1, kGT, 0, s>>>(n, A, 0, std::min(kGB, n), P, info);
  for (int K0 = 0; K0 < n; K0 += kGB) {
    const int bs = std::min(kGB, n - K0);
    count_launch(2);
    k_sw_fg<<<nt, kGT, kGemmSmem, s>>>(n, A, K0, bs, P, F, G);
    k_sw_update<<<dim3(nt, nt), kGT, kGemmSmem, s>>>(n, A, K0, bs, F, G, P, info);
  }
  count_launch();
  k_sw_final<<<dim3(nt, nt), kGT, 0, s>>>(n, A);
}

}  // namespace tpo
