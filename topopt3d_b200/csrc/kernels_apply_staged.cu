// Fine-level matrix-free stiffness operator, staged form.
//
//   y = M K(rho) M u + (1 - M) u          (MODE 0)
//   y = b - [M K(rho) M u + (1 - M) u]    (MODE 1)
//
// K = sum_e E_e K0 (FEAnalysis.cpp:443-468), Dirichlet rows/columns replaced
// by identity (MatZeroRowsColumns, FEAnalysis.cpp:473); M masks the fixed
// components.  u, y, b are interleaved per node (dof 3n+c), E per element.
//
// The element matvec is y_e = T^T Kh T u_e in the 2x2x2 Hadamard basis
// (tpo_internal.h).  T factorises into an x, a y and a z butterfly, and on a
// structured grid the x butterfly of one x-edge is shared by the 4 elements
// around that edge and the y butterfly of one xy-face by the 2 elements
// above and below it.  So each stage is computed once per grid item:
//
//   node u  --x-->  x-edge (s, d)  --y-->  xy-face (4 modes)  --z-->  element
//   (7 modes) -> E Kh -> element --z^T--> face contributions, summed over the
//   two elements sharing the face --y^T--> edge contributions, summed over
//   the two faces sharing the edge --x^T--> node contributions, summed over
//   the two edges sharing the node.
//
// This needs ~165 FP operations per element instead of ~210 for a separate
// butterfly per element (and 1152 for the dense 24x24 product).
//
// Thread (tx, ty) of a 32 x TY CTA owns the grid column (gx, gy) = tile
// origin + (tx, ty): its node, the x-edge to gx+1, the xy-face spanning
// (gx..gx+1, gy..gy+1) and the element column above that face; the CTA
// marches up z.  x-neighbours exchange values by warp shuffles (a warp is
// one tile row), y-neighbours through shared memory with one barrier per
// plane.  Lane 0 and row 0 are the halo: the CTA writes nodes tx >= 1,
// ty >= 1.  Lane 31 and row TY-1 load one extra node (column/row) so every
// face of the tile is complete.  Node values of the next plane are
// prefetched into registers one plane ahead.  The pipeline: at step p the
// plane p is loaded into edges and faces, element layer p-1 is applied, the
// faces of plane p-1 are complete, and nodes of plane p-2 are written.
#include "modal.cuh"

namespace tpo {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <typename T>
struct NodeReg {
  T v[3];
  unsigned f;
};

// the input vector of dof i: u_i (IN_U) or the Chebyshev start from a zero
// guess, invtheta * dinv_i * b_i (IN_CHEB)
template <typename T, int IN>
__device__ __forceinline__ T input_value(const ApplyArgs<T> &a, int64_t i) {
  if (IN == IN_CHEB) return a.invtheta * (__ldg(a.dinv + i) * __ldg(a.b + i));
  return __ldg(a.u + i);
}

template <typename T, int IN>
__device__ __forceinline__ void fetch_node(const ApplyArgs<T> &a,
                                           const uint8_t *__restrict__ fix,
                                           int gx, int gy, int z, int Nx, int Ny,
                                           int Nz, NodeReg<T> &r) {
  if (gx >= 0 && gx < Nx && gy >= 0 && gy < Ny && z >= 0 && z < Nz) {
    const int n = (z * Ny + gy) * Nx + gx;
    r.f = __ldg(fix + n);
    r.v[0] = input_value<T, IN>(a, 3 * n);
    r.v[1] = input_value<T, IN>(a, 3 * n + 1);
    r.v[2] = input_value<T, IN>(a, 3 * n + 2);
  } else {
    r.f = 7u;   // outside the mesh: contributes zero
    r.v[0] = r.v[1] = r.v[2] = T(0);
  }
}

// epilogue of dof i with Au_i = (M K M u + (1-M) u)_i and u_i the input:
//   OUT_Y     y = Au
//   OUT_RESID y = b - Au
//   OUT_CHEB2 Chebyshev(2) from a zero guess, input d0 = invtheta dinv b:
//             r1 = dinv (b - Au); d1 = c1 d0 + c2 r1; y = d0 + d1
//   OUT_POST0 first Chebyshev step from x = u:  d0 = invtheta dinv (b - Au);
//             y = d0, y2 = u + d0
//   OUT_POST1 second step, input d0 = u (so r0 = theta d0):
//             d1 = c1 d0 + c2 (theta d0 - dinv Au); y = x1 + d1 (x1 = y2)
template <typename T, int OUT>
__device__ __forceinline__ void finish_dof(const ApplyArgs<T> &a, int64_t i,
                                           T Au, T u) {
  if (OUT == OUT_Y) {
    a.y[i] = Au;
  } else if (OUT == OUT_RESID) {
    a.y[i] = __ldg(a.b + i) - Au;
  } else if (OUT == OUT_CHEB2) {
    const T di = __ldg(a.dinv + i), bi = __ldg(a.b + i);
    const T r1 = di * bi - di * Au;
    a.y[i] = u + (a.c1 * u + a.c2 * r1);
  } else if (OUT == OUT_POST0) {
    const T d0 = a.invtheta * (__ldg(a.dinv + i) * (__ldg(a.b + i) - Au));
    a.y[i] = d0;
    a.y2[i] = u + d0;
  } else {   // OUT_POST1
    const T r1 = a.theta * u - __ldg(a.dinv + i) * Au;
    a.y[i] = a.y2[i] + (a.c1 * u + a.c2 * r1);
  }
}

template <typename T>
__device__ __forceinline__ T masked(const NodeReg<T> &r, int c) {
  return ((r.f >> c) & 1u) ? T(0) : r.v[c];
}

// COLS: a block of columns, blockIdx.z = column * nchunk + z chunk, the
// column selecting u, b, y, y2 (stride ld).  The single-column
// instantiation reads the parameters in place.
template <typename T, int TY, int IN, int OUT, bool COLS>
__global__ void __launch_bounds__(32 * TY)
    k_apply_staged(int nelx, int nely, int nelz, int zchunk,
                   const T *__restrict__ E, const uint8_t *__restrict__ fix,
                   const ApplyArgs<T> args_in, const Kh<T> kh) {
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int gx = (int)blockIdx.x * 31 - 1 + tx;
  const int gy = (int)blockIdx.y * (TY - 1) - 1 + ty;
  int zs;
  ApplyArgs<T> args_col;
  if (COLS) {
    const int col = (int)blockIdx.z / args_in.nchunk;
    zs = ((int)blockIdx.z - col * args_in.nchunk) * zchunk;
    args_col = args_in;
    const int64_t o = col * args_in.ld;
    if (args_col.u) args_col.u += o;
    if (args_col.b) args_col.b += o;
    args_col.y += o;
    if (args_col.y2) args_col.y2 += o;
  } else {
    zs = (int)blockIdx.z * zchunk;
  }
  const ApplyArgs<T> &args = COLS ? args_col : args_in;
  const int ze = min(zs + zchunk, Nz);
  const bool lane31 = (tx == 31);
  const bool lastrow = (ty == TY - 1);
  const bool exy = gx >= 0 && gx < nelx && gy >= 0 && gy < nely;

  // dynamic shared memory (the FP64 tiles exceed the 48 KB static limit):
  // se = x-edge (s, d) per row plus the extra row, sc = upper-edge
  // contributions, both double-buffered by plane parity
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*se)[6][TY + 1][32] = reinterpret_cast<T(*)[6][TY + 1][32]>(smem_raw);
  T(*sc)[6][TY][32] = reinterpret_cast<T(*)[6][TY][32]>(
      smem_raw + sizeof(T) * 2 * 6 * (TY + 1) * 32);

  NodeReg<T> n0, n1, n2, n3;   // next plane: own, +x, +y, +x+y
  n1.f = n2.f = n3.f = 7u;
#pragma unroll
  for (int c = 0; c < 3; ++c) n1.v[c] = n2.v[c] = n3.v[c] = T(0);
  T nE = T(0);
  auto fetch = [&](int z) {
    fetch_node<T, IN>(args, fix, gx, gy, z, Nx, Ny, Nz, n0);
    if (lane31) fetch_node<T, IN>(args, fix, gx + 1, gy, z, Nx, Ny, Nz, n1);
    if (lastrow) {
      fetch_node<T, IN>(args, fix, gx, gy + 1, z, Nx, Ny, Nz, n2);
      if (lane31) fetch_node<T, IN>(args, fix, gx + 1, gy + 1, z, Nx, Ny, Nz, n3);
    }
    // element layer z-1 is applied when plane z is the top plane
    const int ez = z - 1;
    nE = (exy && ez >= 0 && ez < nelz)
             ? __ldg(E + (ez * nely + gy) * nelx + gx)
             : T(0);
  };

  T Fprev[4][3], ctop[4][3], les[3], led[3];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) Fprev[m][c] = ctop[m][c] = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) les[c] = led[c] = T(0);

  fetch(zs - 1);
#pragma unroll 2
  for (int p = zs - 1; p <= ze + 1; ++p) {
    // ---- plane p: take the prefetched values, prefetch plane p + 1
    T cu[3], cr[3], cq[3], crq[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cu[c] = masked(n0, c);
      cr[c] = masked(n1, c);
      cq[c] = masked(n2, c);
      crq[c] = masked(n3, c);
    }
    const T Ee = nE;
    if (p + 1 <= ze + 1) fetch(p + 1);
    const int buf = p & 1;

    // ---- x-edges of plane p: s = u(x+1) + u(x), d = u(x+1) - u(x)
    T s0[3], d0[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T r = __shfl_down_sync(kFull, cu[c], 1);
      if (lane31) r = cr[c];
      s0[c] = r + cu[c];
      d0[c] = r - cu[c];
      se[buf][c][ty][tx] = s0[c];
      se[buf][3 + c][ty][tx] = d0[c];
    }
    if (lastrow) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T r = __shfl_down_sync(kFull, cq[c], 1);
        if (lane31) r = crq[c];
        se[buf][c][TY][tx] = r + cq[c];
        se[buf][3 + c][TY][tx] = r - cq[c];
      }
    }
    __syncthreads();

    // ---- xy-face of plane p: modes (1, x, y, xy)
    T Fp[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T s1 = se[buf][c][ty + 1][tx], d1 = se[buf][3 + c][ty + 1][tx];
      Fp[0][c] = s0[c] + s1;
      Fp[1][c] = d0[c] + d1;
      Fp[2][c] = s1 - s0[c];
      Fp[3][c] = d1 - d0[c];
    }

    // ---- nodes of plane p-2: complete the edge, transpose the x stage
    if (p - 2 >= zs && p - 2 < ze) {
      T val[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T es = les[c], ed = led[c];
        if (ty > 0) {
          es += sc[buf ^ 1][c][ty - 1][tx];
          ed += sc[buf ^ 1][3 + c][ty - 1][tx];
        }
        const T right = es + ed;
        const T left = __shfl_up_sync(kFull, right, 1);
        val[c] = (es - ed) + left;
      }
      if (tx >= 1 && ty >= 1 && gx < Nx && gy < Ny) {
        const int n = ((p - 2) * Ny + gy) * Nx + gx;
        const unsigned f = __ldg(fix + n);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          // the input is needed for fixed dofs (identity rows) and by the
          // Chebyshev epilogues
          const bool need_u = ((f >> c) & 1u) || OUT == OUT_CHEB2 ||
                              OUT == OUT_POST0 || OUT == OUT_POST1;
          const T uv = need_u ? input_value<T, IN>(args, 3 * n + c) : T(0);
          const T Au = ((f >> c) & 1u) ? uv : val[c];
          finish_dof<T, OUT>(args, 3 * n + c, Au, uv);
        }
      }
    }

    // ---- element layer p-1 between faces p-1 (Fprev) and p (Fp)
    T top[4][3], bot[4][3];
    if (p - 1 >= zs - 1 && p - 1 < ze) {
      T v[8][3], o[8][3];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v[m][c] = (Fp[m][c] + Fprev[m][c]) * Ee;
          v[m + 4][c] = (Fp[m][c] - Fprev[m][c]) * Ee;
        }
      modal_couple(v, o, kh);
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          top[m][c] = o[m][c] + o[m + 4][c];
          bot[m][c] = o[m][c] - o[m + 4][c];
        }
    } else {
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) top[m][c] = bot[m][c] = T(0);
    }

    // ---- face of plane p-1 is complete: transpose the y stage
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T G0 = ctop[0][c] + bot[0][c], G1 = ctop[1][c] + bot[1][c];
      const T G2 = ctop[2][c] + bot[2][c], G3 = ctop[3][c] + bot[3][c];
      les[c] = G0 - G2;
      led[c] = G1 - G3;
      sc[buf][c][ty][tx] = G0 + G2;
      sc[buf][3 + c][ty][tx] = G1 + G3;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ctop[m][c] = top[m][c];
        Fprev[m][c] = Fp[m][c];
      }
  }
}

constexpr int kTY = 8;

template <typename T>
size_t staged_smem() {
  return sizeof(T) * 2 * 6 * (2 * kTY + 1) * 32;
}

template <typename T, int IN, int OUT>
void set_smem_attr() {
  cudaFuncSetAttribute(k_apply_staged<T, kTY, IN, OUT, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)staged_smem<T>());
  cudaFuncSetAttribute(k_apply_staged<T, kTY, IN, OUT, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)staged_smem<T>());
}

// grid of the staged kernel: 31 x (kTY-1) owned node columns per CTA, and z
// chunks that fill whole waves of co-resident CTAs (a partial last wave
// idles SMs for the length of a chunk; each chunk costs 3 extra planes)
template <typename T>
void staged_grid(const Ctx &c, int nb, dim3 &grid, int &zchunk) {
  const int Nx = c.nel[0] + 1, Ny = c.nel[1] + 1, Nz = c.nel[2] + 1;
  const int gx = (Nx + 30) / 31, gy = (Ny + kTY - 2) / (kTY - 1);
  const int dev = c.device & 63;
  static unsigned long long attr_set = 0;   // bit per device
  static int slots_cache[64] = {0};
  if (!((attr_set >> dev) & 1ull)) {
    // opt in to > 48 KB of dynamic shared memory (the FP64 tiles)
    set_smem_attr<T, IN_U, OUT_Y>();
    set_smem_attr<T, IN_U, OUT_RESID>();
    set_smem_attr<T, IN_CHEB, OUT_CHEB2>();
    set_smem_attr<T, IN_U, OUT_POST0>();
    set_smem_attr<T, IN_U, OUT_POST1>();
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_apply_staged<T, kTY, IN_CHEB, OUT_CHEB2, true>, 32 * kTY,
        staged_smem<T>());
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    slots_cache[dev] = std::max(1, per_sm) * std::max(1, sms);
    attr_set |= 1ull << dev;
  }
  const int slots = slots_cache[dev], tiles = gx * gy * nb;
  int chunks = 1;
  for (int w = 1; w <= 8; ++w) {
    const int ch = (w * slots) / tiles;
    if (ch >= 1 && (double)(ch * tiles) >= 0.9 * w * slots) {
      chunks = ch;
      break;
    }
    chunks = std::max(1, ch);
  }
  const int maxc = std::max(1, Nz / 8);   // keep >= 8 planes per chunk
  if (chunks > maxc) chunks = maxc;
  zchunk = (Nz + chunks - 1) / chunks;
  grid = dim3(gx, gy, nb * ((Nz + zchunk - 1) / zchunk));
}

template <typename T, int IN, int OUT>
void launch_mode(const Ctx &c, const T *E, const ApplyArgs<T> &args_in,
                 cudaStream_t s, int nb) {
  dim3 grid;
  int zchunk = 0;
  staged_grid<T>(c, nb, grid, zchunk);
  ApplyArgs<T> args = args_in;
  args.ld = 3 * c.nn;
  args.nchunk = (int)grid.z / nb;
  const Kh<T> &kh = *reinterpret_cast<const Kh<T> *>(
      sizeof(T) == 8 ? (const void *)&c.kh64 : (const void *)&c.kh32);
  count_launch();
  if (nb == 1)
    k_apply_staged<T, kTY, IN, OUT, false><<<grid, dim3(32, kTY), staged_smem<T>(), s>>>(
        c.nel[0], c.nel[1], c.nel[2], zchunk, E, c.idm, args, kh);
  else
    k_apply_staged<T, kTY, IN, OUT, true><<<grid, dim3(32, kTY), staged_smem<T>(), s>>>(
        c.nel[0], c.nel[1], c.nel[2], zchunk, E, c.idm, args, kh);
}

}  // namespace

template <typename T>
void launch_apply_fine(const Ctx &c, const T *E, const T *u, const T *b, T *y,
                       cudaStream_t s, int nb) {
  ApplyArgs<T> a{};
  a.u = u;
  a.b = b;
  a.y = y;
  if (b)
    launch_mode<T, IN_U, OUT_RESID>(c, E, a, s, nb);
  else
    launch_mode<T, IN_U, OUT_Y>(c, E, a, s, nb);
}

template <typename T>
void launch_apply_fused(const Ctx &c, const T *E, int in, int out,
                        const ApplyArgs<T> &args, cudaStream_t s, int nb) {
  if (in == IN_CHEB && out == OUT_CHEB2)
    launch_mode<T, IN_CHEB, OUT_CHEB2>(c, E, args, s, nb);
  else if (in == IN_U && out == OUT_POST0)
    launch_mode<T, IN_U, OUT_POST0>(c, E, args, s, nb);
  else if (in == IN_U && out == OUT_POST1)
    launch_mode<T, IN_U, OUT_POST1>(c, E, args, s, nb);
  else if (in == IN_U && out == OUT_RESID)
    launch_mode<T, IN_U, OUT_RESID>(c, E, args, s, nb);
  else
    launch_mode<T, IN_U, OUT_Y>(c, E, args, s, nb);
}

template void launch_apply_fine<double>(const Ctx &, const double *,
                                        const double *, const double *,
                                        double *, cudaStream_t, int);
template void launch_apply_fine<float>(const Ctx &, const float *,
                                       const float *, const float *, float *,
                                       cudaStream_t, int);
template void launch_apply_fused<double>(const Ctx &, const double *, int, int,
                                         const ApplyArgs<double> &,
                                         cudaStream_t, int);
template void launch_apply_fused<float>(const Ctx &, const float *, int, int,
                                        const ApplyArgs<float> &, cudaStream_t,
                                        int);

}  // namespace tpo
