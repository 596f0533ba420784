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
// About 150 FP operations per element (the dense 24x24 product is 1152):
// x 6, y 12, z 21, Kh 45, and the z transpose with the modulus E_e and the
// sum over the two elements of a face folded into 42 multiply-adds.
//
// Thread (tx, ty) of a 32 x TY CTA owns the grid column (gx, gy) = tile
// origin + (tx, ty): its node, the x-edge to gx+1, the xy-face spanning
// (gx..gx+1, gy..gy+1) and the element column above that face; the CTA
// marches up z.  x-neighbours exchange values by warp shuffles (a warp is
// one tile row), y-neighbours through shared memory with one barrier per
// plane.  Lanes 0 and 31 and row 0 are the halo: the CTA writes the nodes of
// lanes 1..30 and rows 1..TY-1, so every lane's work is the same (lane 31
// only supplies its node to lane 30's edge); the last row (a warp-uniform
// role) also loads the row above the tile so every face of the tile is
// complete.  Node values of the next plane are prefetched into registers
// one plane ahead.  The pipeline: at step p the plane p is loaded into
// edges and faces, element layer p-1 is applied, the faces of plane p-1 are
// complete, and nodes of plane p-2 are written.
#include "modal.cuh"

namespace tpo {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLanesOut = 30;   // written nodes per tile row

// the input vector of dof i: u_i (IN_U) or the Chebyshev start from a zero
// guess, invtheta * dinv_i * b_i (IN_CHEB)
template <typename T, int IN>
__device__ __forceinline__ T input_value(const ApplyArgs<T> &a, int64_t i) {
  if (IN == IN_CHEB) return a.invtheta * (__ldg(a.dinv + i) * __ldg(a.b + i));
  return __ldg(a.u + i);
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

// six values per thread in shared memory with 16-byte accesses: FP32 as one
// float4 (v0, w0, v1, w1) and one float2 (v2, w2) per lane; FP64 as three
// double2 (v_c, w_c)
template <typename T>
struct Six;

template <>
struct Six<float> {
  float4 *a;   // [row][32]
  float2 *b;
  __device__ __forceinline__ void put(int row, int lane, const float (&v)[3],
                                      const float (&w)[3]) const {
    a[row * 32 + lane] = make_float4(v[0], w[0], v[1], w[1]);
    b[row * 32 + lane] = make_float2(v[2], w[2]);
  }
  __device__ __forceinline__ void get(int row, int lane, float (&v)[3],
                                      float (&w)[3]) const {
    const float4 p = a[row * 32 + lane];
    const float2 q = b[row * 32 + lane];
    v[0] = p.x; w[0] = p.y; v[1] = p.z; w[1] = p.w; v[2] = q.x; w[2] = q.y;
  }
  static constexpr size_t bytes_per_row() { return 32 * (16 + 8); }
  __device__ __forceinline__ void bind(unsigned char *base, int rows) {
    a = reinterpret_cast<float4 *>(base);
    b = reinterpret_cast<float2 *>(base + (size_t)rows * 32 * 16);
  }
};

template <>
struct Six<double> {
  double2 *a;   // [c][row][32]
  int stride;
  __device__ __forceinline__ void put(int row, int lane, const double (&v)[3],
                                      const double (&w)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) a[c * stride + row * 32 + lane] = make_double2(v[c], w[c]);
  }
  __device__ __forceinline__ void get(int row, int lane, double (&v)[3],
                                      double (&w)[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 p = a[c * stride + row * 32 + lane];
      v[c] = p.x;
      w[c] = p.y;
    }
  }
  static constexpr size_t bytes_per_row() { return 32 * 3 * 16; }
  __device__ __forceinline__ void bind(unsigned char *base, int rows) {
    a = reinterpret_cast<double2 *>(base);
    stride = rows * 32;
  }
};

// COLS: a block of columns, blockIdx.z = column * nchunk + z chunk, the
// column selecting u, b, y, y2 (stride ld).  The single-column
// instantiation reads the parameters in place.
template <typename T, int TY, int IN, int OUT, bool COLS>
__global__ void __launch_bounds__(32 * TY, sizeof(T) == 4 ? 2 : 1)
    k_apply_staged(int nelx, int nely, int nelz, int zchunk,
                   const T *__restrict__ E, const uint8_t *__restrict__ fix,
                   const ApplyArgs<T> args_in, const Kh<T> kh) {
  constexpr bool kNeedU = OUT == OUT_CHEB2 || OUT == OUT_POST0 || OUT == OUT_POST1;
  const int Nx = nelx + 1, Ny = nely + 1, Nz = nelz + 1;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int gx = (int)blockIdx.x * kLanesOut - 1 + tx;
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
  const bool lastrow = (ty == TY - 1);   // warp-uniform

  // plane-invariant per-thread offsets and predicates
  const bool xin = gx >= 0 && gx < Nx;
  const bool nin = xin && gy >= 0 && gy < Ny;
  const bool nin2 = lastrow && xin && gy + 1 < Ny;
  const bool exy = gx >= 0 && gx < nelx && gy >= 0 && gy < nely;
  const bool own = tx >= 1 && tx <= kLanesOut && ty >= 1 && nin;
  const int NP = Nx * Ny, EP = nelx * nely;
  const int nofs = nin ? gy * Nx + gx : 0;
  const int nofs2 = nin2 ? (gy + 1) * Nx + gx : 0;
  const int eofs = exy ? gy * nelx + gx : 0;

  // dynamic shared memory: se = x-edge (s, d) per row plus the row above
  // the tile, sc = edge contributions of the upper row of a face (row index
  // ty + 1 written by row ty), both double-buffered by plane parity
  // (rows buf * kRows + r of one array per buffer pair)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kRows = TY + 1;
  Six<T> se, sc;
  se.bind(smem_raw, 2 * kRows);
  sc.bind(smem_raw + 2 * kRows * Six<T>::bytes_per_row(), 2 * kRows);

  // prefetched next plane: own node, the row-above node (last row), the
  // fixed-component bits and the modulus of the element layer below it
  T pu[3] = {T(0), T(0), T(0)}, pq[3] = {T(0), T(0), T(0)};
  unsigned pf = 0u, pf2 = 0u;
  T pE = T(0);
  auto fetch = [&](int z) {   // z is uniform over the CTA
    // fresh zeros every plane let the loads target renamed registers
    pf = pf2 = 0u;
#pragma unroll
    for (int c = 0; c < 3; ++c) pu[c] = pq[c] = T(0);
    pE = T(0);
    if (z >= 0 && z < Nz) {
      const int n = nofs + z * NP;
      if (nin) {
        pf = __ldg(fix + n);
#pragma unroll
        for (int c = 0; c < 3; ++c) pu[c] = input_value<T, IN>(args, 3 * (int64_t)n + c);
      }
      if (nin2) {
        const int n2 = nofs2 + z * NP;
        pf2 = __ldg(fix + n2);
#pragma unroll
        for (int c = 0; c < 3; ++c) pq[c] = input_value<T, IN>(args, 3 * (int64_t)n2 + c);
      }
    }
    const int ez = z - 1;
    if (exy && ez >= 0 && ez < nelz) pE = __ldg(E + eofs + ez * EP);
  };

  T FA[4][3], FB[4][3], CA[4][3], CB[4][3], les[3], led[3];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) FA[m][c] = FB[m][c] = CA[m][c] = CB[m][c] = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) les[c] = led[c] = T(0);
  unsigned fpipe = 0u;   // fixed bits of the last three planes, 8 bits each

  // one step of the z-march at plane p: Fprev = faces of plane p-1 (in),
  // Fp = faces of plane p (out), ctop = contributions of element layer p-2
  // to face p-1 (in), top = those of layer p-1 to face p (out)
  auto step = [&](int p, const T(&Fprev)[4][3], T(&Fp)[4][3], const T(&ctop)[4][3],
                  T(&top)[4][3]) {
    T cu[3], cq[3];
    const unsigned f = pf;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cu[c] = ((f >> c) & 1u) ? T(0) : pu[c];
      cq[c] = ((pf2 >> c) & 1u) ? T(0) : pq[c];
    }
    const T Ee = pE;
    fpipe = (fpipe << 8) | f;
    if (p + 1 <= ze) fetch(p + 1);
    const int rb = (p & 1) * kRows, rb1 = kRows - rb;   // this / the other buffer

    // ---- x-edges of plane p (s = u(x+1) + u(x), d = u(x+1) - u(x)) and
    // the xy-faces: modes (1, x, y, xy)
    if (p <= ze) {
      T s0[3], d0[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T r = __shfl_down_sync(kFull, cu[c], 1);
        s0[c] = r + cu[c];
        d0[c] = r - cu[c];
      }
      se.put(rb + ty, tx, s0, d0);
      if (lastrow) {
        T s2[3], d2[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T r = __shfl_down_sync(kFull, cq[c], 1);
          s2[c] = r + cq[c];
          d2[c] = r - cq[c];
        }
        se.put(rb + TY, tx, s2, d2);
      }
      __syncthreads();
      T s1[3], d1[3];
      se.get(rb + ty + 1, tx, s1, d1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Fp[0][c] = s0[c] + s1[c];
        Fp[1][c] = d0[c] + d1[c];
        Fp[2][c] = s1[c] - s0[c];
        Fp[3][c] = d1[c] - d0[c];
      }
    } else {
      __syncthreads();
    }

    // ---- nodes of plane p-2: complete the edge (the face of row ty-1
    // left its part in sc row ty), transpose the x stage
    if (p - 2 >= zs && p - 2 < ze) {
      T gs[3], gd[3], val[3];
      sc.get(rb1 + ty, tx, gs, gd);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T es = les[c] + gs[c], ed = led[c] + gd[c];
        const T right = es + ed;
        const T left = __shfl_up_sync(kFull, right, 1);
        val[c] = (es - ed) + left;
      }
      if (own) {
        const int64_t n = nofs + (int64_t)(p - 2) * NP;
        const unsigned fo = (fpipe >> 16) & 0xffu;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const bool fixed = (fo >> c) & 1u;
          // the input is needed on fixed dofs (identity rows) and by the
          // Chebyshev epilogues
          const T uv = (kNeedU || fixed) ? input_value<T, IN>(args, 3 * n + c) : T(0);
          finish_dof<T, OUT>(args, 3 * n + c, fixed ? uv : val[c], uv);
        }
      }
    }

    // ---- element layer p-1 between faces p-1 (Fprev) and p (Fp); the face
    // of plane p-1 is then complete: G = ctop + bottom contributions
    T G[4][3];
    if (p - 1 >= zs - 1 && p - 1 < ze) {
      T v[8][3], o[8][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        v[0][c] = T(0);   // rigid translation: not coupled
#pragma unroll
        for (int m = 1; m < 4; ++m) v[m][c] = Fp[m][c] + Fprev[m][c];
#pragma unroll
        for (int m = 0; m < 4; ++m) v[m + 4][c] = Fp[m][c] - Fprev[m][c];
      }
      modal_couple(v, o, kh);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        top[0][c] = Ee * o[4][c];
        G[0][c] = fma(-Ee, o[4][c], ctop[0][c]);
#pragma unroll
        for (int m = 1; m < 4; ++m) {
          const T a = Ee * o[m][c];
          top[m][c] = fma(Ee, o[m + 4][c], a);
          G[m][c] = fma(-Ee, o[m + 4][c], ctop[m][c] + a);
        }
      }
    } else {
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          top[m][c] = T(0);
          G[m][c] = ctop[m][c];
        }
    }

    // ---- transpose the y stage of face p-1: the lower edge (own row) keeps
    // its part in registers, the upper edge's part goes to sc row ty + 1
    T gs[3], gd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      les[c] = G[0][c] - G[2][c];
      led[c] = G[1][c] - G[3][c];
      gs[c] = G[0][c] + G[2][c];
      gd[c] = G[1][c] + G[3][c];
    }
    sc.put(rb + ty + 1, tx, gs, gd);
  };

  fetch(zs - 1);
  // two steps per trip with the state arrays swapping roles, so nothing is
  // copied between planes
  for (int p = zs - 1; p <= ze + 1; p += 2) {
    step(p, FA, FB, CA, CB);
    if (p + 1 <= ze + 1) step(p + 1, FB, FA, CB, CA);
  }
}

constexpr int kTY = 8;

template <typename T>
size_t staged_smem() {
  return 4 * Six<T>::bytes_per_row() * (kTY + 1);
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

// grid of the staged kernel: 30 x (kTY-1) owned node columns per CTA, and z
// chunks that fill whole waves of co-resident CTAs (a partial last wave
// idles SMs for the length of a chunk; each chunk recomputes one element
// layer and two face planes)
template <typename T>
void staged_grid(const Ctx &c, int nb, dim3 &grid, int &zchunk) {
  const int Nx = c.nel[0] + 1, Ny = c.nel[1] + 1, Nz = c.nel[2] + 1;
  const int gx = (Nx + kLanesOut - 1) / kLanesOut, gy = (Ny + kTY - 2) / (kTY - 1);
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
