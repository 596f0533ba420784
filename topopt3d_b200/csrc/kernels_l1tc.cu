// Level-1 Galerkin operator A_1 = P^T A_0 P in FP32 on the tensor cores.
//
// The reference forms A_1 with PETSc's Galerkin product (PCMG,
// FEAnalysis.cpp:410-416) and stores it; the stored-stencil form here is
// k_apply_stencil_sym1 (kernels_mg.cu), 117 MB per FP32 apply at
// 192x96x96.  With even fine element counts every level-1 element E holds
// 2x2x2 fine elements i, and P restricted to E is the same trilinear map Q_i
// for every E, so away from the fixed dofs
//   A_1 u = sum_E sum_i E_{E,i} G_i u_E,   G_i = Q_i^T K0 Q_i  (24 x 24),
// with E_{E,i} the fine moduli.  The bytes per apply are the vectors and the
// FP32 moduli, about 20 MB at 192x96x96.
//
// One CTA takes a tile of 16 x 8 level-1 elements and marches through a
// chunk of element planes.  Per plane the 128 element vectors u_E (24 dofs
// each) go to shared memory as the A operand; one tcgen05 MMA (M = 128,
// N = 192, K = 24, kind::tf32, accumulator in TMEM) forms
// D = U [G_0; ...; G_7]^T; the epilogue reads a thread's TMEM row and forms
// y_E = sum_i E_{E,i} D[:, 24i : 24i+24].  Both operands are split into a
// TF32 high part and a TF32 remainder and the MMA runs the products
// hi*hi + lo*hi + hi*lo, so the result carries FP32 accuracy.  Node sums are
// assembled deterministically: x neighbours by warp shuffles, y neighbours
// through shared memory, z neighbours carried in registers from the
// previous plane.  A tile owns the 15 x 7 nodes whose elements are all in
// it; the first element column and row are recomputed by the neighbouring
// tile.  The operand of plane k+1 is gathered while the MMA of plane k runs.
//
// Coarse elements that contain a fixed (identity) fine dof follow the
// general path of the Galerkin product (k_galerkin_general); the nodes next
// to them add a stored correction: their full stencil row (k_galerkin_fine)
// minus the sum above, 27 blocks of 3 x 3.  A small kernel ahead of the
// apply forms C u on those rows (one warp per row) into a dense vector that
// the apply's CTAs holding such nodes add in their epilogue.  The apply is a
// programmatic dependent launch: its CTAs start while the small kernel runs,
// and only the CTAs that read the vector wait for it (griddepcontrol).
#include <algorithm>

#include "fused_out.cuh"
#include "tpo_internal.h"
#include "umma.cuh"

namespace tpo {

namespace {

constexpr int kTX = 16, kTY = 8;                  // element tile
constexpr int kOwnX = kTX - 1, kOwnY = kTY - 1;   // nodes a tile owns
constexpr int kM = kTX * kTY;                     // MMA rows = elements (128)
constexpr int kN = 192;                           // 8 fine elements x 24 dofs
constexpr int kK = 24;                            // dofs of a level-1 element
constexpr int kSBO = (kK / 4) * 128;              // bytes between 8-row groups
constexpr int kTileF = kM * kK;                   // floats of one A operand
constexpr int kBF = kN * kK;                      // floats of one B operand
constexpr int kNX = kTX + 1, kNY = kTY + 1;       // node tile
constexpr int kPlaneF = kNX * kNY * 3;            // floats of one node plane
constexpr int kRing = 4;                          // node planes held
constexpr int kTmemCols = 256;
constexpr int kTerms = 3;
constexpr int kComps = 2;                         // TF32 hi and lo parts
constexpr int kThreads = 256;                     // 4 consumer + 4 producer warps
constexpr uint32_t kWaitPolls = 1u << 20;
constexpr int kSmemBytes =
    (kComps * kBF + 2 * kComps * kTileF + kRing * kPlaneF + 2 * 6 * kM) * 4;
constexpr int kCorrRow = 243;   // 27 blocks of 3 x 3

// byte offset of (row, k) in a K-major, unswizzled operand (umma.cuh)
__host__ __device__ constexpr int op_off(int row, int k) {
  return (row >> 3) * kSBO + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ int ring_slot(int z) { return (z + kRing) % kRing; }

// the operand image of G = [G_0; ...; G_7] (192 x 24): row n = 24 i + 3 ln
// + r, column 3 lm + s holds G_i(3 ln + r, 3 lm + s) = GMi[i][ln][lm][3r+s];
// hi part first, then the TF32 remainder
__global__ void k_l1_bimg(const double *__restrict__ GMi, float *__restrict__ B) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < kBF; t += gridDim.x * blockDim.x) {
    const int n = t / kK, kk = t % kK;
    const int i = n / 24, ln = (n % 24) / 3, r = n % 3, lm = kk / 3, s = kk % 3;
    const double v = GMi[((i * 8 + ln) * 8 + lm) * 9 + 3 * r + s];
    const float hi = umma::to_tf32(static_cast<float>(v));
    const float lo = umma::to_tf32(static_cast<float>(v - static_cast<double>(hi)));
    B[op_off(n, kk) / 4] = hi;
    B[kBF + op_off(n, kk) / 4] = lo;
  }
}

// level-1 nodes next to a general-path coarse element get a correction row:
// row q holds node rows[q]; the CTAs (tile, z chunk) holding such nodes are
// flagged
__global__ void k_l1_flags(int cx, int cy, int cz, int tx_tiles, int ntiles, int zchunk,
                           int64_t cap_rows, const int *__restrict__ slot,
                           int *__restrict__ rows, uint8_t *__restrict__ cflag,
                           unsigned int *__restrict__ count, int *__restrict__ fault) {
  const int ex = cx - 1, ey = cy - 1, ez = cz - 1;
  const int64_t nn = (int64_t)cx * cy * cz;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn;
       n += (int64_t)gridDim.x * blockDim.x) {
    const int X = (int)(n % cx), Y = (int)((n / cx) % cy), Z = (int)(n / ((int64_t)cx * cy));
    bool any = false;
    for (int c = 0; c < 8; ++c) {
      const int EI = X - 1 + (c & 1), EJ = Y - 1 + ((c >> 1) & 1), EK = Z - 1 + (c >> 2);
      if (EI < 0 || EJ < 0 || EK < 0 || EI >= ex || EJ >= ey || EK >= ez) continue;
      any |= slot[((int64_t)EK * ey + EJ) * ex + EI] >= 0;
    }
    if (!any) continue;
    const unsigned int q = atomicAdd(count, 1u);
    if (q < cap_rows)
      rows[q] = (int)n;
    else
      atomicExch(fault, 1);
    cflag[(Z / zchunk) * ntiles + (Y / kOwnY) * tx_tiles + X / kOwnX] = 1;
  }
}

// correction rows: the full stencil row of the node minus
// sum over its elements of sum_i E_{E,i} G_i (both in FP64), one thread per
// (row, neighbour block)
__global__ void k_l1_corr(int cx, int cy, int cz, int64_t cap_rows, const double *__restrict__ E,
                          const double *__restrict__ GMi, const double *__restrict__ Sc,
                          const int *__restrict__ rows, const unsigned int *__restrict__ count,
                          float *__restrict__ C) {
  const int ex = cx - 1, ey = cy - 1, ez = cz - 1;
  const int nelx = 2 * ex, nely = 2 * ey;
  const int64_t nn = (int64_t)cx * cy * cz;
  const int64_t nrows = min((int64_t)*count, cap_rows);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 27 * nrows;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = t / 27;
    const int nb = (int)(t % 27);
    const int64_t n = rows[f];
    const int X = (int)(n % cx), Y = (int)((n / cx) % cy), Z = (int)(n / ((int64_t)cx * cy));
    const int MX = X + nb % 3 - 1, MY = Y + (nb / 3) % 3 - 1, MZ = Z + nb / 9 - 1;
    double acc[9];
    for (int q = 0; q < 9; ++q) acc[q] = Sc[(int64_t)(nb * 9 + q) * nn + n];
    if (MX >= 0 && MY >= 0 && MZ >= 0 && MX < cx && MY < cy && MZ < cz) {
      for (int EK = max(Z, MZ) - 1; EK <= min(Z, MZ); ++EK)
        for (int EJ = max(Y, MY) - 1; EJ <= min(Y, MY); ++EJ)
          for (int EI = max(X, MX) - 1; EI <= min(X, MX); ++EI) {
            if (EI < 0 || EJ < 0 || EK < 0 || EI >= ex || EJ >= ey || EK >= ez) continue;
            const int ln = (X - EI) + 2 * (Y - EJ) + 4 * (Z - EK);
            const int lm = (MX - EI) + 2 * (MY - EJ) + 4 * (MZ - EK);
            for (int i = 0; i < 8; ++i) {
              const int fx = 2 * EI + (i & 1), fy = 2 * EJ + ((i >> 1) & 1),
                        fz = 2 * EK + ((i >> 2) & 1);
              const double Ee = E[((int64_t)fz * nely + fy) * nelx + fx];
              const double *g = GMi + ((i * 8 + ln) * 8 + lm) * 9;
              for (int q = 0; q < 9; ++q) acc[q] -= Ee * g[q];
            }
          }
    }
    float *row = C + f * kCorrRow + nb * 9;
    for (int q = 0; q < 9; ++q) row[q] = static_cast<float>(acc[q]);
  }
}

// programmatic dependent launch: let the next kernel in the stream start,
// and wait for the grids this one depends on (no-ops without the launch
// attribute)
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// cval[3 n + r] = (C u)_r on the correction rows, one warp per row; u in the
// input form IN of the apply
template <int IN>
__global__ void k_l1_corr_apply(int cx, int cy, int cz, int64_t cap_rows,
                                const int *__restrict__ rows,
                                const unsigned int *__restrict__ count,
                                const float *__restrict__ C, const ApplyArgs<float> a,
                                float *__restrict__ cval) {
  pdl_launch_dependents();   // the apply may start; it waits where it reads cval
  const int lane = threadIdx.x & 31;
  const int64_t nrows = min((int64_t)*count, cap_rows);
  const int64_t wstride = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t f = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; f < nrows;
       f += wstride) {
    const int n = rows[f];
    const int X = n % cx, Y = (n / cx) % cy, Z = n / (cx * cy);
    const float *row = C + f * kCorrRow;
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int q = lane + 32 * j;
      if (q < kCorrRow) {
        const int nb = q / 9, rr = (q % 9) / 3, sd = q % 3;
        const int MX = X + nb % 3 - 1, MY = Y + (nb / 3) % 3 - 1, MZ = Z + nb / 9 - 1;
        float uu = 0.0f;
        if (MX >= 0 && MY >= 0 && MZ >= 0 && MX < cx && MY < cy && MZ < cz)
          uu = sym_in<float, IN>(a, 3 * ((MZ * cy + MY) * cx + MX) + sd);
        const float v = row[q] * uu;
        s0 += rr == 0 ? v : 0.0f;
        s1 += rr == 1 ? v : 0.0f;
        s2 += rr == 2 ? v : 0.0f;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      cval[3 * n] = s0;
      cval[3 * n + 1] = s1;
      cval[3 * n + 2] = s2;
    }
  }
}

struct L1Params {
  int cx, cy, cz;         // level-1 nodes
  int tx_tiles;           // tiles along x
  int zchunk;             // node planes per CTA
  const float *E;         // fine moduli (FP32), 2(cx-1) x 2(cy-1) x 2(cz-1)
  const float *B;         // operand image (k_l1_bimg)
  const float *cval;      // C u on the correction rows (dense, zero elsewhere)
  const uint8_t *cflag;   // CTAs holding correction rows
  double *fault;          // fault scalar: 2 when an MMA wait runs out
};

// named barriers (0 is __syncthreads): the consumer warps, the producer
// warps, and "operand b is in shared memory" (producers arrive, the MMA
// issuing warp waits)
constexpr int kBarCons = 1, kBarProd = 2, kBarFull0 = 3;

__device__ __forceinline__ void bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Warps 0-3 consume: they wait for the MMA of plane k, read their TMEM row
// (lane = element), weight it by the moduli and write the owned nodes; warp
// 0 issues the MMAs.  Warps 4-7 produce: node planes into the ring and the
// operand of plane k+1 into the other buffer while plane k is consumed.
// The MMAs reading operand buffer b commit to mbar[b].
template <int IN, int OUT>
__global__ void __launch_bounds__(kThreads, 2)
    k_apply_l1_tc(const L1Params p, const ApplyArgs<float> a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  float *Bs = reinterpret_cast<float *>(smem);
  float *As = Bs + kComps * kBF;             // [2 buffers][2 parts][kTileF]
  float *ring = As + 2 * kComps * kTileF;    // [kRing][kNY][kNX][3]
  float *ys = ring + kRing * kPlaneF;        // [2][6][kM]
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tbase_s;

  const int t = threadIdx.x, warp = t >> 5;
  const bool producer = t >= kM;
  const int e_ = producer ? t - kM : t;     // element row of this thread
  const int tx = blockIdx.x % p.tx_tiles, ty = blockIdx.x / p.tx_tiles;
  const int x0 = tx * kOwnX - 1, y0 = ty * kOwnY - 1;   // tile origin (elements and nodes)
  const int z0 = blockIdx.y * p.zchunk, z1 = min(p.cz, z0 + p.zchunk);
  const int xl = e_ % kTX, yl = e_ / kTX;
  const int ex = p.cx - 1, ey = p.cy - 1, ez = p.cz - 1;
  const int nelx = 2 * ex, nely = 2 * ey;
  const int kfirst = z0 - 1, klast = z1 - 1;   // element planes
  const int X = x0 + xl, Y = y0 + yl;        // element / node of this row

  for (int e = t; e < kComps * kBF / 4; e += kThreads)
    reinterpret_cast<int4 *>(Bs)[e] = __ldg(reinterpret_cast<const int4 *>(p.B) + e);
  if (warp == 0) {
    umma::tmem_alloc(&tbase_s, kTmemCols);
    umma::tmem_relinquish();
  }
  if (t == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
  }
  bool failed = false;
  const int pt = e_;
  // node plane z of the tile (input form IN), producers
  auto plane_load = [&](int z, float (&r)[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = pt + kM * j;
      r[j] = 0.0f;
      if (e < kPlaneF && z >= 0 && z < p.cz) {
        const int node = e / 3, d = e - 3 * node;
        const int NX = x0 + node % kNX, NY = y0 + node / kNX;
        if (NX >= 0 && NX < p.cx && NY >= 0 && NY < p.cy)
          r[j] = sym_in<float, IN>(a, 3 * ((z * p.cy + NY) * p.cx + NX) + d);
      }
    }
  };
  auto plane_store = [&](int z, const float (&r)[4]) {
    float *dst = ring + ring_slot(z) * kPlaneF;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = pt + kM * j;
      if (e < kPlaneF) dst[e] = r[j];
    }
  };
  // moduli of element plane k (zero outside the grid), consumers
  auto moduli = [&](int k, float (&Ev)[8]) {
    const bool in = X >= 0 && X < ex && Y >= 0 && Y < ey && k >= 0 && k < ez;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float2 v = make_float2(0.0f, 0.0f);
      if (in) {
        const int64_t idx =
            ((int64_t)(2 * k + (q >> 1)) * nely + 2 * Y + (q & 1)) * nelx + 2 * X;
        v = __ldg(reinterpret_cast<const float2 *>(p.E + idx));
      }
      Ev[2 * q] = v.x;   // fine element i = 2q: (0, q&1, q>>1)
      Ev[2 * q + 1] = v.y;
    }
  };
  float pf[4];
  float Ecur[8], Enext[8];
  if (producer) {
    float r0[4], r1[4];
    plane_load(kfirst, r0);
    plane_load(kfirst + 1, r1);
    plane_load(kfirst + 2, pf);
    plane_store(kfirst, r0);
    plane_store(kfirst + 1, r1);
  } else {
    moduli(kfirst, Ecur);
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();

  if (producer) {
    for (int j = kfirst; j <= klast; ++j) {
      const int jt = j - kfirst, b = jt & 1;
      // operand buffer b is free once the MMA of plane j-2 has completed
      if (jt >= 2 && !umma::mbar_wait(&mbar[b], (uint32_t)(((jt - 2) >> 1) & 1), kWaitPolls))
        failed = true;
      if (jt >= 1) {
        plane_store(j + 1, pf);
        plane_load(j + 2, pf);
      }
      bar_sync(kBarProd, kM);
      float *Ah = As + b * kComps * kTileF;
      float *Al = Ah + kTileF;
#pragma unroll
      for (int cc = 0; cc < kK / 4; ++cc) {
        float h[4], l[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const int kk = 4 * cc + w, lm = kk / 3, s = kk % 3;
          const int a_ = lm & 1, b_ = (lm >> 1) & 1, c_ = lm >> 2;
          const float v =
              ring[ring_slot(j + c_) * kPlaneF + ((yl + b_) * kNX + xl + a_) * 3 + s];
          h[w] = umma::to_tf32(v);
          l[w] = umma::to_tf32(v - h[w]);
        }
        const int off = op_off(pt, 4 * cc) / 4;
        *reinterpret_cast<float4 *>(Ah + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4 *>(Al + off) = make_float4(l[0], l[1], l[2], l[3]);
      }
      umma::fence_proxy_async();
      bar_arrive(kBarFull0 + b, kM + 32);
    }
  } else {
    const bool own_xy = xl >= 1 && yl >= 1 && X < p.cx && Y < p.cy;
    const bool corr = p.cflag[blockIdx.y * gridDim.x + blockIdx.x] != 0;
    const uint32_t idesc = umma::idesc_tf32(kM, kN);
    auto issue = [&](int buf, uint32_t tmem) {
      const uint32_t ab = umma::smem_u32(As + buf * kComps * kTileF);
      const uint32_t bb = umma::smem_u32(Bs);
#pragma unroll
      for (int q = 0; q < kTerms; ++q) {
        const uint32_t aq = ab + (q == 1 ? kTileF * 4 : 0);   // lo * hi
        const uint32_t bq = bb + (q == 2 ? kBF * 4 : 0);      // hi * lo
#pragma unroll
        for (int s = 0; s < kK / 8; ++s)
          umma::mma_tf32(tmem, umma::sdesc(aq + 256 * s, 128, kSBO),
                         umma::sdesc(bq + 256 * s, 128, kSBO), idesc, q > 0 || s > 0);
      }
      umma::commit(&mbar[buf]);
    };
    const uint32_t tmem = tbase_s;
    if (warp == 0) {
      bar_sync(kBarFull0, kM + 32);
      if (t == 0) {
        umma::fence_after_sync();
        issue(0, tmem);
      }
    }
    if (corr) pdl_wait();   // cval comes from the kernel launched just before
    float carry[3] = {0.0f, 0.0f, 0.0f};
    for (int k = kfirst; k <= klast; ++k) {
      const int it = k - kfirst, b = it & 1;
      const bool more = k + 1 <= klast;
      // epilogue inputs of the owned node on node plane k, and the next
      // plane's moduli, while the MMA runs
      const bool own = own_xy && k >= z0;
      const int gi = own ? 3 * ((k * p.cy + Y) * p.cx + X) : 0;
      float pb[3], pd[3], p2[3], pc[3], pu[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        pb[d] = ((OutNeeds<OUT>::b || IN == IN_CHEB) && own) ? a.b[gi + d] : 0.0f;
        pd[d] = ((OutNeeds<OUT>::dinv || IN == IN_CHEB) && own) ? a.dinv[gi + d] : 0.0f;
        p2[d] = (OutNeeds<OUT>::y2 && own) ? a.y2[gi + d] : 0.0f;
        pc[d] = (corr && own) ? p.cval[gi + d] : 0.0f;
        pu[d] = (IN == IN_U && OUT != OUT_Y && OUT != OUT_RESID && own) ? a.u[gi + d] : 0.0f;
      }
      if (more) moduli(k + 1, Enext);
      const bool ok = umma::mbar_wait(&mbar[b], (uint32_t)((it >> 1) & 1), kWaitPolls);
      if (!ok) failed = true;
      umma::fence_after_sync();
      // y_E = sum_i E_i D[:, 24 i + j]
      float y[24];
#pragma unroll
      for (int j = 0; j < 24; ++j) y[j] = 0.0f;
      if (ok) {
#pragma unroll
        for (int qc = 0; qc < kN / 32; ++qc) {
          float v[32];
          umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32 * qc, v);
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = 32 * qc + j;
            y[n % 24] = fmaf(Ecur[n / 24], v[j], y[n % 24]);
          }
        }
      }
      umma::fence_before_sync();
      // x: node xl takes this element's a = 0 corners and the left
      // neighbour's a = 1 corners; y: the row below's b = 1 corners
      float nx[2][2][3];
#pragma unroll
      for (int b_ = 0; b_ < 2; ++b_)
#pragma unroll
        for (int c_ = 0; c_ < 2; ++c_)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const float right = y[(1 + 2 * b_ + 4 * c_) * 3 + d];
            const float left = __shfl_up_sync(0xffffffffu, right, 1, 16);
            nx[b_][c_][d] = y[(2 * b_ + 4 * c_) * 3 + d] + (xl > 0 ? left : 0.0f);
          }
      float *yb = ys + b * 6 * kM;
#pragma unroll
      for (int c_ = 0; c_ < 2; ++c_)
#pragma unroll
        for (int d = 0; d < 3; ++d) yb[(c_ * 3 + d) * kM + t] = nx[1][c_][d];
      // every consumer has read its TMEM row: the next MMA may overwrite it
      bar_sync(kBarCons, kM);
      if (more && warp == 0) {
        bar_sync(kBarFull0 + (b ^ 1), kM + 32);
        if (t == 0) {
          umma::fence_after_sync();
          issue(b ^ 1, tmem);
        }
      }
      float tot[3], up[3];
#pragma unroll
      for (int c_ = 0; c_ < 2; ++c_)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float below = yl > 0 ? yb[(c_ * 3 + d) * kM + t - kTX] : 0.0f;
          const float v = nx[0][c_][d] + below;
          if (c_ == 0)
            tot[d] = carry[d] + v;
          else
            up[d] = v;
        }
      // node plane k is complete
      if (own && !failed) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float u_own = IN == IN_CHEB ? a.invtheta * (pd[d] * pb[d]) : pu[d];
          sym_out_v<float, OUT>(a, gi + d, tot[d] + pc[d], u_own, pb[d], pd[d], p2[d]);
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) carry[d] = up[d];
#pragma unroll
      for (int q = 0; q < 8; ++q) Ecur[q] = Enext[q];
    }
    // the last TMEM reads were fenced before the last consumer barrier
    if (warp == 0) {
      umma::fence_after_sync();
      umma::tmem_dealloc(tmem, kTmemCols);
    }
  }
  if (failed) *p.fault = 2.0;
  pdl_wait();   // this grid completes after the kernel it was launched behind
}

// pdl: launched behind k_l1_corr_apply as a programmatic dependent launch
template <int IN, int OUT>
void launch_mode(const L1Params &p, dim3 grid, const ApplyArgs<float> &a, bool pdl,
                 cudaStream_t s) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_apply_l1_tc<IN, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSmemBytes);
    // two CTAs per SM need the largest shared-memory carveout
    cudaFuncSetAttribute(k_apply_l1_tc<IN, OUT>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    attr_dev = dev;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemBytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_apply_l1_tc<IN, OUT>, p, a);
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

void l1tc_grid(const Level &v, int *tx, int *ty, int *zchunk, int *nz) {
  const int cx = v.dims[0], cy = v.dims[1], cz = v.dims[2];
  *tx = (cx + kOwnX - 1) / kOwnX;
  *ty = (cy + kOwnY - 1) / kOwnY;
  // about two CTAs per SM (their TMEM and shared memory allow two); the SM
  // count of the current device, read once per device
  static int sm_count[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  int &sms = sm_count[dev & 63];
  if (sms == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
      n = 148;
    sms = n;
  }
  const int tiles = *tx * *ty;
  int want = (2 * sms + tiles / 2) / tiles;
  want = std::max(1, std::min(want, cz));
  *zchunk = (cz + want - 1) / want;
  *nz = (cz + *zchunk - 1) / *zchunk;
}

int l1tc_prepare(Ctx &c, const double *Sc, int nslots, cudaStream_t s) {
  if (!c.l1tc_ok) return TPO_OK;
  const Level &v = c.lev[1];
  if (!c.l1_bimg_ready) {
    count_launch();
    k_l1_bimg<<<(kBF + 255) / 256, 256, 0, s>>>(c.GMi, c.l1_B);
    c.l1_bimg_ready = true;
  }
  // at most 8 nodes per general-path element carry a correction row
  const size_t rows = std::max<size_t>(8 * (size_t)nslots, 1);
  if (rows > c.l1_cap) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return TPO_E_CUDA;
    if (c.l1_C) cudaFree(c.l1_C);
    if (c.l1_rows) cudaFree(c.l1_rows);
    c.l1_C = nullptr;
    c.l1_rows = nullptr;
    c.l1_cap = 0;
    if (cudaMalloc(&c.l1_C, sizeof(float) * rows * kCorrRow) != cudaSuccess ||
        cudaMalloc(&c.l1_rows, sizeof(int) * rows) != cudaSuccess)
      return TPO_E_CUDA;
    c.l1_cap = rows;
  }
  int tx, ty, zc, nz;
  l1tc_grid(v, &tx, &ty, &zc, &nz);
  if (cudaMemsetAsync(c.l1_count, 0, sizeof(unsigned int), s) != cudaSuccess ||
      cudaMemsetAsync(c.l1_cflag, 0, (size_t)tx * ty * nz, s) != cudaSuccess ||
      cudaMemsetAsync(c.l1_cval, 0, sizeof(float) * 3 * v.nn, s) != cudaSuccess)
    return TPO_E_CUDA;
  count_launch(2);
  k_l1_flags<<<grid_for(v.nn, 256), 256, 0, s>>>(v.dims[0], v.dims[1], v.dims[2], tx, tx * ty,
                                                  zc, (int64_t)c.l1_cap, c.gk_slot, c.l1_rows,
                                                  c.l1_cflag, c.l1_count, c.l1_fault);
  k_l1_corr<<<grid_for(27 * (int64_t)c.l1_cap, 256), 256, 0, s>>>(
      v.dims[0], v.dims[1], v.dims[2], (int64_t)c.l1_cap, c.E64, c.GMi, Sc, c.l1_rows,
      c.l1_count, c.l1_C);
  return TPO_OK;
}

void launch_l1tc(const Ctx &c, int in, int out, const ApplyArgs<float> &a, cudaStream_t s) {
  const Level &v = c.lev[1];
  int tx, ty, zc, nz;
  l1tc_grid(v, &tx, &ty, &zc, &nz);
  // C u on the correction rows first (a warp per row; the row count is the
  // one the last set-up read back)
  const bool pdl = c.l1_nrows > 0;
  if (pdl) {
    const int blocks = (c.l1_nrows + 3) / 4;
    count_launch();
    if (in == IN_CHEB)
      k_l1_corr_apply<IN_CHEB><<<blocks, 128, 0, s>>>(v.dims[0], v.dims[1], v.dims[2],
                                                       (int64_t)c.l1_cap, c.l1_rows, c.l1_count,
                                                       c.l1_C, a, c.l1_cval);
    else
      k_l1_corr_apply<IN_U><<<blocks, 128, 0, s>>>(v.dims[0], v.dims[1], v.dims[2],
                                                    (int64_t)c.l1_cap, c.l1_rows, c.l1_count,
                                                    c.l1_C, a, c.l1_cval);
  }
  L1Params p;
  p.cx = v.dims[0];
  p.cy = v.dims[1];
  p.cz = v.dims[2];
  p.tx_tiles = tx;
  p.zchunk = zc;
  p.E = c.E32;
  p.B = c.l1_B;
  p.cval = c.l1_cval;
  p.cflag = c.l1_cflag;
  p.fault = c.scal + kSlotFault;
  const dim3 grid(tx * ty, nz);
  count_launch();
  if (in == IN_CHEB && out == OUT_CHEB2)
    launch_mode<IN_CHEB, OUT_CHEB2>(p, grid, a, pdl, s);
  else if (out == OUT_POST0)
    launch_mode<IN_U, OUT_POST0>(p, grid, a, pdl, s);
  else if (out == OUT_POST1)
    launch_mode<IN_U, OUT_POST1>(p, grid, a, pdl, s);
  else if (out == OUT_RESID)
    launch_mode<IN_U, OUT_RESID>(p, grid, a, pdl, s);
  else
    launch_mode<IN_U, OUT_Y>(p, grid, a, pdl, s);
}

}  // namespace tpo
