// Vector kernels of the Krylov solvers.  Every reduction accumulates in FP64
// and is deterministic: a fixed grid of kRedBlocks blocks writes one partial
// each in a fixed order, and the last block to finish (ticket counter) sums
// the partials in a fixed tree order and writes the result to a device
// scalar, so the CG recurrences never round-trip through the host.
#include <algorithm>
#include <cstdint>

#include "tpo_internal.h"

namespace tpo {

namespace {

constexpr int kRedThreads = 256;

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0;
  if (threadIdx.x < 32) {
    v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;   // valid in thread 0
}

// partial -> last block -> *out (previous *out moved to *shift_to if set).
// Column j of a block reduction owns blocks (*, j): part + j * gridDim.x
// and ticket + j.
__device__ __forceinline__ void finish_reduction(double v, double *part,
                                                 unsigned int *ticket,
                                                 double *out, double *shift_to) {
  __shared__ double sh[32];
  __shared__ bool last;
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v;
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s = 0;
  for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x)
    s += ((volatile double *)part)[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    if (shift_to) *shift_to = *out;
    *out = s;
    *ticket = 0u;
  }
}

// 16-byte vectors of the streamed kernels: 4 floats or 2 doubles
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using V = float4;
  static constexpr int W = 4;
  __device__ static float get(const V &v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
  }
  __device__ static void set(V &v, int k, float x) {
    if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
  }
};
template <>
struct Vec16<double> {
  using V = double2;
  static constexpr int W = 2;
  __device__ static double get(const V &v, int k) { return k == 0 ? v.x : v.y; }
  __device__ static void set(V &v, int k, double x) {
    if (k == 0) v.x = x; else v.y = x;
  }
};

__device__ __forceinline__ bool aligned16(const void *p) {
  return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// The streamed kernels walk a column in 16-byte vectors when its pointers
// allow (then the tail, fewer than one vector, element by element), else
// element by element; either way each thread's share and the order of its
// sums are fixed, so the reductions stay deterministic.

// a.b per column (blockIdx.y); a column whose skip flag is set (every block
// of it returns, so its ticket stays zero) keeps its out/shift_to slots
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
    k_dot(int64_t n, const T *__restrict__ a, const T *__restrict__ b,
          double *part, unsigned int *ticket, double *out, double *shift_to,
          const double *skip) {
  using VT = Vec16<T>;
  using V = typename VT::V;
  const int j = blockIdx.y;
  if (skip && skip[j * kColScal] != 0.0) return;
  a += j * n;
  b += j * n;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  double s = 0;
  int64_t tail = 0;
  if (aligned16(a) && aligned16(b)) {
    const int64_t nv = n / VT::W;
    const V *av = reinterpret_cast<const V *>(a);
    const V *bv = reinterpret_cast<const V *>(b);
    for (int64_t i = t0; i < nv; i += st) {
      const V x = av[i], y = bv[i];
#pragma unroll
      for (int k = 0; k < VT::W; ++k)
        s += static_cast<double>(VT::get(x, k)) * static_cast<double>(VT::get(y, k));
    }
    tail = nv * VT::W;
  }
  for (int64_t i = tail + t0; i < n; i += st)
    s += static_cast<double>(a[i]) * static_cast<double>(b[i]);
  finish_reduction(s, part + j * gridDim.x, ticket + j, out + j * kColScal,
                   shift_to ? shift_to + j * kColScal : nullptr);
}

// p = z (first) or p = z + (rho / rho_old) p, per column; a frozen column
// keeps its p
template <typename T>
__global__ void k_cg_p(int64_t n, const T *__restrict__ z, T *__restrict__ p,
                       const double *__restrict__ scal, bool first) {
  using VT = Vec16<T>;
  using V = typename VT::V;
  const int j = blockIdx.y;
  const double *sc = scal + j * kColScal;
  if (sc[6] != 0.0) return;
  z += j * n;
  p += j * n;
  const T beta = first ? T(0) : static_cast<T>(sc[0] / sc[1]);
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  int64_t tail = 0;
  if (aligned16(z) && aligned16(p)) {
    const int64_t nv = n / VT::W;
    const V *zv = reinterpret_cast<const V *>(z);
    V *pv = reinterpret_cast<V *>(p);
    for (int64_t i = t0; i < nv; i += st) {
      const V zz = zv[i];
      V pp = first ? zz : pv[i];
      if (!first) {
#pragma unroll
        for (int k = 0; k < VT::W; ++k) VT::set(pp, k, VT::get(zz, k) + beta * VT::get(pp, k));
      }
      pv[i] = pp;
    }
    tail = nv * VT::W;
  }
  for (int64_t i = tail + t0; i < n; i += st) p[i] = first ? z[i] : z[i] + beta * p[i];
}

// x += alpha p ; r -= alpha q ; rr = r.r   with alpha = rho / (p.q), per
// column; a frozen column only recomputes rr
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
    k_cg_update(int64_t n, T *__restrict__ x, T *__restrict__ r,
                const T *__restrict__ p, const T *__restrict__ q,
                const double *__restrict__ scal, double *part,
                unsigned int *ticket, double *rr) {
  using VT = Vec16<T>;
  using V = typename VT::V;
  const int j = blockIdx.y;
  const double *sc = scal + j * kColScal;
  const bool frozen = sc[6] != 0.0;
  const T alpha = frozen ? T(0) : static_cast<T>(sc[0] / sc[2]);
  x += j * n;
  r += j * n;
  p += j * n;
  q += j * n;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  double s = 0;
  int64_t tail = 0;
  if (aligned16(x) && aligned16(r) && aligned16(p) && aligned16(q)) {
    const int64_t nv = n / VT::W;
    V *xv = reinterpret_cast<V *>(x);
    V *rv = reinterpret_cast<V *>(r);
    const V *pv = reinterpret_cast<const V *>(p);
    const V *qv = reinterpret_cast<const V *>(q);
    for (int64_t i = t0; i < nv; i += st) {
      V rr_ = rv[i];
      if (!frozen) {
        V xx = xv[i];
        const V pp = pv[i], qq = qv[i];
#pragma unroll
        for (int k = 0; k < VT::W; ++k) {
          VT::set(xx, k, VT::get(xx, k) + alpha * VT::get(pp, k));
          VT::set(rr_, k, VT::get(rr_, k) - alpha * VT::get(qq, k));
        }
        xv[i] = xx;
        rv[i] = rr_;
      }
#pragma unroll
      for (int k = 0; k < VT::W; ++k)
        s += static_cast<double>(VT::get(rr_, k)) * static_cast<double>(VT::get(rr_, k));
    }
    tail = nv * VT::W;
  }
  for (int64_t i = tail + t0; i < n; i += st) {
    T ri = r[i];
    if (!frozen) {
      x[i] += alpha * p[i];
      ri -= alpha * q[i];
      r[i] = ri;
    }
    s += static_cast<double>(ri) * static_cast<double>(ri);
  }
  finish_reduction(s, part + j * gridDim.x, ticket + j, rr + j * kColScal,
                   nullptr);
}

__device__ __forceinline__ double start_value(uint64_t i) {
  // splitmix64 of the dof index mapped to [-1, 1)
  uint64_t z = i + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

template <typename T>
__global__ void k_power_start(int64_t n, T *a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = static_cast<T>(start_value((uint64_t)i));
}

// w *= dinv and ||w||^2, accumulated in FP64 for either storage type
template <typename T>
__global__ void __launch_bounds__(kRedThreads)
    k_scale_diag_dot(int64_t n, T *__restrict__ w, const T *__restrict__ dinv,
                     double *part, unsigned int *ticket, double *out,
                     double *shift_to) {
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T wi = w[i] * dinv[i];
    w[i] = wi;
    s += static_cast<double>(wi) * static_cast<double>(wi);
  }
  finish_reduction(s, part, ticket, out, shift_to);
}

// b = float(a / sqrt(*nrm2)) per column (a zero column stays zero)
__global__ void k_to_f32_scaled(int64_t n, const double *a, const double *nrm2,
                                float *b) {
  const int j = blockIdx.y;
  const double nr = nrm2[j * kColScal];
  const double s = nr > 0.0 ? 1.0 / sqrt(nr) : 0.0;
  a += j * n;
  b += j * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = static_cast<float>(a[i] * s);
}

// U += sqrt(*nrm2) * double(d) per column
__global__ void k_axpy_f32(int64_t n, double *U, const float *d,
                           const double *nrm2) {
  const int j = blockIdx.y;
  const double s = sqrt(nrm2[j * kColScal]);
  U += j * n;
  d += j * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    U[i] += s * static_cast<double>(d[i]);
}

__global__ void k_d2f(int64_t n, const double *a, float *b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = static_cast<float>(a[i]);
}

__global__ void k_f2d(int64_t n, const float *a, double *b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = static_cast<double>(a[i]);
}

__global__ void k_fill(int64_t n, double *a, double v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

}  // namespace

// elementwise grid over nb columns: about the single-column grid in total
static dim3 col_grid(int64_t n, int nb) {
  int g = grid_for(n, 256);
  if (nb > 1) g = std::max(148, g / nb);
  return dim3(g, nb);
}

template <typename T>
void launch_dot(const Ctx &c, int64_t n, const T *a, const T *b, double *out,
                double *shift_to, cudaStream_t s, int nb, double *part,
                unsigned int *ticket) {
  count_launch();
  k_dot<T><<<dim3(red_grid(nb), nb), kRedThreads, 0, s>>>(
      n, a, b, part ? part : c.part, ticket ? ticket : c.ticket, out, shift_to,
      nullptr);
}

template <typename T>
void launch_rho_dot(const Ctx &c, int64_t n, const T *r, const T *z, cudaStream_t s,
                    int nb) {
  count_launch();
  k_dot<T><<<dim3(red_grid(nb), nb), kRedThreads, 0, s>>>(
      n, r, z, c.part, c.ticket, c.scal + 0, c.scal + 1, c.scal + 6);
}
template void launch_rho_dot<double>(const Ctx &, int64_t, const double *,
                                     const double *, cudaStream_t, int);
template void launch_rho_dot<float>(const Ctx &, int64_t, const float *,
                                    const float *, cudaStream_t, int);
template void launch_dot<double>(const Ctx &, int64_t, const double *,
                                 const double *, double *, double *,
                                 cudaStream_t, int, double *, unsigned int *);
template void launch_dot<float>(const Ctx &, int64_t, const float *,
                                const float *, double *, double *,
                                cudaStream_t, int, double *, unsigned int *);

template <typename T>
void launch_cg_p(int64_t n, const T *z, T *p, const double *scal, bool first,
                 cudaStream_t s, int nb) {
  count_launch();
  k_cg_p<T><<<col_grid(n, nb), 256, 0, s>>>(n, z, p, scal, first);
}
template void launch_cg_p<double>(int64_t, const double *, double *,
                                  const double *, bool, cudaStream_t, int);
template void launch_cg_p<float>(int64_t, const float *, float *,
                                 const double *, bool, cudaStream_t, int);

template <typename T>
void launch_cg_update(const Ctx &c, int64_t n, T *x, T *r, const T *p,
                      const T *q, const double *scal, double *rr,
                      cudaStream_t s, int nb) {
  count_launch();
  k_cg_update<T><<<dim3(red_grid(nb), nb), kRedThreads, 0, s>>>(
      n, x, r, p, q, scal, c.part, c.ticket, rr);
}
template void launch_cg_update<double>(const Ctx &, int64_t, double *,
                                       double *, const double *,
                                       const double *, const double *,
                                       double *, cudaStream_t, int);
template void launch_cg_update<float>(const Ctx &, int64_t, float *, float *,
                                      const float *, const float *,
                                      const double *, double *, cudaStream_t,
                                      int);

template <typename T>
void launch_power_start(int64_t n, T *a, cudaStream_t s) {
  count_launch();
  k_power_start<T><<<grid_for(n, 256), 256, 0, s>>>(n, a);
}
template void launch_power_start<double>(int64_t, double *, cudaStream_t);
template void launch_power_start<float>(int64_t, float *, cudaStream_t);

template <typename T>
void launch_scale_diag_dot(const Ctx &c, int64_t n, T *w, const T *dinv, double *out,
                           double *shift_to, cudaStream_t s, double *part,
                           unsigned int *ticket) {
  count_launch();
  k_scale_diag_dot<T><<<red_grid(1), kRedThreads, 0, s>>>(
      n, w, dinv, part ? part : c.part, ticket ? ticket : c.ticket, out, shift_to);
}
template void launch_scale_diag_dot<double>(const Ctx &, int64_t, double *, const double *,
                                            double *, double *, cudaStream_t, double *,
                                            unsigned int *);
template void launch_scale_diag_dot<float>(const Ctx &, int64_t, float *, const float *,
                                           double *, double *, cudaStream_t, double *,
                                           unsigned int *);

void launch_to_f32_scaled(int64_t n, const double *a, const double *scal,
                          float *b, cudaStream_t s, int nb) {
  count_launch();
  k_to_f32_scaled<<<col_grid(n, nb), 256, 0, s>>>(n, a, scal, b);
}

void launch_axpy_f32(int64_t n, double *U, const float *d, const double *scal,
                     cudaStream_t s, int nb) {
  count_launch();
  k_axpy_f32<<<col_grid(n, nb), 256, 0, s>>>(n, U, d, scal);
}

void launch_d2f(int64_t n, const double *a, float *b, cudaStream_t s) {
  count_launch();
  k_d2f<<<grid_for(n, 256), 256, 0, s>>>(n, a, b);
}

void launch_f2d(int64_t n, const float *a, double *b, cudaStream_t s) {
  count_launch();
  k_f2d<<<grid_for(n, 256), 256, 0, s>>>(n, a, b);
}

void launch_fill(int64_t n, double *a, double v, cudaStream_t s) {
  count_launch();
  k_fill<<<grid_for(n, 256), 256, 0, s>>>(n, a, v);
}

}  // namespace tpo
