// tpo_sensitivity_noalloc: the filtered compliance sensitivity for callers
// that cannot allocate device memory.
//
// Some hosts run this library where cudaMalloc is not available to them: a
// plugin inside a framework that owns every device allocation through its
// own pool, code that runs while a CUDA graph is being captured, or a process
// that budgets device memory up front and forbids allocations afterwards.
// They hold only the buffers they were handed.  This entry point needs no
// context (tpo_create allocates) and no allocation at all: the per-element
// intermediate lives in the fixed array below, which every GPU that loads
// the library holds (8 MiB) until the process exits.
//
// dC/dx = P^T g,  g_e = -dEdz_e * u_e^T K0 u_e   (Compliance.cpp:37-51)
//
// with P the row-normalised radius-rmin cone filter (Filter.cpp:21-150).  The
// array holds g; the transpose recomputes each row sum from the filter
// template, so nothing else is stored.
//
// The array is shared by every call in the process: two calls whose kernels
// overlap on one GPU (different streams or host threads without ordering)
// race on it.  Each call overwrites every entry it reads, so nothing has to
// start at zero.
#include <mutex>

#include "modal.cuh"

namespace tpo {

namespace {

constexpr int kNaMaxTaps = 128;

__device__ __align__(256) double g_noalloc_scratch[TPO_NOALLOC_MAX_ELEMS];

struct NaTaps {
  int n;
  int8_t off[kNaMaxTaps][3];
  double w[kNaMaxTaps];
};

__device__ __forceinline__ double na_rowsum_inv(const NaTaps &T, int i, int j,
                                                int k, int nx, int ny, int nz) {
  double s = 0;
  for (int t = 0; t < T.n; ++t) {
    const int a = i + T.off[t][0], b = j + T.off[t][1], c = k + T.off[t][2];
    if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
    s += T.w[t];
  }
  return 1.0 / s;
}

// g_e = -dEdz_e * u_e^T K0 u_e into the scratch array
__global__ void k_na_energy(int nelx, int nely, int nelz,
                            const double *__restrict__ U,
                            const double *__restrict__ dEdz, double *g,
                            const Kh<double> kh) {
  const int Nx = nelx + 1, Ny = nely + 1;
  const int64_t ne = (int64_t)nelx * nely * nelz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nelx, j = (e / nelx) % nely, k = e / ((int64_t)nelx * nely);
    double v[8][3];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      const int64_t n = ((int64_t)(k + (l >> 2)) * Ny + (j + ((l >> 1) & 1))) * Nx +
                        (i + (l & 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) v[l][c] = U[3 * n + c];
    }
    g[e] = -dEdz[e] * element_energy(v, kh);
  }
}

// out_j = sum over rows i (increasing) of (W_ij / rowsum_i) g_i
__global__ void k_na_adjoint(int nx, int ny, int nz, const NaTaps T,
                             const double *__restrict__ g,
                             double *__restrict__ out) {
  const int64_t ne = (int64_t)nx * ny * nz;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
    double s = 0;
    for (int t = T.n - 1; t >= 0; --t) {
      const int a = i - T.off[t][0], b = j - T.off[t][1], c = k - T.off[t][2];
      if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
      const double fi = na_rowsum_inv(T, a, b, c, nx, ny, nz);
      s += (T.w[t] * fi) * g[((int64_t)c * ny + b) * nx + a];
    }
    out[e] = s;
  }
}

std::mutex g_na_mutex;
double *g_na_ptr[64] = {nullptr};   // device address of the array, per device
int g_na_sms[64] = {0};             // multiprocessor count, per device

// a caller buffer must be device (or managed) memory of the current GPU;
// a host pointer would reach the kernels as an illegal address
bool na_device_buffer(const void *p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

void na_message(char *msg, int32_t len, const char *text) {
  if (!msg || len <= 0) return;
  int32_t k = 0;
  for (; k + 1 < len && text[k]; ++k) msg[k] = text[k];
  msg[k] = '\0';
}

}  // namespace

}  // namespace tpo

extern "C" int tpo_sensitivity_noalloc(const int32_t nel[3], const double dx[3],
                                       double E0, double nu, double rmin,
                                       const double *U, const double *dEdz,
                                       double *dCdx, void *stream, char *msg,
                                       int32_t msg_len) {
  using namespace tpo;
  na_message(msg, msg_len, "");
  if (!nel || !dx) {
    na_message(msg, msg_len, "null mesh description");
    return TPO_E_ARG;
  }
  for (int d = 0; d < 3; ++d)
    if (nel[d] < 1 || !(dx[d] > 0)) {
      na_message(msg, msg_len, "invalid mesh size");
      return TPO_E_ARG;
    }
  const int64_t ne = (int64_t)nel[0] * nel[1] * nel[2];
  if (ne > (int64_t)TPO_NOALLOC_MAX_ELEMS) {
    na_message(msg, msg_len,
               "mesh has more elements than TPO_NOALLOC_MAX_ELEMS (1048576): "
               "use tpo_compliance on a context instead");
    return TPO_E_ARG;
  }
  if (!U || !dEdz || !dCdx || !(E0 > 0) || !(nu > -1.0 && nu < 0.5) || !(rmin > 0)) {
    na_message(msg, msg_len, "null buffer or invalid material/filter parameter");
    return TPO_E_ARG;
  }
  // element and filter constants on the host (no device memory involved)
  static thread_local Ctx host;   // only the host-side constant fields are used
  host.prm.dx[0] = dx[0];
  host.prm.dx[1] = dx[1];
  host.prm.dx[2] = dx[2];
  host.prm.E0 = E0;
  host.prm.nu = nu;
  if (build_element_constants(host) != TPO_OK) {
    na_message(msg, msg_len, "element stiffness does not decouple in the modal basis");
    return TPO_E_UNSUPPORTED;
  }
  const int nel3[3] = {nel[0], nel[1], nel[2]};
  if (!build_filter_taps(nel3, dx, rmin, host.taps) || host.taps.n > kNaMaxTaps) {
    na_message(msg, msg_len, "filter radius invalid or too large for this entry point (> 128 taps)");
    return TPO_E_UNSUPPORTED;
  }
  NaTaps taps{};
  taps.n = host.taps.n;
  for (int t = 0; t < taps.n; ++t) {
    for (int d = 0; d < 3; ++d) taps.off[t][d] = host.taps.off[t][d];
    taps.w[t] = host.taps.w[t];
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    na_message(msg, msg_len, "no CUDA device");
    return TPO_E_CUDA;
  }
  if (!na_device_buffer(U, dev) || !na_device_buffer(dEdz, dev) ||
      !na_device_buffer(dCdx, dev)) {
    na_message(msg, msg_len, "U, dEdz and dCdx must be device memory of the current GPU");
    return TPO_E_ARG;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    na_message(msg, msg_len, "invalid stream");
    return TPO_E_ARG;
  }
  // the array's device address, looked up with the device current (the
  // host-side symbol is not a device address): at the first call on each
  // device, and again on every call made outside a stream capture, so that
  // a context re-created after cudaDeviceReset gets its own address
  double *scratch = nullptr;
  int sms = 0;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev] || cap == cudaStreamCaptureStatusNone) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        na_message(msg, msg_len, cudaGetErrorString(e));
        return TPO_E_CUDA;
      }
      g_na_ptr[dev] = static_cast<double *>(p);
      if (cudaDeviceGetAttribute(&g_na_sms[dev], cudaDevAttrMultiProcessorCount, dev) !=
          cudaSuccess) {
        cudaGetLastError();
        g_na_sms[dev] = 1;
      }
    }
    scratch = g_na_ptr[dev];
    sms = g_na_sms[dev] > 0 ? g_na_sms[dev] : 1;
  }
  int64_t blocks = (ne + 127) / 128;
  if (blocks > (int64_t)sms * 32) blocks = (int64_t)sms * 32;
  k_na_energy<<<(int)blocks, 128, 0, s>>>(nel[0], nel[1], nel[2], U, dEdz,
                                          scratch, host.kh64);
  k_na_adjoint<<<(int)blocks, 128, 0, s>>>(nel[0], nel[1], nel[2], taps,
                                           scratch, dCdx);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    na_message(msg, msg_len, cudaGetErrorString(e));
    return TPO_E_CUDA;
  }
  count_launch(2);
  return TPO_OK;
}
