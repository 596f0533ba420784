// The C ABI (include/topopt_b200.h): context life cycle, boundary
// conditions, the TopOpt call surface and data movement between caller
// buffers and the context's HBM-resident state.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <string>

#include "coarse.h"
#include "grid_barrier.cuh"
#include "io.h"
#include "solver.h"

using tpo::Ctx;

struct tpo_ctx {
  Ctx c;
};

namespace tpo {
std::atomic<long long> g_launches{0};
}

namespace {

#define CK(call)                                                       \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      c.err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return TPO_E_CUDA;                                               \
    }                                                                  \
  } while (0)

#define REQUIRE(cond, msg)   \
  do {                       \
    if (!(cond)) {           \
      c.err = (msg);         \
      return TPO_E_ARG;      \
    }                        \
  } while (0)

template <typename T>
int dalloc(Ctx &c, T **p, size_t n) {
  if (*p) return TPO_OK;
  CK(cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(n, 1)));
  CK(cudaMemsetAsync(*p, 0, sizeof(T) * std::max<size_t>(n, 1), c.stream));
  return TPO_OK;
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// message of the last failed context-free call (file I/O, tpo_load_mesh),
// per thread; tpo_last_error(NULL) returns it
thread_local std::string g_io_err;

int io_fail(const std::string &msg, int rc = TPO_E_ARG) {
  g_io_err = msg;
  return rc;
}

std::string folder_prefix(const char *folder) {
  std::string d = folder;
  if (!d.empty() && d.back() != '/') d += '/';
  return d;
}

// Eigen 3.3 LinSpaced (floating point) as used for the node coordinates
// (RecMesh.cpp:582-597)
double linspaced(double lo, double hi, int64_t n, int64_t i) {
  if (n == 1) return hi;
  const double step = (hi - lo) / static_cast<double>(n - 1);
  if (std::fabs(hi) < std::fabs(lo))
    return (i == 0) ? lo : hi - static_cast<double>(n - 1 - i) * step;
  return (i == n - 1) ? hi : lo + static_cast<double>(i) * step;
}

int begin(tpo_ctx *ctx) {
  if (!ctx) return TPO_E_ARG;
  cudaError_t e = cudaSetDevice(ctx->c.device);
  if (e != cudaSuccess) {
    ctx->c.err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    return TPO_E_CUDA;
  }
  ctx->c.err.clear();
  return TPO_OK;
}

int finish(Ctx &c, int rc) {
  if (rc < 0) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    c.err = std::string("kernel launch: ") + cudaGetErrorString(e);
    return TPO_E_CUDA;
  }
  return rc;
}

// device view of a caller buffer: device pointers pass through, host
// buffers are staged into `buf`
int stage_in(Ctx &c, const double *p, size_t n, int mem, double *buf,
             const double **out) {
  if (mem == TPO_MEM_DEVICE) {
    *out = p;
    return TPO_OK;
  }
  CK(cudaMemcpyAsync(buf, p, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
  *out = buf;
  return TPO_OK;
}

int copy_out(Ctx &c, double *dst, const double *src, size_t n, int mem) {
  if (!dst) return TPO_OK;
  if (dst == src) return TPO_OK;
  CK(cudaMemcpyAsync(dst, src, sizeof(double) * n,
                     mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                           : cudaMemcpyDeviceToHost,
                     c.stream));
  if (mem != TPO_MEM_DEVICE) CK(cudaStreamSynchronize(c.stream));
  return TPO_OK;
}

// the identity-row mask follows E and the fixed mask
void refresh_idm(Ctx &c) {
  if (c.have_material) tpo::launch_identity_mask(c, c.stream);
}

// a caller buffer flagged TPO_MEM_DEVICE must be device (or managed)
// memory of the context's GPU: a host pointer handed to a kernel would be
// an illegal-address fault, so it is refused before anything is issued
int check_device_ptr(Ctx &c, const void *p) {
  if (!p) return TPO_OK;
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();   // clear the sticky-free error of the query
    c.err = std::string("TPO_MEM_DEVICE buffer is not device memory (") +
            cudaGetErrorString(e) + ")";
    return TPO_E_ARG;
  }
  if (a.type == cudaMemoryTypeManaged) return TPO_OK;
  if (a.type != cudaMemoryTypeDevice) {
    c.err = "TPO_MEM_DEVICE buffer is host memory";
    return TPO_E_ARG;
  }
  if (a.device != c.device) {
    c.err = "TPO_MEM_DEVICE buffer lives on another GPU than the context";
    return TPO_E_ARG;
  }
  return TPO_OK;
}

// `mem` is one of the two flags, and with TPO_MEM_DEVICE every buffer the
// call reads or writes in `mem` is device memory of the context's GPU
int check_mem(Ctx &c, int mem, std::initializer_list<const void *> bufs = {}) {
  REQUIRE(mem == TPO_MEM_HOST || mem == TPO_MEM_DEVICE, "mem must be TPO_MEM_HOST or TPO_MEM_DEVICE");
  if (mem == TPO_MEM_DEVICE)
    for (const void *p : bufs)
      if (int rc = check_device_ptr(c, p)) return rc;
  return TPO_OK;
}

// per-level V-cycle vectors and the fine-level Krylov vectors: nb_cap
// columns each
int alloc_columns(Ctx &c) {
  const size_t n0 = 3 * c.nn, cap = c.nb_cap;
  int rc = 0;
#define A(p, n) \
  if ((rc = dalloc(c, &(p), (n))) != TPO_OK) return rc
  for (int l = 0; l < c.L; ++l) {
    tpo::Level &v = c.lev[l];
    const size_t n = 3 * v.nn * cap;
    A(v.r64, n); A(v.d64, n); A(v.a64, n);
    A(v.r32, n); A(v.d32, n); A(v.a32, n);
    if (l > 0) {
      A(v.b64, n); A(v.x64, n); A(v.b32, n); A(v.x32, n);
      A(v.e64, n); A(v.w64, n); A(v.e32, n); A(v.w32, n);
    }
  }
  A(c.r64, n0 * cap); A(c.z64, n0 * cap); A(c.p64, n0 * cap); A(c.q64, n0 * cap);
  A(c.r32, n0 * cap); A(c.z32, n0 * cap); A(c.p32, n0 * cap); A(c.q32, n0 * cap);
  A(c.x32, n0 * cap);
  if (cap > 1) {
    A(c.io_ba, n0 * cap);
    A(c.io_bb, n0 * cap);
  }
#undef A
  return TPO_OK;
}

void free_columns(Ctx &c) {
  for (tpo::Level &v : c.lev) {
    dfree(v.b64); dfree(v.x64); dfree(v.r64); dfree(v.d64); dfree(v.a64);
    dfree(v.b32); dfree(v.x32); dfree(v.r32); dfree(v.d32); dfree(v.a32);
    dfree(v.e64); dfree(v.w64); dfree(v.e32); dfree(v.w32);
  }
  dfree(c.r64); dfree(c.z64); dfree(c.p64); dfree(c.q64);
  dfree(c.r32); dfree(c.z32); dfree(c.p32); dfree(c.q32); dfree(c.x32);
  dfree(c.io_ba); dfree(c.io_bb);
}


int alloc_solver(Ctx &c) {
  int rc = 0;
#define A(p, n) \
  if ((rc = dalloc(c, &(p), (n))) != TPO_OK) return rc
  // the assembled fine stencil is only the coarsest operator of a
  // one-level hierarchy; level 1 is formed from the element moduli
  if (c.L == 1) A(c.S0, 243 * c.nn);
  for (int l = 0; l < c.L; ++l) {
    tpo::Level &v = c.lev[l];
    const size_t n = 3 * v.nn;
    A(v.dinv64, n);
    A(v.dinv32, n);
    if (l > 0) {
      A(v.S64, 243 * v.nn);
      if (l < c.ps) {
        A(v.H64, 126 * v.nn);
        A(v.H32, 126 * ((v.nn + 31) / 32) * 32);   // tiles of 32 nodes (kernels_mg.cu)
      }
      if (l >= c.ps && l + 1 < c.L) {
        A(v.A64, 243 * v.nn);
        A(v.A32, 243 * v.nn);
      }
    }
  }
  if (c.L > 2) A(c.gd_tmp, tpo::galerkin_dims_scratch(c.lev[1]));
  const int64_t nc = 3 * c.lev[c.L - 1].nn;
  A(c.Adense, tpo::coarse_inverse_work(nc));   // inversion workspace
  A(c.Ainv, (size_t)(nc * nc));
  A(c.w64, 3 * c.nn);
#undef A
  return alloc_columns(c);
}

void free_all(Ctx &c) {
  tpo::invalidate_graphs(c);
  free_columns(c);
  for (tpo::Level &v : c.lev) {
    dfree(v.S64); dfree(v.S32); dfree(v.dinv64); dfree(v.dinv32);
    dfree(v.A64); dfree(v.A32); dfree(v.H64); dfree(v.H32);
  }
  dfree(c.fix); dfree(c.idm); dfree(c.F); dfree(c.U); dfree(c.x); dfree(c.rho);
  dfree(c.E64); dfree(c.dEdz); dfree(c.E32); dfree(c.S0); dfree(c.K0lex);
  dfree(c.GMi); dfree(c.gk_slot); dfree(c.gk_elem); dfree(c.gk_count);
  dfree(c.gk_G); c.gk_cap = 0; dfree(c.gd_tmp);
  dfree(c.l1_B); dfree(c.l1_rows); dfree(c.l1_C); c.l1_cap = 0; dfree(c.l1_cval);
  dfree(c.l1_cflag); dfree(c.l1_count); dfree(c.l1_fault); c.l1_bimg_ready = false;
  dfree(c.Ainv); dfree(c.Adense); dfree(c.dev_info);
  dfree(c.finv); dfree(c.taps_d);
  dfree(c.w64);
  dfree(c.Es64); dfree(c.dEsdz64); dfree(c.bk_buf); c.bk_n = 0; dfree(c.fq_buf); c.fq_n = 0; dfree(c.mma_buf); c.mma_n = 0;
  if (c.mma_h) cudaFreeHost(c.mma_h);
  c.mma_h = nullptr; dfree(c.ks_S); dfree(c.ks_H); dfree(c.eig_buf);
  c.eig_n = 0;
  dfree(c.scal); dfree(c.part); dfree(c.ticket); dfree(c.gbar); dfree(c.tmpe); dfree(c.tmpe2);
  dfree(c.io_a); dfree(c.io_b);
  dfree(c.oc_ws);
  if (c.scal_h) cudaFreeHost(c.scal_h);
  c.scal_h = nullptr;
  for (cudaStream_t &q : c.aux_stream)
    if (q) cudaStreamSynchronize(q);
  for (cudaEvent_t &e : c.lev_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  for (cudaEvent_t &e : c.aux_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  for (cudaStream_t &q : c.aux_stream) {
    if (q) cudaStreamDestroy(q);
    q = nullptr;
  }
  if (c.setup_stream) {
    cudaStreamSynchronize(c.setup_stream);
    cudaStreamDestroy(c.setup_stream);
  }
  c.setup_stream = nullptr;
  for (cudaEvent_t &e : c.setup_ev) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (c.own_stream) cudaStreamDestroy(c.own_stream);
  c.own_stream = c.stream = nullptr;
}

double *vec_ptr(Ctx &c, const char *which, size_t *n) {
  if (!which) return nullptr;
  if (!std::strcmp(which, "U")) { *n = 3 * c.nn; return c.U; }
  if (!std::strcmp(which, "F")) { *n = 3 * c.nn; return c.F; }
  if (!std::strcmp(which, "x")) { *n = c.ne; return c.x; }
  if (!std::strcmp(which, "rho")) { *n = c.ne; return c.rho; }
  if (!std::strcmp(which, "E")) { *n = c.ne; return c.E64; }
  if (!std::strcmp(which, "dEdz")) { *n = c.ne; return c.dEdz; }
  if (!std::strcmp(which, "Es")) { *n = c.ne; return c.Es64; }
  return nullptr;
}

}  // namespace

namespace tpo {
// room for nb columns: the column vectors are re-allocated for kMaxBatch
// columns the first time a block of more than one is asked for
int ensure_columns(Ctx &c, int nb) {
  if (nb <= c.nb_cap) return TPO_OK;
  CK(cudaStreamSynchronize(c.stream));
  tpo::invalidate_graphs(c);
  free_columns(c);
  c.nb_cap = tpo::kMaxBatch;
  return alloc_columns(c);
}
}  // namespace tpo

using tpo::ensure_columns;

extern "C" {

void tpo_default_solve_opts(tpo_solve_opts *o) {
  if (!o) return;
  o->rtol = 1e-8;
  o->maxit = 500;
  o->precision = TPO_PREC_FP64;
  o->cheb_degree = 2;
  o->cheb_lo = 0.1;
  o->cheb_hi = 1.1;
  o->power_its = 15;
  o->inner_rtol = 1e-2;
  o->max_outer = 10;
  o->use_graph = 1;
  o->rhs_block = 0;
}

const char *tpo_last_error(const tpo_ctx *ctx) {
  if (ctx) return ctx->c.err.c_str();
  return g_io_err.empty() ? "null context" : g_io_err.c_str();
}

int tpo_create(const tpo_mesh_params *p, tpo_ctx **out) {
  if (!p || !out) return TPO_E_ARG;
  *out = nullptr;
  for (int d = 0; d < 3; ++d)
    if (p->nel[d] < 1 || !(p->dx[d] > 0)) return TPO_E_ARG;
  if (!(p->E0 > 0) || !(p->nu > -1.0 && p->nu < 0.5) || !(p->rmin > 0))
    return TPO_E_ARG;
  tpo_ctx *ctx = new tpo_ctx();
  Ctx &c = ctx->c;
  c.prm = *p;
  for (int d = 0; d < 3; ++d) c.nel[d] = p->nel[d];
  c.ne = (int64_t)c.nel[0] * c.nel[1] * c.nel[2];
  c.nn = (int64_t)(c.nel[0] + 1) * (c.nel[1] + 1) * (c.nel[2] + 1);
  if (3 * c.nn >= (int64_t)1 << 31) {
    delete ctx;
    return TPO_E_UNSUPPORTED;
  }
  // levels: floor(log2(min nel)) unless given (RecMesh.cpp:552-557), cut
  // when a level has <= 10 dofs (Interpolation.cpp:61-69)
  int L = p->mg_levels;
  if (L <= 0) {
    const int mn = std::min(c.nel[0], std::min(c.nel[1], c.nel[2]));
    L = (int)std::log2((double)mn);
  }
  if (L < 1) L = 1;
  int dims[3] = {c.nel[0] + 1, c.nel[1] + 1, c.nel[2] + 1};
  c.lev.clear();
  for (int l = 0; l < L; ++l) {
    tpo::Level v;
    std::memcpy(v.dims, dims, sizeof(dims));
    v.nn = (int64_t)dims[0] * dims[1] * dims[2];
    c.lev.push_back(v);
    for (int d = 0; d < 3; ++d) dims[d] = (dims[d] + 1) / 2;
    if (l + 1 < L && 3LL * dims[0] * dims[1] * dims[2] <= 10) {
      L = l + 2;
    }
  }
  c.L = (int)c.lev.size();
  if (c.L > tpo::kMaxLevels) {
    delete ctx;
    return TPO_E_UNSUPPORTED;
  }
  // the small levels and the dense coarsest solve run in one persistent
  // kernel: from the first level (>= 1) with at most kPersistentMaxNodes
  c.ps = c.L - 1;
  for (int l = 1; l < c.L; ++l)
    if (c.lev[l].nn <= tpo::kPersistentMaxNodes) {
      c.ps = l;
      break;
    }
  if (c.L - c.ps - 1 > tpo::kMaxCoarseLevels) c.ps = c.L - 1 - tpo::kMaxCoarseLevels;
  const int64_t ncoarse = 3 * c.lev[c.L - 1].nn;
  if (ncoarse > 12000) {
    c.err = "coarsest level too large for the dense solve; use more levels";
    delete ctx;
    return TPO_E_UNSUPPORTED;
  }
  int rc = tpo::build_element_constants(c);
  if (rc != TPO_OK) {
    delete ctx;
    return rc;
  }
  if (!tpo::build_filter_taps(c.nel, p->dx, p->rmin, c.taps)) {
    delete ctx;
    return TPO_E_UNSUPPORTED;
  }
  c.fix_h.assign(c.nn, 0);
  c.F_h.assign(3 * c.nn, 0.0);
  if (cudaGetDevice(&c.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return TPO_E_CUDA;
  }
  c.stream = c.own_stream;
  auto fail = [&](int code) {
    free_all(c);
    delete ctx;
    return code;
  };
  {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c.setup_stream, cudaStreamNonBlocking, greatest) !=
            cudaSuccess)
      return fail(TPO_E_CUDA);
    for (cudaEvent_t &e : c.setup_ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        return fail(TPO_E_CUDA);
  }
  for (int i = 0; i < tpo::kAuxStreams; ++i)
    if (cudaStreamCreateWithFlags(&c.aux_stream[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.aux_ev[i], cudaEventDisableTiming) != cudaSuccess)
      return fail(TPO_E_CUDA);
  for (cudaEvent_t &e : c.lev_ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return fail(TPO_E_CUDA);
  const size_t nio = std::max<size_t>(3 * c.nn, c.ne);
#define A(p, n) \
  if (dalloc(c, &(p), (n)) != TPO_OK) return fail(TPO_E_CUDA)
  A(c.taps_d, 1);
  A(c.finv, c.ne); A(c.K0lex, 576); A(c.GMi, 8 * 8 * 8 * 9);
  {
    const size_t nce = (size_t)((c.nel[0] + 1) / 2) * ((c.nel[1] + 1) / 2) * ((c.nel[2] + 1) / 2);
    A(c.gk_slot, nce); A(c.gk_elem, nce); A(c.gk_count, 1);
  }
  A(c.x, c.ne); A(c.rho, c.ne); A(c.E64, c.ne); A(c.dEdz, c.ne); A(c.E32, c.ne);
  A(c.Es64, c.ne); A(c.dEsdz64, c.ne);
  // level 1 on the tensor cores: even element counts (every level-1
  // element holds 2 x 2 x 2 fine ones) and level 1 above the persistent
  // levels
  c.l1tc_ok = c.L >= 2 && c.ps > 1 && c.nel[0] % 2 == 0 && c.nel[1] % 2 == 0 &&
              c.nel[2] % 2 == 0;
  if (c.l1tc_ok) {
    int tx = 0, ty = 0, zc = 0, nz = 0;
    tpo::l1tc_grid(c.lev[1], &tx, &ty, &zc, &nz);
    A(c.l1_B, 2 * 192 * 24); A(c.l1_cval, 3 * c.lev[1].nn); A(c.l1_cflag, (size_t)tx * ty * nz);
    A(c.l1_count, 1); A(c.l1_fault, 1);
  }
  A(c.fix, c.nn); A(c.idm, c.nn); A(c.F, 3 * c.nn); A(c.U, 3 * c.nn);
  A(c.scal, tpo::kScalCount); A(c.part, tpo::kPartCount); A(c.ticket, tpo::kMaxBatch + tpo::kAuxStreams);
  A(c.gbar, 1);
  A(c.tmpe, c.ne); A(c.tmpe2, c.ne); A(c.dev_info, 1);
  A(c.io_a, nio); A(c.io_b, nio);
#undef A
  // scalar mirror plus one staging row per column slot for per-column uploads
  if (cudaMallocHost(&c.scal_h, (tpo::kScalCount + tpo::kColScal * tpo::kMaxBatch) *
                                     sizeof(double)) !=
      cudaSuccess)
    return fail(TPO_E_CUDA);
  static constexpr int kLexToLocal[8] = {0, 1, 3, 2, 4, 5, 7, 6};
  double Kl[576];
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b)
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q)
          Kl[24 * (3 * a + r) + 3 * b + q] =
              c.K0[24 * (3 * kLexToLocal[a] + r) + 3 * kLexToLocal[b] + q];
  if (cudaMemcpyAsync(c.K0lex, Kl, sizeof(Kl), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
      cudaMemcpyAsync(c.GMi, c.GMi_h, sizeof(c.GMi_h), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
      cudaMemcpyAsync(c.taps_d, &c.taps, sizeof(c.taps), cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
    return fail(TPO_E_CUDA);
  tpo::launch_filter_rowsum(c, c.stream);
  if (cudaStreamSynchronize(c.stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return fail(TPO_E_CUDA);
  *out = ctx;
  return TPO_OK;
}

int tpo_destroy(tpo_ctx *ctx) {
  if (!ctx) return TPO_OK;
  cudaSetDevice(ctx->c.device);
  if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
  free_all(ctx->c);
  delete ctx;
  return TPO_OK;
}

int tpo_sizes(const tpo_ctx *ctx, int64_t *n_elem, int64_t *n_node,
              int32_t *n_levels) {
  if (!ctx) return TPO_E_ARG;
  if (n_elem) *n_elem = ctx->c.ne;
  if (n_node) *n_node = ctx->c.nn;
  if (n_levels) *n_levels = ctx->c.L;
  return TPO_OK;
}

int tpo_level_dims(const tpo_ctx *ctx, int32_t level, int32_t dims[3]) {
  if (!ctx || !dims || level < 0 || level >= ctx->c.L) return TPO_E_ARG;
  for (int d = 0; d < 3; ++d) dims[d] = ctx->c.lev[level].dims[d];
  return TPO_OK;
}

int tpo_add_bc(tpo_ctx *ctx, int32_t type, const double center[3],
               const double radius[3], const double limits[6],
               const double values[3], int64_t *n_selected) {
  if (!ctx) return TPO_E_ARG;
  Ctx &c = ctx->c;
  c.err.clear();
  REQUIRE(center && radius && limits && values, "null BC argument");
  REQUIRE(type == TPO_BC_SUPPORT || type == TPO_BC_LOAD, "unknown BC type");
  // Set_BC node selection (Inputs.cpp:116-124), nodes in increasing order
  const int64_t N[3] = {c.nel[0] + 1, c.nel[1] + 1, c.nel[2] + 1};
  int64_t cnt = 0;
  for (int64_t n = 0; n < c.nn; ++n) {
    const int64_t idx[3] = {n % N[0], (n / N[0]) % N[1], n / (N[0] * N[1])};
    double dist = 0;
    bool valid = true;
    for (int d = 0; d < 3; ++d) {
      const double xd = linspaced(0.0, c.prm.dx[d] * c.nel[d], N[d], idx[d]);
      const double t = (xd - center[d]) / radius[d];
      dist += t * t;
      valid = valid && xd >= limits[2 * d] && xd <= limits[2 * d + 1];
    }
    if (!(valid && dist <= 1)) continue;
    ++cnt;
    (type == TPO_BC_SUPPORT ? c.supp_node : c.load_node).push_back(n);
    for (int d = 0; d < 3; ++d) {
      if (type == TPO_BC_SUPPORT) {
        if (values[d] != 0) c.fix_h[n] |= (uint8_t)(1u << d);
        c.supp_val.push_back(values[d] != 0);
      } else {
        c.F_h[3 * n + d] += values[d];   // FEAnalysis.cpp:352-355
        c.load_val.push_back(values[d]);
      }
    }
  }
  if (n_selected) *n_selected = cnt;
  if (c.initialized) {
    cudaSetDevice(c.device);
    CK(cudaMemcpyAsync(c.fix, c.fix_h.data(), c.nn, cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.F, c.F_h.data(), sizeof(double) * 3 * c.nn, cudaMemcpyHostToDevice, c.stream));
    refresh_idm(c);
    CK(cudaStreamSynchronize(c.stream));
    c.assembled = false;
  }
  return TPO_OK;
}

int tpo_set_bc(tpo_ctx *ctx, const uint8_t *fixmask, const double *F, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {fixmask, F})) return rc;
  const cudaMemcpyKind k = mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
  if (fixmask) CK(cudaMemcpy(c.fix_h.data(), fixmask, c.nn, k));
  if (F) CK(cudaMemcpy(c.F_h.data(), F, sizeof(double) * 3 * c.nn, k));
  // the BC lists from the arrays: supported nodes and loaded nodes, in
  // increasing order
  if (fixmask) {
    c.supp_node.clear();
    c.supp_val.clear();
    for (int64_t n = 0; n < c.nn; ++n)
      if (c.fix_h[n]) {
        c.supp_node.push_back(n);
        for (int d = 0; d < 3; ++d) c.supp_val.push_back((c.fix_h[n] >> d) & 1);
      }
  }
  if (F) {
    c.load_node.clear();
    c.load_val.clear();
    for (int64_t n = 0; n < c.nn; ++n)
      if (c.F_h[3 * n] != 0 || c.F_h[3 * n + 1] != 0 || c.F_h[3 * n + 2] != 0) {
        c.load_node.push_back(n);
        for (int d = 0; d < 3; ++d) c.load_val.push_back(c.F_h[3 * n + d]);
      }
  }
  if (c.initialized) {
    CK(cudaMemcpyAsync(c.fix, c.fix_h.data(), c.nn, cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.F, c.F_h.data(), sizeof(double) * 3 * c.nn, cudaMemcpyHostToDevice, c.stream));
    refresh_idm(c);
    CK(cudaStreamSynchronize(c.stream));
    c.assembled = false;
  }
  return TPO_OK;
}

int tpo_get_bc(const tpo_ctx *cctx, uint8_t *fixmask, double *F, int mem) {
  tpo_ctx *ctx = const_cast<tpo_ctx *>(cctx);
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {fixmask, F})) return rc;
  const cudaMemcpyKind k = mem == TPO_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
  if (fixmask) CK(cudaMemcpy(fixmask, c.fix_h.data(), c.nn, k));
  if (F) CK(cudaMemcpy(F, c.F_h.data(), sizeof(double) * 3 * c.nn, k));
  return TPO_OK;
}

int tpo_fe_initialize(tpo_ctx *ctx) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = alloc_solver(c)) return rc;
  CK(cudaMemcpyAsync(c.fix, c.fix_h.data(), c.nn, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(c.F, c.F_h.data(), sizeof(double) * 3 * c.nn, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemsetAsync(c.U, 0, sizeof(double) * 3 * c.nn, c.stream));
  refresh_idm(c);
  CK(cudaStreamSynchronize(c.stream));
  c.initialized = true;
  c.assembled = false;
  return TPO_OK;
}

int tpo_mat_int_fnc(tpo_ctx *ctx, const double *x, double penal, double eps,
                    int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {x})) return rc;
  REQUIRE(x, "null design vector");
  REQUIRE(penal > 0 && eps >= 0 && eps < 1, "invalid penalty or eps");
  if (mem == TPO_MEM_DEVICE)
    CK(cudaMemcpyAsync(c.x, x, sizeof(double) * c.ne, cudaMemcpyDeviceToDevice, c.stream));
  else
    CK(cudaMemcpyAsync(c.x, x, sizeof(double) * c.ne, cudaMemcpyHostToDevice, c.stream));
  tpo::launch_filter(c, c.x, c.rho, false, c.stream);   // rho = P x (:35)
  tpo::launch_simp(c, penal, eps, c.stream);
  c.have_material = true;
  refresh_idm(c);
  c.assembled = false;
  return finish(c, TPO_OK);
}

int tpo_set_moduli(tpo_ctx *ctx, const double *E, const double *dEdz, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {E, dEdz})) return rc;
  REQUIRE(E, "null E");
  const cudaMemcpyKind k = mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(c.E64, E, sizeof(double) * c.ne, k, c.stream));
  if (dEdz) CK(cudaMemcpyAsync(c.dEdz, dEdz, sizeof(double) * c.ne, k, c.stream));
  tpo::launch_d2f(c.ne, c.E64, c.E32, c.stream);
  // given moduli carry no E_min split: the stress stiffness uses E itself,
  // and its derivative dEdz (zero when none is given)
  CK(cudaMemcpyAsync(c.Es64, c.E64, sizeof(double) * c.ne, cudaMemcpyDeviceToDevice, c.stream));
  if (dEdz)
    CK(cudaMemcpyAsync(c.dEsdz64, c.dEdz, sizeof(double) * c.ne, cudaMemcpyDeviceToDevice,
                       c.stream));
  else
    CK(cudaMemsetAsync(c.dEsdz64, 0, sizeof(double) * c.ne, c.stream));
  c.have_material = true;
  refresh_idm(c);
  CK(cudaStreamSynchronize(c.stream));
  c.assembled = false;
  return finish(c, TPO_OK);
}

int tpo_fe_assemble(tpo_ctx *ctx, const tpo_solve_opts *opts) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(c.initialized, "tpo_fe_initialize must be called first");
  REQUIRE(c.have_material, "no material: call tpo_mat_int_fnc or tpo_set_moduli");
  tpo_solve_opts o;
  if (opts) o = *opts; else tpo_default_solve_opts(&o);
  REQUIRE(o.cheb_degree >= 1 && o.cheb_hi > o.cheb_lo && o.cheb_lo >= 0 && o.power_its >= 1,
          "invalid smoother options");
  return finish(c, tpo::setup_hierarchy(c, o));
}

static int validate_solve(Ctx &c, const tpo_solve_opts &o) {
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first");
  REQUIRE(o.rtol > 0 && o.maxit >= 0, "invalid rtol/maxit");
  REQUIRE(o.precision == TPO_PREC_FP64 || o.precision == TPO_PREC_MIXED, "invalid precision");
  REQUIRE(o.cheb_degree == c.setup_opts.cheb_degree && o.cheb_lo == c.setup_opts.cheb_lo &&
              o.cheb_hi == c.setup_opts.cheb_hi,
          "smoother options differ from those given to tpo_fe_assemble");
  REQUIRE(o.precision == TPO_PREC_FP64 || (o.inner_rtol > 0 && o.inner_rtol < 1 && o.max_outer >= 1),
          "invalid mixed-precision options");
  return TPO_OK;
}

int tpo_fe_solve(tpo_ctx *ctx, const tpo_solve_opts *opts, tpo_solve_info *info) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  tpo_solve_opts o;
  if (opts) o = *opts; else { tpo_default_solve_opts(&o); o.cheb_degree = c.setup_opts.cheb_degree; }
  if (int rc = validate_solve(c, o)) return rc;
  return finish(c, tpo::solve(c, o, c.F, c.U, info));
}

// largest power of two <= min(n, cap)
static int pow2_block(int n, int cap) {
  int w = 1;
  while (2 * w <= n && 2 * w <= cap) w *= 2;
  return w;
}

// right-hand-side block for a solve: the caller's choice, else the faster
// per column of 4 and 8 on this context, measured once: one V-cycle and one
// fine apply of each block size on scratch columns (CUDA events on the
// context's stream)
static int rhs_block_for(Ctx &c, const tpo_solve_opts &o, int nrhs, int *block) {
  if (o.rhs_block > 0) {
    *block = o.rhs_block;
    return TPO_OK;
  }
  if (nrhs < 8) {
    *block = pow2_block(nrhs, 4);
    return TPO_OK;
  }
  if (!c.rhs_block_tuned) {
    if (int rc = ensure_columns(c, tpo::kMaxBatch)) return rc;
    float ms[2] = {0, 0};
    const int cand[2] = {4, 8};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int t = 0; t < 2; ++t) {
      for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(e0, c.stream));
        if (int rc = tpo::vcycle_block(c, c.setup_opts, o.precision, cand[t])) return rc;
        CK(cudaEventRecord(e1, c.stream));
        CK(cudaEventSynchronize(e1));
        float v = 0;
        CK(cudaEventElapsedTime(&v, e0, e1));
        if (rep > 0) ms[t] += v / cand[t];   // first run warms up
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.rhs_block_tuned = ms[1] < ms[0] ? 8 : 4;
  }
  *block = c.rhs_block_tuned;
  return TPO_OK;
}

int tpo_solve(tpo_ctx *ctx, const double *b, double *U, int32_t nrhs, int mem,
              const tpo_solve_opts *opts, tpo_solve_info *info) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {b, U})) return rc;
  REQUIRE(b && U && nrhs >= 1, "invalid solve arguments");
  tpo_solve_opts o;
  if (opts) o = *opts; else tpo_default_solve_opts(&o);
  if (int rc = validate_solve(c, o)) return rc;
  REQUIRE(o.rhs_block == 0 || o.rhs_block == 1 || o.rhs_block == 2 || o.rhs_block == 4 ||
              o.rhs_block == 8,
          "rhs_block must be 0, 1, 2, 4 or 8");
  int block = 1;
  if (int rc = rhs_block_for(c, o, nrhs, &block)) return finish(c, rc);
  const size_t n = 3 * c.nn;
  int worst = TPO_OK;
  tpo_solve_info acc{};
  for (int j0 = 0; j0 < nrhs;) {
    const int nb = pow2_block(nrhs - j0, block);
    if (int rc = ensure_columns(c, nb)) return rc;
    const double *bj = b + j0 * n;
    double *uj = U + j0 * n;
    const double *db = bj;
    double *du = uj;
    if (mem != TPO_MEM_DEVICE) {
      double *sb = nb > 1 ? c.io_ba : c.io_a;
      double *su = nb > 1 ? c.io_bb : c.io_b;
      CK(cudaMemcpyAsync(sb, bj, sizeof(double) * n * nb, cudaMemcpyHostToDevice, c.stream));
      CK(cudaMemcpyAsync(su, uj, sizeof(double) * n * nb, cudaMemcpyHostToDevice, c.stream));
      db = sb;
      du = su;
    }
    tpo_solve_info one{};
    const int rc = tpo::solve(c, o, db, du, &one, nb);
    if (rc < 0 && rc != TPO_E_BREAKDOWN) return finish(c, rc);
    if (int rc2 = copy_out(c, uj, du, n * nb, mem)) return rc2;
    if (rc < 0 ? rc < worst : (worst == TPO_OK && rc != TPO_OK)) worst = rc;
    acc.iterations += one.iterations;
    acc.outer += one.outer;
    acc.relres = std::max(acc.relres, one.relres);
    acc.solve_ms += one.solve_ms;
    j0 += nb;
  }
  acc.status = worst;
  acc.setup_ms = c.setup_ms;
  if (info) *info = acc;
  return finish(c, worst);
}

int tpo_apply(tpo_ctx *ctx, const double *u, double *y, int32_t nrhs,
              int32_t precision, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {u, y})) return rc;
  REQUIRE(u && y && nrhs >= 1, "invalid apply arguments");
  REQUIRE(c.initialized && c.have_material, "mesh not initialised or no material");
  REQUIRE(precision == TPO_PREC_FP64 || precision == TPO_PREC_MIXED, "invalid precision");
  const size_t n = 3 * c.nn;
  for (int j0 = 0; j0 < nrhs;) {
    const int nb = std::min<int>(nrhs - j0, tpo::kMaxBatch);
    if (int rc = ensure_columns(c, nb)) return rc;
    const double *du = u + j0 * n;
    double *dy = y + j0 * n;
    if (mem != TPO_MEM_DEVICE) {
      double *sa = nb > 1 ? c.io_ba : c.io_a;
      CK(cudaMemcpyAsync(sa, du, sizeof(double) * n * nb, cudaMemcpyHostToDevice, c.stream));
      du = sa;
      dy = nb > 1 ? c.io_bb : c.io_b;
    }
    if (precision == TPO_PREC_FP64) {
      tpo::launch_apply_fine<double>(c, c.E64, du, nullptr, dy, c.stream, nb);
    } else {
      tpo::launch_d2f(n * nb, du, c.r32, c.stream);
      tpo::launch_apply_fine<float>(c, c.E32, c.r32, nullptr, c.q32, c.stream, nb);
      tpo::launch_f2d(n * nb, c.q32, dy, c.stream);
    }
    if (int rc = copy_out(c, y + j0 * n, dy, n * nb, mem)) return rc;
    j0 += nb;
  }
  return finish(c, TPO_OK);
}

void tpo_default_eig_opts(tpo_eig_opts *o) {
  if (!o) return;
  o->nev = 6;
  o->block = 12;
  o->maxit = 500;
  o->tol = 1e-6;
  o->precond = TPO_PREC_FP64;
  o->seed = 1;
}

int tpo_ks_assemble(tpo_ctx *ctx) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(c.initialized && c.have_material, "mesh not initialised or no material");
  if (!c.ks_S) CK(cudaMalloc(&c.ks_S, sizeof(double) * 27 * c.nn));
  if (!c.ks_H) CK(cudaMalloc(&c.ks_H, sizeof(double) * 36 * c.ne));
  tpo::launch_ks_assemble(c, c.stream);
  CK(cudaStreamSynchronize(c.stream));
  c.ks_ready = true;
  return finish(c, TPO_OK);
}

int tpo_ks_apply(tpo_ctx *ctx, const double *u, double *y, int32_t nrhs, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {u, y})) return rc;
  REQUIRE(u && y && nrhs >= 1, "invalid apply arguments");
  REQUIRE(c.ks_ready, "tpo_ks_assemble must be called first");
  const size_t n = 3 * c.nn;
  for (int j0 = 0; j0 < nrhs;) {
    const int nb = std::min<int>(nrhs - j0, tpo::kMaxBatch);
    if (int rc = ensure_columns(c, nb)) return rc;
    const double *du = u + j0 * n;
    double *dy = y + j0 * n;
    if (mem != TPO_MEM_DEVICE) {
      double *sa = nb > 1 ? c.io_ba : c.io_a;
      CK(cudaMemcpyAsync(sa, du, sizeof(double) * n * nb, cudaMemcpyHostToDevice, c.stream));
      du = sa;
      dy = nb > 1 ? c.io_bb : c.io_b;
    }
    tpo::launch_ks_apply(c, du, dy, nb);
    if (int rc = copy_out(c, y + j0 * n, dy, n * nb, mem)) return rc;
    j0 += nb;
  }
  return finish(c, TPO_OK);
}

int tpo_buckling(tpo_ctx *ctx, const tpo_eig_opts *opts, double *lambda,
                 double *phi, int mem, tpo_eig_info *info) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {phi})) return rc;
  tpo_eig_opts o;
  if (opts) o = *opts; else tpo_default_eig_opts(&o);
  REQUIRE(lambda, "null lambda");
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first (preconditioner)");
  REQUIRE(c.ks_ready, "tpo_ks_assemble must be called first");
  REQUIRE(o.nev >= 1 && o.block >= o.nev && o.block <= 32, "need 1 <= nev <= block <= 32");
  REQUIRE(o.tol > 0 && o.maxit >= 0, "invalid tol/maxit");
  REQUIRE(o.precond == TPO_PREC_FP64 || o.precond == TPO_PREC_MIXED, "invalid precond");
  REQUIRE((int64_t)o.block <= 3 * c.nn, "block exceeds the number of dofs");
  tpo_eig_info one{};
  const int rc = tpo::buckling(c, o, lambda, phi, mem, &one);
  if (info) *info = one;
  if (rc < 0 && rc != TPO_E_BREAKDOWN) return finish(c, rc);
  return finish(c, rc);
}

int tpo_buckling_sensitivity(tpo_ctx *ctx, int32_t nev, const double *lambda,
                             const double *phi, double p, const tpo_solve_opts *opts,
                             double *value, double *dvdx, double *dvdrho, int mem,
                             tpo_solve_info *info) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {phi, dvdx, dvdrho})) return rc;
  REQUIRE(lambda && phi && value && dvdx, "null lambda, phi, value or dvdx");
  REQUIRE(nev >= 1 && nev <= tpo::kMaxEigPairs, "need 1 <= nev <= 32");
  REQUIRE(std::isfinite(p) && p >= 1.0, "the aggregation power p must be >= 1");
  REQUIRE(c.ks_ready, "tpo_ks_assemble must be called first");
  tpo_solve_opts o;
  if (opts) o = *opts; else tpo_default_solve_opts(&o);
  if (int rc = validate_solve(c, o)) return rc;
  const size_t n = 3 * c.nn, ne = c.ne;
  const size_t need = 2 * nev * n + 24 * ne + 2 * ne + (mem == TPO_MEM_DEVICE ? 0 : nev * n);
  if (c.bk_n < need) {
    dfree(c.bk_buf);
    c.bk_n = 0;
    CK(cudaMalloc(&c.bk_buf, sizeof(double) * need));
    c.bk_n = need;
  }
  double *rhs = c.bk_buf, *v = rhs + nev * n, *W = v + nev * n, *g = W + 24 * ne,
         *dx = g + ne;
  const double *ph = phi;
  if (mem != TPO_MEM_DEVICE) {
    double *st = dx + ne;
    CK(cudaMemcpyAsync(st, phi, sizeof(double) * nev * n, cudaMemcpyHostToDevice, c.stream));
    ph = st;
  }
  tpo_solve_info one{};
  const int rc = tpo::buckling_sensitivity(c, nev, lambda, ph, p, o, rhs, v, W, g,
                                           mem == TPO_MEM_DEVICE ? dvdx : dx, value, &one);
  if (info) *info = one;
  if (rc < 0 && rc != TPO_E_BREAKDOWN) return finish(c, rc);
  if (mem != TPO_MEM_DEVICE)
    if (int rc2 = copy_out(c, dvdx, dx, ne, mem)) return rc2;
  if (dvdrho)
    if (int rc2 = copy_out(c, dvdrho, g, ne, mem)) return rc2;
  CK(cudaStreamSynchronize(c.stream));
  return finish(c, rc);
}

int tpo_frequency(tpo_ctx *ctx, int32_t nvals, double density, const double *mlump,
                  const tpo_eig_opts *opts, double p, double *lambda, int32_t *nconv,
                  double *value, double *dvdx, int mem, tpo_eig_info *info) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {mlump, dvdx})) return rc;
  tpo_eig_opts o;
  if (opts) o = *opts; else tpo_default_eig_opts(&o);
  REQUIRE(lambda && nconv && value, "null lambda, nconv or value");
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first (K and preconditioner)");
  REQUIRE(nvals >= 1 && nvals + 3 <= tpo::kMaxEigPairs, "need 1 <= nvals <= 29");
  REQUIRE(std::isfinite(density) && density > 0.0, "density must be positive");
  REQUIRE(std::isfinite(p) && p >= 1.0, "the aggregation power p must be >= 1");
  REQUIRE(o.tol > 0 && o.maxit >= 0, "invalid tol/maxit");
  REQUIRE(o.precond == TPO_PREC_FP64 || o.precond == TPO_PREC_MIXED, "invalid precond");
  const size_t n = 3 * c.nn, ne = c.ne;
  const size_t need = n + tpo::kMaxEigPairs * n + 2 * ne + n;
  if (c.fq_n < need) {
    dfree(c.fq_buf);
    c.fq_n = 0;
    CK(cudaMalloc(&c.fq_buf, sizeof(double) * need));
    c.fq_n = need;
  }
  double *mdiag = c.fq_buf, *phi = mdiag + n, *g = phi + tpo::kMaxEigPairs * n,
         *dx = g + ne, *ml = dx + ne;
  const double *mld = mlump;
  if (mlump && mem != TPO_MEM_DEVICE) {
    CK(cudaMemcpyAsync(ml, mlump, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    mld = ml;
  }
  double lam[tpo::kMaxEigPairs] = {0.0};
  int nc = 0;
  tpo_eig_info one{};
  double *dout = dvdx ? (mem == TPO_MEM_DEVICE ? dvdx : dx) : nullptr;
  const int rc = tpo::frequency(c, nvals, density, mld, o, p, lam, &nc, mdiag, phi, g,
                                dout, value, &one);
  if (info) *info = one;
  if (rc < 0 && rc != TPO_E_BREAKDOWN) return finish(c, rc);
  *nconv = nc;
  for (int k = 0; k < nc; ++k) lambda[k] = lam[k];
  if (dvdx && mem != TPO_MEM_DEVICE) {
    if (int rc2 = copy_out(c, dvdx, dx, ne, mem)) return rc2;
    CK(cudaStreamSynchronize(c.stream));
  }
  return finish(c, rc);
}

void tpo_default_mma_opts(tpo_mma_opts *o) {
  if (!o) return;
  o->move = 0.5;     // MMA.h:21-23
  o->asyinit = 0.5;
  o->asyincr = 1.2;
  o->asydecr = 0.7;
  o->albefa = 0.1;
  o->raa0 = 1e-5;
  o->epsimin = 1e-7;
}

int tpo_mma_update(tpo_ctx *ctx, const tpo_mma_opts *opts, int32_t iter,
                   int32_t *fresh_start, int32_t m, double *x, double *xold1,
                   double *xold2, double *low, double *upp, const double *xmin,
                   const double *xmax, const double *dfdx, const double *g,
                   const double *dgdx, double *change, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {x, xold1, xold2, low, upp, xmin, xmax, dfdx, dgdx})) return rc;
  tpo_mma_opts o;
  if (opts) o = *opts; else tpo_default_mma_opts(&o);
  REQUIRE(fresh_start && x && xold1 && xold2 && low && upp && xmin && xmax && dfdx && g &&
              dgdx && change,
          "null MMA argument");
  REQUIRE(m >= 1 && m <= tpo::kMmaMaxM, "need 1 <= m <= 8 constraints");
  REQUIRE(o.epsimin > 0 && o.epsimin < 1, "epsimin must lie in (0, 1)");
  const int64_t n = c.ne;
  const int nv = m + m * (m + 1) / 2;
  const size_t npart = 2 * (size_t)tpo::kRedBlocks * nv;
  const size_t need = 4 * n + 2 * n * m + 8 * n + n * m + npart + 4;
  cudaStream_t s = c.stream;
  if (c.mma_n < need) {
    dfree(c.mma_buf);
    c.mma_n = 0;
    CK(cudaMalloc(&c.mma_buf, sizeof(double) * need));
    c.mma_n = need;
  }
  if (!c.mma_h) CK(cudaMallocHost(&c.mma_h, sizeof(double) * 4));
  double *alfa = c.mma_buf, *beta = alfa + n, *p0 = beta + n, *q0 = p0 + n, *P = q0 + n,
         *Q = P + n * m, *st = Q + n * m, *part = st + 8 * n + n * m, *out = part + npart;
  // device views of the caller's arrays (staged through st for host memory)
  double *dx = x, *d1 = xold1, *d2 = xold2, *dlo = low, *dup = upp;
  const double *dmin = xmin, *dmax = xmax, *ddf = dfdx, *ddg = dgdx;
  if (mem != TPO_MEM_DEVICE) {
    double *v[8] = {st, st + n, st + 2 * n, st + 3 * n, st + 4 * n, st + 5 * n, st + 6 * n,
                    st + 7 * n};
    const double *h[8] = {x, xold1, xold2, low, upp, xmin, xmax, dfdx};
    for (int i = 0; i < 8; ++i)
      CK(cudaMemcpyAsync(v[i], h[i], sizeof(double) * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st + 8 * n, dgdx, sizeof(double) * n * m, cudaMemcpyHostToDevice, s));
    dx = v[0]; d1 = v[1]; d2 = v[2]; dlo = v[3]; dup = v[4];
    dmin = v[5]; dmax = v[6]; ddf = v[7]; ddg = st + 8 * n;
  }
  // MMAsub (MMA.cpp:185-343) with DualSolve (:353-595) in one cooperative
  // launch; Set_m's constants a0 = b0 = 1, a = 0, c = 1000, d = 1 (:40-52)
  const bool fresh = *fresh_start && iter < 3;
  if (!fresh) *fresh_start = 0;
  tpo::MmaSolveArgs A{};
  A.n = n;
  A.m = m;
  A.fresh = fresh ? 1 : 0;
  A.k = tpo::MmaConst{o.move, o.asyinit, o.asyincr, o.asydecr, o.albefa, o.raa0};
  A.epsimin = o.epsimin;
  for (int j = 0; j < m; ++j) A.g[j] = g[j];
  A.x = dx; A.x1 = d1; A.x2 = d2; A.low = dlo; A.upp = dup;
  A.xmin = dmin; A.xmax = dmax; A.dfdx = ddf; A.dgdx = ddg;
  A.alfa = alfa; A.beta = beta; A.p0 = p0; A.q0 = q0; A.P = P; A.Q = Q;
  A.part = part; A.out = out; A.bar = c.gbar; A.fault = c.scal + tpo::kSlotFault;
  cudaError_t lerr = cudaSuccess;
  if (!tpo::launch_mma_solve(A, s, &lerr)) {
    c.err = "MMA update: the persistent kernel does not fit on this device";
    return TPO_E_CUDA;
  }
  CK(lerr);
  CK(cudaMemcpyAsync(c.mma_h, out, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(c.scal_h + tpo::kSlotFault, c.scal + tpo::kSlotFault, sizeof(double),
                     cudaMemcpyDeviceToHost, s));
  if (mem != TPO_MEM_DEVICE) {
    double *hv[5] = {x, xold1, xold2, low, upp};
    const double *dv[5] = {dx, d1, d2, dlo, dup};
    for (int i = 0; i < 5; ++i)
      CK(cudaMemcpyAsync(hv[i], dv[i], sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  if (c.scal_h[tpo::kSlotFault] != 0.0) {
    // a grid-barrier wait of the persistent kernel gave up: reset and report
    c.scal_h[tpo::kSlotFault] = 0.0;
    CK(cudaMemsetAsync(c.gbar, 0, sizeof(unsigned int), s));
    CK(cudaMemsetAsync(c.scal + tpo::kSlotFault, 0, sizeof(double), s));
    CK(cudaStreamSynchronize(s));
    c.err = "MMA update: a grid-barrier wait ran out";
    return TPO_E_CUDA;
  }
  if (c.mma_h[2] != 0.0) {
    c.err = "MMA dual Newton step: singular system";
    return TPO_E_BREAKDOWN;
  }
  *change = c.mma_h[0];
  c.mma_steps = (int)c.mma_h[1];
  return finish(c, TPO_OK);
}

int tpo_mma_last_info(const tpo_ctx *ctx, int32_t *newton_steps) {
  if (!ctx || !newton_steps) return TPO_E_ARG;
  *newton_steps = ctx->c.mma_steps;
  return TPO_OK;
}

int tpo_apply_f32(tpo_ctx *ctx, const float *u, float *y) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(u && y && u != y, "invalid apply arguments");
  if (int rc = check_mem(c, TPO_MEM_DEVICE, {u, y})) return rc;
  REQUIRE(c.initialized && c.have_material, "mesh not initialised or no material");
  tpo::launch_apply_fine<float>(c, c.E32, u, nullptr, y, c.stream);
  return finish(c, TPO_OK);
}

int tpo_apply_level(tpo_ctx *ctx, int32_t level, const double *u, double *y,
                    int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {u, y})) return rc;
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first");
  REQUIRE(level >= 0 && level < c.L && u && y, "invalid level or buffer");
  const size_t n = 3 * c.lev[level].nn;
  const double *du = nullptr;
  if (int rc = stage_in(c, u, n, mem, c.io_a, &du)) return rc;
  double *dy = (mem == TPO_MEM_DEVICE) ? y : c.io_b;
  if (level == 0)
    tpo::launch_apply_fine<double>(c, c.E64, du, nullptr, dy, c.stream);
  else
    tpo::launch_apply_stencil<double>(c.lev[level], c.lev[level].S64, du, nullptr, dy, c.stream);
  if (int rc = copy_out(c, y, dy, n, mem)) return rc;
  return finish(c, TPO_OK);
}

int tpo_apply_level_prec(tpo_ctx *ctx, int32_t level, const double *u, double *y,
                         int32_t precision, int mem) {
  if (precision == TPO_PREC_FP64) return tpo_apply_level(ctx, level, u, y, mem);
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {u, y})) return rc;
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first");
  REQUIRE(precision == TPO_PREC_MIXED, "precision must be TPO_PREC_FP64 or TPO_PREC_MIXED");
  REQUIRE(level >= 0 && (level == 0 || level < c.ps) && u && y,
          "FP32 operators exist on the levels above the persistent ones");
  const size_t n = 3 * c.lev[level].nn;
  const double *du = nullptr;
  if (int rc = stage_in(c, u, n, mem, c.io_a, &du)) return rc;
  double *dy = (mem == TPO_MEM_DEVICE) ? y : c.io_b;
  tpo::launch_d2f((int64_t)n, du, c.r32, c.stream);
  if (level == 0) {
    tpo::launch_apply_fine<float>(c, c.E32, c.r32, nullptr, c.q32, c.stream);
  } else if (level == 1 && tpo::l1_tensor(c)) {
    tpo::ApplyArgs<float> a{};
    a.u = c.r32;
    a.y = c.q32;
    tpo::launch_l1tc(c, tpo::IN_U, tpo::OUT_Y, a, c.stream);
  } else {
    tpo::launch_apply_stencil_sym<float>(c.lev[level], c.lev[level].H32, c.r32, nullptr,
                                         c.q32, c.stream, 1);
  }
  tpo::launch_f2d((int64_t)n, c.q32, dy, c.stream);
  if (int rc = copy_out(c, y, dy, n, mem)) return rc;
  return finish(c, TPO_OK);
}

int tpo_set_level1_form(tpo_ctx *ctx, int32_t form, int32_t *tensor) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(form == 0 || form == 1, "form must be 0 (automatic) or 1 (stored stencil)");
  c.l1_form = form;
  tpo::invalidate_graphs(c);
  if (tensor) *tensor = tpo::l1_tensor(c) ? 1 : 0;
  return finish(c, TPO_OK);
}

int tpo_vcycle(tpo_ctx *ctx, const double *r, double *z, int32_t precision, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {r, z})) return rc;
  REQUIRE(c.assembled, "tpo_fe_assemble must be called first");
  REQUIRE(r && z, "null buffer");
  const size_t n = 3 * c.nn;
  const double *dr = nullptr;
  if (int rc = stage_in(c, r, n, mem, c.io_a, &dr)) return rc;
  double *dz = (mem == TPO_MEM_DEVICE) ? z : c.io_b;
  if (int rc = tpo::vcycle_apply(c, c.setup_opts, precision, dr, dz)) return rc;
  if (int rc = copy_out(c, z, dz, n, mem)) return rc;
  return finish(c, TPO_OK);
}

int tpo_level_lambda(const tpo_ctx *ctx, int32_t level, double *lambda) {
  if (!ctx || !lambda || level < 0 || level >= ctx->c.L) return TPO_E_ARG;
  *lambda = ctx->c.lev[level].lam;
  return TPO_OK;
}

int tpo_get_vector(const tpo_ctx *cctx, const char *which, double *out, int mem) {
  tpo_ctx *ctx = const_cast<tpo_ctx *>(cctx);
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {out})) return rc;
  size_t n = 0;
  double *p = vec_ptr(c, which, &n);
  REQUIRE(p && out, "unknown vector name or null buffer");
  CK(cudaMemcpyAsync(out, p, sizeof(double) * n,
                     mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return TPO_OK;
}

int tpo_set_vector(tpo_ctx *ctx, const char *which, const double *in, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {in})) return rc;
  size_t n = 0;
  double *p = vec_ptr(c, which, &n);
  REQUIRE(p && in, "unknown vector name or null buffer");
  CK(cudaMemcpyAsync(p, in, sizeof(double) * n,
                     mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     c.stream));
  if (p == c.E64) {
    // new moduli invalidate the hierarchy
    tpo::launch_d2f(c.ne, c.E64, c.E32, c.stream);
    c.have_material = true;
    refresh_idm(c);
    c.assembled = false;
  }
  CK(cudaStreamSynchronize(c.stream));
  return finish(c, TPO_OK);
}

int tpo_compliance(tpo_ctx *ctx, double *C, double *dCdx, double *dCdrho, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {dCdx, dCdrho})) return rc;
  REQUIRE(c.initialized && c.have_material, "mesh not initialised or no material");
  const int64_t n = 3 * c.nn;
  if (C) {
    tpo::launch_dot<double>(c, n, c.U, c.F, c.scal + tpo::SC_COMPLIANCE, nullptr, c.stream);  // :19
    CK(cudaMemcpyAsync(c.scal_h + tpo::SC_COMPLIANCE, c.scal + tpo::SC_COMPLIANCE, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  }
  if (dCdx || dCdrho) {
    tpo::launch_sensitivity(c, c.U, c.tmpe, c.stream);                      // :37-46
    if (dCdrho)
      if (int rc = copy_out(c, dCdrho, c.tmpe, c.ne, mem)) return rc;
    if (dCdx) {
      tpo::launch_filter(c, c.tmpe, c.tmpe2, true, c.stream);              // :51
      if (int rc = copy_out(c, dCdx, c.tmpe2, c.ne, mem)) return rc;
    }
  }
  CK(cudaStreamSynchronize(c.stream));
  if (C) *C = c.scal_h[tpo::SC_COMPLIANCE];
  return finish(c, TPO_OK);
}

int tpo_volume(tpo_ctx *ctx, double *V, double *dVdx, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {dVdx})) return rc;
  REQUIRE(c.have_material, "no material");
  if (V) {
    tpo::launch_fill(c.ne, c.tmpe2, 1.0, c.stream);
    tpo::launch_dot<double>(c, c.ne, c.rho, c.tmpe2, c.scal + tpo::SC_VOLUME, nullptr, c.stream);
    CK(cudaMemcpyAsync(c.scal_h + tpo::SC_VOLUME, c.scal + tpo::SC_VOLUME, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  }
  if (dVdx) {
    tpo::launch_filter_adj_uniform(c, 1.0 / (double)c.ne, c.tmpe, c.stream);
    if (int rc = copy_out(c, dVdx, c.tmpe, c.ne, mem)) return rc;
  }
  CK(cudaStreamSynchronize(c.stream));
  if (V) *V = c.scal_h[tpo::SC_VOLUME] / (double)c.ne;
  return finish(c, TPO_OK);
}

int tpo_filter(tpo_ctx *ctx, const double *in, double *out, int32_t transpose, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {in, out})) return rc;
  REQUIRE(in && out, "null buffer");
  const double *din = nullptr;
  if (int rc = stage_in(c, in, c.ne, mem, c.io_a, &din)) return rc;
  double *dout = (mem == TPO_MEM_DEVICE) ? out : c.io_b;
  REQUIRE(din != dout, "filter input and output must differ");
  tpo::launch_filter(c, din, dout, transpose != 0, c.stream);
  if (int rc = copy_out(c, out, dout, c.ne, mem)) return rc;
  return finish(c, TPO_OK);
}

int tpo_oc_update(tpo_ctx *ctx, double *x, const double *xmin, const double *xmax,
                  double *dfdx, double g, const double *dgdx, double move,
                  double *change, int mem) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  if (int rc = check_mem(c, mem, {x, xmin, xmax, dfdx, dgdx})) return rc;
  REQUIRE(x && xmin && xmax && dfdx && dgdx, "null OC argument");
  const int64_t n = c.ne;
  if (!c.oc_ws) CK(cudaMalloc(&c.oc_ws, sizeof(double) * 6 * n));
  double *dx = c.oc_ws, *dxold = dx + n, *dmin = dx + 2 * n, *dmax = dx + 3 * n,
         *ddf = dx + 4 * n, *ddg = dx + 5 * n;
  const cudaMemcpyKind k = mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(dxold, x, sizeof(double) * n, k, c.stream));
  CK(cudaMemcpyAsync(dmin, xmin, sizeof(double) * n, k, c.stream));
  CK(cudaMemcpyAsync(dmax, xmax, sizeof(double) * n, k, c.stream));
  CK(cudaMemcpyAsync(ddf, dfdx, sizeof(double) * n, k, c.stream));
  CK(cudaMemcpyAsync(ddg, dgdx, sizeof(double) * n, k, c.stream));
  tpo::launch_oc_clip(n, ddf, c.stream);
  // bisection on the Lagrange multiplier (MMA.cpp:136-161): on the device in
  // one persistent launch; where the device cannot hold its grid, one
  // launch per trial with the branch taken on the host
  cudaError_t lerr = cudaSuccess;
  if (tpo::launch_oc_bisect(c, n, dx, dxold, dmin, dmax, ddf, ddg, move, g, c.stream, &lerr)) {
    CK(lerr);
  } else {
    double l1 = 0, l2 = 1e6;
    while (l2 - l1 > 1e-4) {
      const double lmid = 0.5 * (l1 + l2);
      tpo::launch_oc_step(c, n, dx, dxold, dmin, dmax, ddf, ddg, move, lmid, c.scal + tpo::SC_OC_DG, c.stream);
      CK(cudaMemcpyAsync(c.scal_h + tpo::SC_OC_DG, c.scal + tpo::SC_OC_DG, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
      CK(cudaStreamSynchronize(c.stream));
      if (g + c.scal_h[tpo::SC_OC_DG] > 0) l1 = lmid; else l2 = lmid;
    }
  }
  tpo::launch_oc_finish(c, n, dx, dxold, dmin, dmax, c.scal + tpo::SC_OC_CHANGE, c.stream);
  CK(cudaMemcpyAsync(c.scal_h + tpo::SC_OC_CHANGE, c.scal + tpo::SC_OC_CHANGE, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaMemcpyAsync(c.scal_h + tpo::kSlotFault, c.scal + tpo::kSlotFault, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  const cudaMemcpyKind ko = mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  CK(cudaMemcpyAsync(x, dx, sizeof(double) * n, ko, c.stream));
  CK(cudaMemcpyAsync(dfdx, ddf, sizeof(double) * n, ko, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (c.scal_h[tpo::kSlotFault] != 0.0) {
    // a grid-barrier wait of the bisection gave up: reset and report
    c.scal_h[tpo::kSlotFault] = 0.0;
    CK(cudaMemsetAsync(c.gbar, 0, sizeof(unsigned int), c.stream));
    CK(cudaMemsetAsync(c.scal + tpo::kSlotFault, 0, sizeof(double), c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.err = "OC bisection: a grid-barrier wait ran out";
    return TPO_E_CUDA;
  }
  if (change) *change = c.scal_h[tpo::SC_OC_CHANGE];
  return finish(c, TPO_OK);
}

int tpo_barrier_selftest(tpo_ctx *ctx, int32_t blocks, int32_t phases,
                         int32_t skip_block, int32_t max_polls, int32_t *completed) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(blocks >= 1 && blocks <= 64, "need 1 <= blocks <= 64");
  REQUIRE(phases >= 1 && phases <= 1024, "need 1 <= phases <= 1024");
  REQUIRE(max_polls >= 1 && max_polls <= tpo::kBarrierPolls, "need 1 <= max_polls <= 2^22");
  if (completed) *completed = 0;
  CK(tpo::launch_barrier_selftest(c, blocks, phases, skip_block, max_polls, c.stream));
  CK(cudaMemcpyAsync(c.scal_h + tpo::SC_SELFTEST, c.scal + tpo::SC_SELFTEST, sizeof(double),
                     cudaMemcpyDeviceToHost, c.stream));
  CK(cudaMemcpyAsync(c.scal_h + tpo::kSlotFault, c.scal + tpo::kSlotFault, sizeof(double),
                     cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (completed) *completed = (int32_t)c.scal_h[tpo::SC_SELFTEST];
  if (c.scal_h[tpo::kSlotFault] != 0.0) {
    // the same recovery as the persistent kernels' read-backs: the blocks
    // returned, the counter may be mid-barrier, so clear it and the flag
    c.scal_h[tpo::kSlotFault] = 0.0;
    CK(cudaMemsetAsync(c.gbar, 0, sizeof(unsigned int), c.stream));
    CK(cudaMemsetAsync(c.scal + tpo::kSlotFault, 0, sizeof(double), c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.err = "barrier self-test: a grid-barrier wait ran out";
    return TPO_E_CUDA;
  }
  return finish(c, TPO_OK);
}

int tpo_sync(tpo_ctx *ctx) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  CK(cudaStreamSynchronize(c.stream));
  return finish(c, TPO_OK);
}

int tpo_set_stream(tpo_ctx *ctx, void *stream) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : c.own_stream;
  if (next != c.stream) {
    // order the switch: the new stream waits for work already issued
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, c.stream));
    CK(cudaStreamWaitEvent(next, ev, 0));
    CK(cudaEventDestroy(ev));
    c.stream = next;
  }
  return TPO_OK;
}

int64_t tpo_kernel_launches(void) { return tpo::g_launches.load(); }

// ---- the reference's output and restart files ----------------------------

int tpo_write_vec_bin(const char *path, const double *v, int64_t n, int32_t index_bytes) {
  if (!path || (!v && n > 0) || n < 0) return io_fail("invalid Vec arguments");
  std::string err;
  return tpo::io::write_vec(path, v, n, index_bytes, err) ? TPO_OK : io_fail(err);
}

int tpo_read_vec_bin(const char *path, double *v, int64_t cap, int64_t *n,
                     int32_t index_bytes) {
  if (!path || !n) return io_fail("invalid Vec arguments");
  std::string err;
  std::vector<double> w;
  if (!tpo::io::read_vec(path, w, index_bytes, err)) return io_fail(err);
  *n = (int64_t)w.size();
  if (!v) return TPO_OK;
  if (cap < *n) return io_fail("Vec buffer too small");
  std::copy(w.begin(), w.end(), v);
  return TPO_OK;
}

int tpo_write_mat_bin(const char *path, int64_t M, int64_t N, const int64_t *rowptr,
                      const int64_t *col, const double *val, int32_t index_bytes) {
  if (!path || M < 0 || N < 0 || !rowptr) return io_fail("invalid matrix arguments");
  const int64_t nnz = rowptr[M];
  if (nnz > 0 && (!col || !val)) return io_fail("invalid matrix arguments");
  tpo::io::Csr A;
  A.M = M;
  A.N = N;
  A.rowptr.assign(rowptr, rowptr + M + 1);
  A.col.assign(col, col + nnz);
  A.val.assign(val, val + nnz);
  std::string err;
  return tpo::io::write_mat(path, A, index_bytes, err) ? TPO_OK : io_fail(err);
}

int tpo_read_mat_bin(const char *path, int64_t *M, int64_t *N, int64_t *nnz,
                     int64_t *rowptr, int64_t *col, double *val, int64_t cap_rows,
                     int64_t cap_nnz, int32_t index_bytes) {
  if (!path || !M || !N || !nnz) return io_fail("invalid matrix arguments");
  tpo::io::Csr A;
  std::string err;
  if (!tpo::io::read_mat(path, A, index_bytes, err)) return io_fail(err);
  *M = A.M;
  *N = A.N;
  *nnz = A.rowptr.back();
  if (!rowptr) return TPO_OK;
  if (cap_rows < A.M + 1 || cap_nnz < *nnz || !col || !val)
    return io_fail("matrix buffers too small");
  std::copy(A.rowptr.begin(), A.rowptr.end(), rowptr);
  std::copy(A.col.begin(), A.col.end(), col);
  std::copy(A.val.begin(), A.val.end(), val);
  return TPO_OK;
}

int tpo_mesh_out(tpo_ctx *ctx, const char *folder, double rmax, int32_t index_bytes) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(folder, "null folder");
  REQUIRE(rmax > 0, "rmax must be positive");
  REQUIRE(index_bytes == 4 || index_bytes == 8, "PetscInt size must be 4 or 8 bytes");
  const std::string d = folder_prefix(folder);
  const int ib = index_bytes;
  std::string err;
  auto ints = [&](const char *name, const std::vector<int64_t> &v) {
    return tpo::io::write_ints(d + name, v.data(), v.size(), ib, err);
  };
  auto raw = [&](const char *name, const void *p, size_t bytes) {
    return tpo::io::write_raw(d + name, p, bytes, err);
  };
  // distributions of one process (TopOpt.cpp:103-110)
  bool ok = ints("Element_Distribution.bin", {0, c.ne}) &&
            ints("Node_Distribution.bin", {0, c.nn});
  // elements (global node numbers, 8 per element) and node coordinates,
  // both row-major (:127-155)
  std::vector<int64_t> el(8 * (size_t)c.ne);
  for (int64_t e = 0; ok && e < c.ne; ++e) tpo::io::element_nodes(c.nel, e, el.data() + 8 * e);
  ok = ok && ints("elements.bin", el);
  el.clear();
  el.shrink_to_fit();
  std::vector<double> xyz(3 * (size_t)c.nn);
  const int64_t N[3] = {c.nel[0] + 1, c.nel[1] + 1, c.nel[2] + 1};
  for (int64_t n = 0; n < c.nn; ++n) {
    const int64_t idx[3] = {n % N[0], (n / N[0]) % N[1], n / (N[0] * N[1])};
    for (int k = 0; k < 3; ++k)
      xyz[3 * n + k] = linspaced(0.0, c.prm.dx[k] * c.nel[k], N[k], idx[k]);
  }
  ok = ok && raw("nodes.bin", xyz.data(), sizeof(double) * xyz.size());
  // BC lists (:157-310): loads, supports; no eigen-only supports, springs
  // or point masses are held by a context, so those files are empty
  std::vector<uint8_t> sv(c.supp_val.begin(), c.supp_val.end());
  ok = ok && ints("loadNodes.bin", c.load_node) &&
       raw("loads.bin", c.load_val.data(), sizeof(double) * c.load_val.size()) &&
       ints("supportNodes.bin", c.supp_node) && raw("supports.bin", sv.data(), sv.size()) &&
       ints("eigenSupportNodes.bin", {}) && raw("eigenSupports.bin", nullptr, 0) &&
       ints("springNodes.bin", {}) && raw("springs.bin", nullptr, 0) &&
       ints("massNodes.bin", {}) && raw("masses.bin", nullptr, 0);
  // the density filter, the max-length-scale filter and its edge vector
  // (:312-328; RecMesh.cpp:705-718)
  if (ok) ok = tpo::io::write_mat(d + "Filter.bin",
                                  tpo::io::filter_matrix(c.nel, c.prm.dx, c.prm.rmin, true),
                                  ib, err);
  if (ok) {
    const tpo::io::Csr R = tpo::io::filter_matrix(c.nel, c.prm.dx, rmax, false);
    std::vector<double> edge(R.M, 0.0);
    double mx = -INFINITY;
    for (int64_t r = 0; r < R.M; ++r) {
      double s = 0;
      for (int64_t t = R.rowptr[r]; t < R.rowptr[r + 1]; ++t) s += R.val[t];
      edge[r] = s;
      mx = std::max(mx, s);
    }
    for (double &v : edge) v = mx - v;   // VecAYPX(REdge, -1, max)
    ok = tpo::io::write_mat(d + "Max_Filter.bin", R, ib, err) &&
         tpo::io::write_vec(d + "Void_Edge_Volume.bin", edge.data(), R.M, ib, err);
  }
  // every element active (:330-340)
  if (ok) {
    std::vector<uint8_t> act(c.ne, 1);
    ok = raw("active.bin", act.data(), act.size());
  }
  // the multigrid interpolations and their column splits (:342-357)
  for (int l = 0; ok && l + 1 < c.L; ++l) {
    const tpo::io::Csr P = tpo::io::prolongation_matrix(c.lev[l].dims, c.lev[l + 1].dims);
    const std::string name = "P" + std::to_string(l) + ".bin";
    ok = tpo::io::write_mat(d + name, P, ib, err) &&
         tpo::io::write_ints(d + name + ".split", &P.N, 1, ib, err);
  }
  if (!ok) {
    c.err = err;
    return TPO_E_ARG;
  }
  return TPO_OK;
}

int tpo_print_vals(tpo_ctx *ctx, const char *folder, const char *name_suffix,
                   const double *phiB, int32_t nB, const double *phiD, int32_t nD,
                   int32_t index_bytes) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(folder && name_suffix, "null folder or suffix");
  REQUIRE(c.initialized && c.have_material, "mesh not initialised or no material");
  REQUIRE(nB >= 0 && nD >= 0 && (nB == 0 || phiB) && (nD == 0 || phiD), "invalid mode arrays");
  const std::string d = folder_prefix(folder), sfx = name_suffix;
  std::string err;
  // U, x, V, Es, E (TopOpt.cpp:451-479)
  struct Item {
    const char *file, *vec;
  } items[] = {{"U", "U"}, {"x", "x"}, {"V", "rho"}, {"Es", "Es"}, {"E", "E"}};
  for (const Item &it : items) {
    size_t n = 0;
    double *p = vec_ptr(c, it.vec, &n);
    REQUIRE(p, "vector not allocated");
    std::vector<double> h(n);
    CK(cudaMemcpyAsync(h.data(), p, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (!tpo::io::write_vec(d + it.file + sfx + ".bin", h.data(), (int64_t)n, index_bytes, err)) {
      c.err = err;
      return TPO_E_ARG;
    }
  }
  // buckling and dynamic mode shapes, one file per column (:481-507)
  const int64_t nd = 3 * c.nn;
  for (int i = 0; i < nB; ++i)
    if (!tpo::io::write_vec(d + "phiB" + sfx + "_mode" + std::to_string(i) + ".bin",
                            phiB + nd * i, nd, index_bytes, err)) {
      c.err = err;
      return TPO_E_ARG;
    }
  for (int i = 0; i < nD; ++i)
    if (!tpo::io::write_vec(d + "phiD_" + sfx + "_mode" + std::to_string(i) + ".bin",
                            phiD + nd * i, nd, index_bytes, err)) {
      c.err = err;
      return TPO_E_ARG;
    }
  return TPO_OK;
}

int tpo_load_mesh(const char *folder, const tpo_mesh_params *params, int32_t index_bytes,
                  tpo_ctx **out) {
  if (!folder || !params || !out) return io_fail("invalid load arguments");
  *out = nullptr;
  const std::string d = folder_prefix(folder);
  const int ib = index_bytes;
  std::string err;
  std::vector<int64_t> edist, ndist, el;
  std::vector<char> nodes_raw;
  // distributions, elements, nodes (RecMesh.cpp:42-86)
  if (!tpo::io::read_ints(d + "Element_Distribution.bin", edist, ib, err) ||
      !tpo::io::read_ints(d + "Node_Distribution.bin", ndist, ib, err) ||
      !tpo::io::read_ints(d + "elements.bin", el, ib, err) ||
      !tpo::io::read_raw(d + "nodes.bin", nodes_raw, err))
    return io_fail(err);
  if (edist.size() < 2 || ndist.size() < 2) return io_fail("empty distribution file");
  const int64_t ne = edist.back(), nn = ndist.back();
  if (ne < 1 || (int64_t)el.size() != 8 * ne || (int64_t)nodes_raw.size() != 24 * nn)
    return io_fail("elements.bin / nodes.bin do not hold a 3-D hex8 mesh of the given sizes");
  const double *xyz = reinterpret_cast<const double *>(nodes_raw.data());
  // the structured grid: spacing from element 0 (as LoadMesh's elemSize,
  // :300-306), counts from the extent, then every node and element checked
  double dx[3], lo[3], hi[3];
  const int corner[3] = {1, 3, 4};
  for (int k = 0; k < 3; ++k) {
    dx[k] = xyz[3 * el[corner[k]] + k] - xyz[3 * el[0] + k];
    lo[k] = hi[k] = xyz[k];
  }
  for (int64_t n = 0; n < nn; ++n)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], xyz[3 * n + k]);
      hi[k] = std::max(hi[k], xyz[3 * n + k]);
    }
  int nel[3];
  for (int k = 0; k < 3; ++k) {
    if (!(dx[k] > 0)) return io_fail("not a structured mesh: non-positive element size");
    nel[k] = (int)std::llround((hi[k] - lo[k]) / dx[k]);
  }
  if ((int64_t)nel[0] * nel[1] * nel[2] != ne ||
      (int64_t)(nel[0] + 1) * (nel[1] + 1) * (nel[2] + 1) != nn)
    return io_fail("not a structured box mesh (element and node counts)");
  for (int64_t e = 0; e < ne; ++e) {
    int64_t nd[8];
    tpo::io::element_nodes(nel, e, nd);
    for (int a = 0; a < 8; ++a)
      if (el[8 * e + a] != nd[a]) return io_fail("element connectivity is not the structured numbering");
  }
  const int64_t NN[3] = {nel[0] + 1, nel[1] + 1, nel[2] + 1};
  for (int64_t n = 0; n < nn; ++n) {
    const int64_t idx[3] = {n % NN[0], (n / NN[0]) % NN[1], n / (NN[0] * NN[1])};
    for (int k = 0; k < 3; ++k) {
      const double want = lo[k] + idx[k] * dx[k];
      if (std::fabs(xyz[3 * n + k] - want) > 1e-9 * (std::fabs(hi[k] - lo[k]) + dx[k]))
        return io_fail("node coordinates are not a regular grid");
    }
  }
  // BC lists (:112-290); springs, eigen-only supports and passive elements
  // have no counterpart in a context
  std::vector<int64_t> ln, sn, spn, en;
  std::vector<char> lv, sv, act;
  if (!tpo::io::read_ints(d + "loadNodes.bin", ln, ib, err) ||
      !tpo::io::read_raw(d + "loads.bin", lv, err) ||
      !tpo::io::read_ints(d + "supportNodes.bin", sn, ib, err) ||
      !tpo::io::read_raw(d + "supports.bin", sv, err) ||
      !tpo::io::read_ints(d + "springNodes.bin", spn, ib, err))
    return io_fail(err);
  if (lv.size() != 24 * ln.size() || sv.size() != 3 * sn.size())
    return io_fail("BC value files do not match their node lists");
  if (!spn.empty()) return io_fail("springs are not supported", TPO_E_UNSUPPORTED);
  if (tpo::io::read_ints(d + "eigenSupportNodes.bin", en, ib, err) && !en.empty())
    return io_fail("eigen-analysis supports are not supported", TPO_E_UNSUPPORTED);
  if (tpo::io::read_raw(d + "active.bin", act, err))
    for (char a : act)
      if (!a) return io_fail("passive elements are not supported", TPO_E_UNSUPPORTED);
  for (int64_t n : ln)
    if (n < 0 || n >= nn) return io_fail("load node out of range");
  for (int64_t n : sn)
    if (n < 0 || n >= nn) return io_fail("support node out of range");
  // levels: as given, else one more than the interpolations saved
  tpo_mesh_params p = *params;
  for (int k = 0; k < 3; ++k) {
    p.nel[k] = nel[k];
    p.dx[k] = dx[k];
  }
  if (p.mg_levels <= 0) {
    int cnt = 0;
    std::vector<char> probe;
    while (tpo::io::read_raw(d + "P" + std::to_string(cnt) + ".bin", probe, err)) ++cnt;
    if (cnt > 0) p.mg_levels = cnt + 1;
  }
  tpo_ctx *ctx = nullptr;
  if (int rc = tpo_create(&p, &ctx)) {
    if (ctx) tpo_destroy(ctx);
    return io_fail("context creation failed", rc);
  }
  Ctx &c = ctx->c;
  // the saved filter must be the one this context rebuilds from rmin
  // (:314-325 reads it instead)
  tpo::io::Csr Pf;
  if (tpo::io::read_mat(d + "Filter.bin", Pf, ib, err)) {
    const tpo::io::Csr Q = tpo::io::filter_matrix(c.nel, c.prm.dx, c.prm.rmin, true);
    bool same = Pf.M == Q.M && Pf.N == Q.N && Pf.rowptr == Q.rowptr && Pf.col == Q.col;
    for (size_t t = 0; same && t < Q.val.size(); ++t)
      same = std::fabs(Pf.val[t] - Q.val[t]) <= 1e-12 * std::fabs(Q.val[t]);
    if (!same) {
      tpo_destroy(ctx);
      return io_fail("Filter.bin is not the density filter of radius rmin on this mesh");
    }
  }
  // BCs as the Set_BC lists held them: support flags OR-ed, loads summed
  const double *lval = reinterpret_cast<const double *>(lv.data());
  for (size_t i = 0; i < sn.size(); ++i) {
    c.supp_node.push_back(sn[i]);
    for (int k = 0; k < 3; ++k) {
      const bool f = sv[3 * i + k] != 0;
      c.supp_val.push_back(f);
      if (f) c.fix_h[sn[i]] |= (uint8_t)(1u << k);
    }
  }
  for (size_t i = 0; i < ln.size(); ++i) {
    c.load_node.push_back(ln[i]);
    for (int k = 0; k < 3; ++k) {
      c.load_val.push_back(lval[3 * i + k]);
      c.F_h[3 * ln[i] + k] += lval[3 * i + k];
    }
  }
  *out = ctx;
  return TPO_OK;
}

int tpo_load_design(tpo_ctx *ctx, const char *folder, const double *penalties, int32_t npen,
                    double *x, double *penal, int32_t *start, int32_t index_bytes) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(folder && x && (npen == 0 || penalties), "invalid design-load arguments");
  const std::string d = folder_prefix(folder);
  // RecMesh.cpp:391-404: x = 0.5, then x_pen<p>.bin for each penalty in
  // turn until one is missing; the penalty reached is the one the run
  // resumes at (Main.cpp:52-56)
  std::fill(x, x + c.ne, 0.5);
  double pen = penal ? *penal : 0.0;
  std::string err;
  for (int32_t i = 0; i < npen; ++i) {
    pen = penalties[i];
    char name[64];
    std::snprintf(name, sizeof name, "x_pen%g.bin", pen);   // ostream << double
    std::vector<double> v;
    std::vector<char> probe;
    if (!tpo::io::read_raw(d + name, probe, err)) break;
    if (!tpo::io::read_vec(d + name, v, index_bytes, err)) {
      c.err = err;
      return TPO_E_ARG;
    }
    REQUIRE((int64_t)v.size() == c.ne, "saved design has the wrong length");
    std::copy(v.begin(), v.end(), x);
  }
  int32_t s = 0;
  while (s < npen && penalties[s] < pen) ++s;
  if (penal) *penal = pen;
  if (start) *start = s;
  return TPO_OK;
}

int tpo_load_point_masses(tpo_ctx *ctx, const char *folder, double *mlump,
                          int32_t index_bytes) {
  if (int rc = begin(ctx)) return rc;
  Ctx &c = ctx->c;
  REQUIRE(folder && mlump, "invalid mass-load arguments");
  const std::string d = folder_prefix(folder);
  std::string err;
  std::vector<int64_t> mn;
  std::vector<char> mv;
  // RecMesh.cpp:147-180: massNodes.bin and masses.bin (3 per node)
  if (!tpo::io::read_ints(d + "massNodes.bin", mn, index_bytes, err) ||
      !tpo::io::read_raw(d + "masses.bin", mv, err)) {
    c.err = err;
    return TPO_E_ARG;
  }
  REQUIRE(mv.size() == 24 * mn.size(), "masses.bin does not match massNodes.bin");
  std::fill(mlump, mlump + 3 * c.nn, 0.0);
  const double *m = reinterpret_cast<const double *>(mv.data());
  for (size_t i = 0; i < mn.size(); ++i) {
    REQUIRE(mn[i] >= 0 && mn[i] < c.nn, "mass node out of range");
    for (int k = 0; k < 3; ++k) mlump[3 * mn[i] + k] += m[3 * i + k];
  }
  return TPO_OK;
}

}  // extern "C"
