// Host orchestration of the FE solve: GMG set-up (PCSetUp), the V-cycle,
// FP64 PCG and the mixed FP32 PCG with FP64 residual replacement.
//
// Reference behaviour restated here (FEAnalysis.cpp:387-416, :541-573,
// :673): KSP CG, nonzero initial guess, convergence on the unpreconditioned
// residual ||b - K u|| <= rtol ||b||, PCMG with Galerkin coarse operators,
// Chebyshev/Jacobi smoothing and a direct (here Cholesky) coarse solve.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <type_traits>

#include "coarse.h"
#include "solver.h"

namespace tpo {

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Cheb {
  double inv_theta, sigma, delta, rho0, theta;
};

Cheb cheb_of(double lam, const tpo_solve_opts &o) {
  const double a = o.cheb_lo * lam, b = o.cheb_hi * lam;
  const double theta = 0.5 * (b + a), delta = 0.5 * (b - a);
  const double sigma = theta / delta;
  return {1.0 / theta, sigma, delta, 1.0 / sigma, theta};
}

template <typename T>
struct LV {
  T *b, *x, *r, *d, *a;
  const T *S, *dinv;
};

LV<double> lv(Level &v, double *) {
  return {v.b64, v.x64, v.r64, v.d64, v.a64, v.S64, v.dinv64};
}
LV<float> lv(Level &v, float *) {
  return {v.b32, v.x32, v.r32, v.d32, v.a32, v.S32, v.dinv32};
}

const double *fineE(const Ctx &c, double *) { return c.E64; }
const float *fineE(const Ctx &c, float *) { return c.E32; }

const double *halfS(const Level &v, double *) { return v.H64; }
const float *halfS(const Level &v, float *) { return v.H32; }

// A_l u (or b - A_l u): matrix-free on the finest level, the symmetric
// half-stored Galerkin stencil between it and the persistent levels, the
// full FP64 stencil on the persistent levels (used there only for the set-up
// eigenvalue estimate)
template <typename T>
void level_apply(Ctx &c, int l, const T *u, const T *b, T *y, cudaStream_t s,
                 int nb = 1) {
  if (l == 0) {
    launch_apply_fine<T>(c, fineE(c, (T *)nullptr), u, b, y, s, nb);
  } else if (l < c.ps) {
    if constexpr (std::is_same<T, float>::value) {
      if (l == 1 && nb == 1 && l1_tensor(c)) {
        ApplyArgs<float> a{};
        a.u = u;
        a.b = b;
        a.y = y;
        launch_l1tc(c, IN_U, b ? OUT_RESID : OUT_Y, a, s);
        return;
      }
    }
    launch_apply_stencil_sym<T>(c.lev[l], halfS(c.lev[l], (T *)nullptr), u, b,
                                y, s, nb);
  } else {
    const int64_t ld = 3 * c.lev[l].nn;
    for (int j = 0; j < nb; ++j)
      launch_apply_stencil<T>(c.lev[l], lv(c.lev[l], (T *)nullptr).S, u + j * ld,
                              b ? b + j * ld : nullptr, y + j * ld, s);
  }
}

// parameters of the persistent kernel for levels ps .. L-1 (kernels_coarse.cu)
template <typename T>
CoarseCycle<T> coarse_cycle_params(Ctx &c, const tpo_solve_opts &o) {
  CoarseCycle<T> P{};
  P.nlev = c.L - 1 - c.ps;
  for (int i = 0; i < P.nlev; ++i) {
    Level &v = c.lev[c.ps + i];
    LV<T> w = lv(v, (T *)nullptr);
    CoarseLevel<T> &L = P.lev[i];
    for (int d = 0; d < 3; ++d) L.dims[d] = v.dims[d];
    L.nn = v.nn;
    L.A = (sizeof(T) == 8) ? reinterpret_cast<const T *>(v.A64)
                           : reinterpret_cast<const T *>(v.A32);
    L.dinv = w.dinv;
    L.b = w.b;
    L.xout = w.x;
    L.r = w.r;
    L.d0 = w.d;
    L.res = w.a;
    if (sizeof(T) == 8) {
      L.xpre = reinterpret_cast<T *>(v.w64);
      L.d1 = reinterpret_cast<T *>(v.e64);
    } else {
      L.xpre = reinterpret_cast<T *>(v.w32);
      L.d1 = reinterpret_cast<T *>(v.e32);
    }
    const Cheb ch = cheb_of(v.lam, o);
    L.inv_theta = static_cast<T>(ch.inv_theta);
    L.deg = std::min(o.cheb_degree, kMaxChebDegree);
    double rho = ch.rho0;
    for (int k = 1; k < L.deg; ++k) {
      const double rn = 1.0 / (2.0 * ch.sigma - rho);
      L.c1[k] = static_cast<T>(rn * rho);
      L.c2[k] = static_cast<T>(2.0 * rn / ch.delta);
      rho = rn;
    }
  }
  Level &cl = c.lev[c.L - 1];
  LV<T> cw = lv(cl, (T *)nullptr);
  P.Ainv = c.Ainv;
  P.nc = c.nc;
  for (int d = 0; d < 3; ++d) P.cdims[d] = cl.dims[d];
  P.bc = cw.b;
  P.xc = cw.x;
  P.bar = c.gbar;
  P.fault = c.scal + kSlotFault;
  return P;
}

template <typename T>
void vcycle_rec(Ctx &c, int l, const T *b, T *x, const tpo_solve_opts &o,
                cudaStream_t s, int nb) {
  if (l == c.L - 1) {
    launch_coarse_gemv<T>(c.nc, c.Ainv, b, x, s, nb);
    return;
  }
  if (l >= 1 && l == c.ps) {
    // levels ps..L-1 in one cooperative launch; b and x are this level's
    // own b and x buffers (the restriction above wrote b)
    CoarseCycle<T> P = coarse_cycle_params<T>(c, o);
    P.nb = nb;
    c.coarse_err = launch_coarse_cycle<T>(P, s);
    return;
  }
  Level &v = c.lev[l];
  LV<T> w = lv(v, (T *)nullptr);
  const int64_t n = 3 * v.nn;
  const Cheb ch = cheb_of(v.lam, o);
  const bool fine_fused = (l == 0);
  const bool sym_fused = (l >= 1 && l < c.ps && nb == 1);
  if (o.cheb_degree == 2 && (fine_fused || sym_fused)) {
    // Chebyshev(2): the smoother updates run in the epilogues of the
    // operator kernel (the matrix-free apply on the fine level,
    // kernels_apply_staged.cu; the half-stored stencil below the
    // persistent levels, kernels_mg.cu), 4 launches per level
    const T *E = fineE(c, (T *)nullptr);
    const T *H = halfS(v, (T *)nullptr);
    const double rn = 1.0 / (2.0 * ch.sigma - ch.rho0);
    ApplyArgs<T> a{};
    a.b = b;
    a.dinv = w.dinv;
    a.invtheta = static_cast<T>(ch.inv_theta);
    a.theta = static_cast<T>(ch.theta);
    a.c1 = static_cast<T>(rn * ch.rho0);
    a.c2 = static_cast<T>(2.0 * rn / ch.delta);
    bool tensor = false;   // level 1 in FP32 on the tensor cores
    if constexpr (std::is_same<T, float>::value) tensor = l == 1 && l1_tensor(c);
    auto fused = [&](int in, int out) {
      if (fine_fused) {
        launch_apply_fused<T>(c, E, in, out, a, s, nb);
      } else if (tensor) {
        if constexpr (std::is_same<T, float>::value) launch_l1tc(c, in, out, a, s);
      } else {
        launch_apply_sym_fused<T>(v, H, in, out, a, s);
      }
    };
    a.y = x;
    fused(IN_CHEB, OUT_CHEB2);                                 // pre-smooth
    a.u = x;                                                   // residual
    a.y = w.a;
    fused(IN_U, OUT_RESID);
    Level &cv = c.lev[l + 1];
    LV<T> cw = lv(cv, (T *)nullptr);
    launch_restrict<T>(v, cv, w.a, cw.b, s, nb);
    vcycle_rec<T>(c, l + 1, cw.b, cw.x, o, s, nb);
    launch_prolong_add<T>(v, cv, cw.x, x, s, nb);
    a.u = x;                                                   // post-smooth
    a.y = w.d;
    a.y2 = w.r;
    fused(IN_U, OUT_POST0);
    a.u = w.d;
    a.y = x;
    a.y2 = w.r;
    fused(IN_U, OUT_POST1);
    return;
  }
  // pre-smoothing from a zero guess
  launch_cheb_init<T>(n, w.dinv, b, w.r, w.d, x, ch.inv_theta, true, s, nb);
  double rho = ch.rho0;
  for (int k = 1; k < o.cheb_degree; ++k) {
    level_apply<T>(c, l, w.d, nullptr, w.a, s, nb);
    const double rn = 1.0 / (2.0 * ch.sigma - rho);
    launch_cheb_step<T>(n, w.dinv, w.a, w.r, w.d, x, rn * rho, 2.0 * rn / ch.delta, s, nb);
    rho = rn;
  }
  // residual, restriction, coarse correction, prolongation
  level_apply<T>(c, l, x, b, w.a, s, nb);
  Level &cv = c.lev[l + 1];
  LV<T> cw = lv(cv, (T *)nullptr);
  launch_restrict<T>(v, cv, w.a, cw.b, s, nb);
  vcycle_rec<T>(c, l + 1, cw.b, cw.x, o, s, nb);
  launch_prolong_add<T>(v, cv, cw.x, x, s, nb);
  // post-smoothing from the corrected x
  level_apply<T>(c, l, x, b, w.r, s, nb);
  launch_cheb_init<T>(n, w.dinv, b, w.r, w.d, x, ch.inv_theta, false, s, nb);
  rho = ch.rho0;
  for (int k = 1; k < o.cheb_degree; ++k) {
    level_apply<T>(c, l, w.d, nullptr, w.a, s, nb);
    const double rn = 1.0 / (2.0 * ch.sigma - rho);
    launch_cheb_step<T>(n, w.dinv, w.a, w.r, w.d, x, rn * rho, 2.0 * rn / ch.delta, s, nb);
    rho = rn;
  }
}

// one CG iteration (p = z + beta p after the first): V-cycle, rho, p, q,
// pq, update, for nb columns.  Kept free of host synchronisation so it can
// be captured.
template <typename T>
void cg_body(Ctx &c, int64_t n, T *x, T *r, T *z, T *p, T *q,
             const tpo_solve_opts &o, bool first, cudaStream_t s, int nb) {
  double *sc = c.scal;
  vcycle_rec<T>(c, 0, r, z, o, s, nb);
  launch_rho_dot<T>(c, n, r, z, s, nb);
  launch_cg_p<T>(n, z, p, sc, first, s, nb);
  launch_apply_fine<T>(c, fineE(c, (T *)nullptr), p, nullptr, q, s, nb);
  launch_dot<T>(c, n, p, q, sc + 2, nullptr, s, nb);
  launch_cg_update<T>(c, n, x, r, p, q, sc, sc + 3, s, nb);
}

#define CK(call)                                                       \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      c.err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return TPO_E_CUDA;                                               \
    }                                                                  \
  } while (0)

// copy the scalars of nb columns to the host mirror
int readback(Ctx &c, int nb) {
  CK(cudaMemcpyAsync(c.scal_h, c.scal, sizeof(double) * kColScal * nb,
                     cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (c.scal_h[kSlotFault] != 0.0) {
    // 1: a grid barrier of the coarse-grid kernel gave up waiting (the
    // blocks returned and the counter may be mid-barrier, so clear both);
    // 2: the level-1 tensor-core kernel gave up waiting for an MMA
    const bool mma = c.scal_h[kSlotFault] == 2.0;
    c.scal_h[kSlotFault] = 0.0;
    CK(cudaMemsetAsync(c.gbar, 0, sizeof(unsigned int), c.stream));
    CK(cudaMemsetAsync(c.scal + kSlotFault, 0, sizeof(double), c.stream));
    c.err = mma ? "level-1 tensor-core kernel: an MMA wait ran out"
                : "coarse-grid kernel: a grid-barrier wait ran out";
    return TPO_E_CUDA;
  }
  return TPO_OK;
}

// device scalar slot `slot` of nb columns <- host values, through a pinned
// staging row of its own after the scalar mirror: the copy is asynchronous,
// so uploads of different slots may follow one another without a
// synchronisation, but a slot must not be uploaded twice before the stream
// has passed the first copy
int upload_slot(Ctx &c, int slot, const double *v, int nb) {
  double *st = c.scal_h + kScalCount + slot * kMaxBatch;
  for (int j = 0; j < nb; ++j) st[j] = v[j];
  CK(cudaMemcpy2DAsync(c.scal + slot, sizeof(double) * kColScal, st,
                       sizeof(double), sizeof(double), nb,
                       cudaMemcpyHostToDevice, c.stream));
  return TPO_OK;
}

// device slot dst <- slot src for nb columns
int copy_slot(Ctx &c, int dst, int src, int nb) {
  CK(cudaMemcpy2DAsync(c.scal + dst, sizeof(double) * kColScal, c.scal + src,
                       sizeof(double) * kColScal, sizeof(double), nb,
                       cudaMemcpyDeviceToDevice, c.stream));
  return TPO_OK;
}

// The device-resident PCG loop.  A CUDA graph holds a while node whose
// body is one CG iteration followed by k_loop_check, which applies the
// host loop's per-column test on the device (breakdown: rho, pq not
// positive or r.r not finite; convergence: r.r <= target) and freezes the
// finished columns, then keeps the loop going while a column is active,
// fewer than maxit iterations are done and no coarse-grid barrier has run
// out.  k_loop_start opens the loop under the same condition; the while
// node's default is closed, so a loop that is never opened runs nothing.
__global__ void k_loop_start(double *scal, int nb, cudaGraphConditionalHandle h) {
  bool any = false;
  for (int j = 0; j < nb; ++j) any |= scal[j * kColScal + 6] == 0.0;
  const bool go = any && scal[SC_LOOP_K] < scal[SC_LOOP_MAXIT] && scal[kSlotFault] == 0.0;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

__global__ void k_loop_check(double *scal, int nb, cudaGraphConditionalHandle h) {
  const double k = scal[SC_LOOP_K] + 1.0;
  scal[SC_LOOP_K] = k;
  bool any = false;
  for (int j = 0; j < nb; ++j) {
    double *sc = scal + j * kColScal;
    if (sc[6] != 0.0) continue;
    scal[SC_LOOP_ITS + j] = k;
    const double rho = sc[0], pq = sc[2], rr = sc[3];
    if (!(rho > 0) || !(pq > 0) || !isfinite(rr)) {
      scal[SC_LOOP_STATUS + j] = -1.0;
      sc[6] = 1.0;
    } else if (rr <= scal[SC_LOOP_TARGET + j]) {
      scal[SC_LOOP_STATUS + j] = 1.0;
      sc[6] = 1.0;
    } else {
      any = true;
    }
  }
  const bool go = any && k < scal[SC_LOOP_MAXIT] && scal[kSlotFault] == 0.0;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// the loop graph of cg_body (not the first iteration) for nb columns;
// *body_nodes receives the kernel launches of one iteration
template <typename T>
int build_loop_graph(Ctx &c, const tpo_solve_opts &o, T *x, T *r, T *z, T *p, T *q,
                     int nb, cudaGraphExec_t *exec, long long *body_nodes) {
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  cudaGraph_t graph = nullptr;
  CK(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault));
  cudaGraphNode_t start;
  {
    cudaKernelNodeParams kp = {};
    double *scal = c.scal;
    void *args[] = {&scal, &nb, &h};
    kp.func = (void *)k_loop_start;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    CK(cudaGraphAddKernelNode(&start, graph, nullptr, 0, &kp));
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t loop;
  CK(cudaGraphAddNode(&loop, graph, &start, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const long long before = g_launches.load();
  CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                   cudaStreamCaptureModeThreadLocal));
  cg_body<T>(c, n, x, r, z, p, q, o, false, s, nb);
  k_loop_check<<<1, 1, 0, s>>>(c.scal, nb, h);
  count_launch();
  const cudaError_t ce = cudaStreamEndCapture(s, &body);
  // captured launches run when the graph is launched, not now
  *body_nodes = g_launches.load() - before;
  count_launch(-*body_nodes);
  CK(ce);
  CK(cudaGraphInstantiate(exec, graph, 0));
  CK(cudaGraphDestroy(graph));
  return TPO_OK;
}

// PCG on the fine operator in precision T for nb columns.  x holds the
// initial guesses and r must already hold b - K x; ||r_j||^2 is in slot 3
// of the host mirror.  Column j stops at ||r_j||^2 <= target_rr[j]; columns
// with frozen[j] set do not iterate.  On return its[j] = iterations of
// column j and st[j] = its status.  resume: continue the previous run's
// recurrence (the first iteration forms p = z + beta p from the p and rho
// left in place) instead of starting with p = z.  With o.use_graph the
// iterations after the first run in one launch of the loop graph, with the
// per-iteration test on the device; otherwise each iteration is launched
// from the host and tested there.
template <typename T>
int pcg_loop(Ctx &c, const tpo_solve_opts &o, T *x, T *r, T *z, T *p, T *q,
             const double *target_rr, int maxit, int nb, double *frozen,
             int *its, int *st, bool resume = false) {
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  cudaGraphExec_t &g = (sizeof(T) == 8) ? c.graph64 : c.graph32;
  const void *&gx = (sizeof(T) == 8) ? c.graph64_x : c.graph32_x;
  int &gnb = (sizeof(T) == 8) ? c.graph64_nb : c.graph32_nb;
  long long &gnodes = (sizeof(T) == 8) ? c.graph64_nodes : c.graph32_nodes;
  int active = 0;
  for (int j = 0; j < nb; ++j) {
    its[j] = 0;
    st[j] = TPO_NOT_CONVERGED;
    if (frozen[j] == 0.0 && c.scal_h[j * kColScal + 3] <= target_rr[j]) {
      frozen[j] = 1.0;
      st[j] = TPO_OK;
    }
    if (frozen[j] != 0.0 && st[j] == TPO_NOT_CONVERGED) st[j] = TPO_OK;
    if (frozen[j] == 0.0) ++active;
  }
  if (!active) return TPO_OK;
  if (int rc = upload_slot(c, 6, frozen, nb)) return rc;
  // the host test of one iteration's scalars (in the mirror)
  auto host_test = [&](int k) -> int {
    bool changed = false;
    for (int j = 0; j < nb; ++j) {
      if (frozen[j] != 0.0) continue;
      const double *hs = c.scal_h + j * kColScal;
      const double rho = hs[0], pq = hs[2], rr = hs[3];
      its[j] = k;
      if (!(rho > 0) || !(pq > 0) || !std::isfinite(rr)) {
        st[j] = TPO_E_BREAKDOWN;
        c.err = "CG breakdown (indefinite preconditioner/operator or non-finite residual)";
      } else if (rr <= target_rr[j]) {
        st[j] = TPO_OK;
      } else {
        continue;
      }
      frozen[j] = 1.0;
      changed = true;
      --active;
    }
    if (changed && active)
      if (int rc = upload_slot(c, 6, frozen, nb)) return rc;
    return TPO_OK;
  };
  int k = 0;
  // a device without conditional graph nodes runs the host-tested loop
  static bool loop_graphs_ok = true;
  if (!o.use_graph || !loop_graphs_ok) {
    while (k < maxit && active) {
      cg_body<T>(c, n, x, r, z, p, q, o, k == 0 && !resume, s, nb);
      CK(cudaGetLastError());
      CK(c.coarse_err);
      ++k;
      if (int rc = readback(c, nb)) return rc;
      if (int rc = host_test(k)) return rc;
    }
  } else {
    if (!resume && maxit > 0) {   // the first iteration (p = z), from the host
      cg_body<T>(c, n, x, r, z, p, q, o, true, s, nb);
      CK(cudaGetLastError());
      CK(c.coarse_err);
      k = 1;
      if (int rc = readback(c, nb)) return rc;
      if (int rc = host_test(k)) return rc;
    }
    if (active && k < maxit) {
      if (!g || gx != (const void *)x || gnb != nb) {
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
        if (build_loop_graph<T>(c, o, x, r, z, p, q, nb, &g, &gnodes) != TPO_OK) {
          // not available here: clear the (non-sticky) error and continue
          // with the host-tested loop from iteration k
          cudaGetLastError();
          c.err.clear();
          if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
          }
          loop_graphs_ok = false;
          while (k < maxit && active) {
            cg_body<T>(c, n, x, r, z, p, q, o, false, s, nb);
            CK(cudaGetLastError());
            CK(c.coarse_err);
            ++k;
            if (int rc = readback(c, nb)) return rc;
            if (int rc = host_test(k)) return rc;
          }
          goto done;
        }
        CK(c.coarse_err);
        gx = x;
        gnb = nb;
      }
      // loop state: per column target, iterations so far and status; the
      // iterations done and the limit (one copy from the pinned mirror; the
      // host does not touch those mirror slots until the read-back below)
      double *hs = c.scal_h;
      for (int j = 0; j < kMaxBatch; ++j) {
        hs[SC_LOOP_TARGET + j] = j < nb ? target_rr[j] : 0.0;
        hs[SC_LOOP_ITS + j] = j < nb ? its[j] : 0.0;
        hs[SC_LOOP_STATUS + j] = 0.0;
      }
      hs[SC_LOOP_K] = k;
      hs[SC_LOOP_MAXIT] = maxit;
      CK(cudaMemcpyAsync(c.scal + SC_LOOP_TARGET, hs + SC_LOOP_TARGET,
                         sizeof(double) * (SC_LOOP_MAXIT + 1 - SC_LOOP_TARGET),
                         cudaMemcpyHostToDevice, s));
      CK(cudaGraphLaunch(g, s));
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(hs + SC_LOOP_ITS, c.scal + SC_LOOP_ITS,
                         sizeof(double) * (SC_LOOP_K + 1 - SC_LOOP_ITS),
                         cudaMemcpyDeviceToHost, s));
      if (int rc = readback(c, nb)) return rc;   // synchronises
      const int k_end = (int)hs[SC_LOOP_K];
      count_launch(1 + (long long)(k_end - k) * gnodes);
      k = k_end;
      for (int j = 0; j < nb; ++j) {
        if (frozen[j] != 0.0) continue;
        its[j] = (int)hs[SC_LOOP_ITS + j];
        const double stj = hs[SC_LOOP_STATUS + j];
        if (stj < 0.0) {
          st[j] = TPO_E_BREAKDOWN;
          c.err = "CG breakdown (indefinite preconditioner/operator or non-finite residual)";
        } else if (stj > 0.0) {
          st[j] = TPO_OK;
        } else {
          continue;
        }
        frozen[j] = 1.0;
        --active;
      }
    }
  }
done:
  int worst = TPO_OK;
  for (int j = 0; j < nb; ++j)
    if (st[j] < 0 ? st[j] < worst : (worst == TPO_OK && st[j] != TPO_OK))
      worst = st[j];
  return worst;
}

}  // namespace

void invalidate_graphs(Ctx &c) {
  if (c.graph64) cudaGraphExecDestroy(c.graph64);
  if (c.graph32) cudaGraphExecDestroy(c.graph32);
  c.graph64 = c.graph32 = nullptr;
  c.graph64_x = c.graph32_x = nullptr;
  c.graph64_nb = c.graph32_nb = 0;
}

// power iteration for lambda_max(D^-1 A_l) on stream s, no host sync.  The
// start vector is the splitmix64 sequence the oracle shares.  The iterates
// v_{k+1} = D^-1 A v_k are not normalised (lambda_max(D^-1 A) is a small
// number, so 15 steps stay far inside the FP64 range): each step is the
// apply and one fused pass for the diagonal scaling and the squared norm,
// which leaves ||v_k||^2 in scal[SC_POWER + l] and ||v_{k-1}||^2 in
// scal[SC_POWER_PREV + l].  lambda = ||v_k|| / ||v_{k-1}|| is then the
// estimate ||D^-1 A a|| of the normalised iteration, a = v_{k-1}/||v_{k-1}||.
template <typename T>
void power_iteration_t(Ctx &c, int l, int its, cudaStream_t s, double *part,
                       unsigned int *ticket) {
  Level &v = c.lev[l];
  const int64_t n = 3 * v.nn;
  LV<T> wv = lv(v, (T *)nullptr);
  T *a = wv.d, *w = wv.a;
  double *nrm = c.scal + SC_POWER + l, *prev = c.scal + SC_POWER_PREV + l;
  launch_power_start<T>(n, a, s);
  launch_dot<T>(c, n, a, a, nrm, nullptr, s, 1, part, ticket);
  for (int k = 0; k < its; ++k) {
    level_apply<T>(c, l, a, nullptr, w, s);
    launch_scale_diag_dot<T>(c, n, w, wv.dinv, nrm, prev, s, part, ticket);
    std::swap(a, w);
  }
}

// fp32: the hierarchy is set up for the mixed form, whose smoothers run in
// FP32; the fine level and the half-stored level below it (the levels with
// FP32 operators) then take their Chebyshev bounds from FP32 iterations
void power_iteration(Ctx &c, int l, int its, cudaStream_t s, double *part,
                     unsigned int *ticket, bool fp32) {
  if (fp32 && (l == 0 || l < c.ps))
    power_iteration_t<float>(c, l, its, s, part, ticket);
  else
    power_iteration_t<double>(c, l, its, s, part, ticket);
}

// lambda of level l from the power iteration's two last squared norms in
// the host mirror
double power_lambda(const Ctx &c, int l) {
  return std::sqrt(c.scal_h[SC_POWER + l] / c.scal_h[SC_POWER_PREV + l]);
}

int estimate_lambda(Ctx &c, int l, int its, double *lam) {
  cudaStream_t s = c.stream;
  power_iteration(c, l, its, s, nullptr, nullptr, false);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c.scal_h + SC_POWER, c.scal + SC_POWER,
                     sizeof(double) * (SC_POWER_PREV + kMaxLevels - SC_POWER),
                     cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *lam = power_lambda(c, l);
  return TPO_OK;
}

namespace {

// the hierarchy on stream s (see setup_hierarchy)
int setup_on(Ctx &c, const tpo_solve_opts &o, cudaStream_t s) {
  const double t0 = now_ms();
  invalidate_graphs(c);
  // Chebyshev bounds (power iterations) of each smoothed level run on a
  // side stream as soon as that level's operator is built on s, with their
  // own reduction scratch: level l on side stream l % kAuxStreams, so the
  // levels' latency-bound iterations overlap one another as well as the
  // Galerkin chain and the coarsest factorisation on s
  auto level_ready = [&](int l) -> int {
    if (l + 1 >= c.L) return TPO_OK;   // the coarsest level is not smoothed
    const int i = l % kAuxStreams;
    CK(cudaEventRecord(c.lev_ev[l], s));
    CK(cudaStreamWaitEvent(c.aux_stream[i], c.lev_ev[l], 0));
    power_iteration(c, l, o.power_its, c.aux_stream[i],
                    c.part + kAuxPart + i * kRedBlocks, c.ticket + kMaxBatch + i,
                    o.precision == TPO_PREC_MIXED);
    return TPO_OK;
  };
  auto join = [&]() {
    for (int i = 0; i < kAuxStreams; ++i) {
      cudaEventRecord(c.aux_ev[i], c.aux_stream[i]);
      cudaStreamWaitEvent(s, c.aux_ev[i], 0);
    }
  };
  // fine level: Jacobi diagonal (and the assembled stencil when it is the
  // only level)
  launch_fine_diag(c, c.lev[0].dinv64, c.lev[0].dinv32, s);
  if (c.L == 1) launch_fine_stencil(c, c.S0, s);
  if (int rc = level_ready(0)) return rc;
  for (int l = 0; l + 1 < c.L; ++l) {
    if (l == 0) {
      if (launch_galerkin_fine(c, c.lev[1].S64, s) != TPO_OK) {
        join();
        c.err = "level-1 Galerkin product failed";
        return TPO_E_CUDA;
      }
    } else {
      launch_galerkin_dims(c.lev[l], c.lev[l].S64, c.lev[l + 1].S64, c.gd_tmp, s);
    }
    launch_stencil_diag(c.lev[l + 1], c.lev[l + 1].S64, c.lev[l + 1].dinv64,
                        c.lev[l + 1].dinv32, s);
    if (l + 1 < c.ps) {
      launch_stencil_to_half(c.lev[l + 1].nn, c.lev[l + 1].S64, c.lev[l + 1].H64,
                             c.lev[l + 1].H32, s);
    }
    if (l + 1 >= c.ps && l + 1 < c.L - 1)
      launch_soa_to_aos(c.lev[l + 1].nn, c.lev[l + 1].S64, c.lev[l + 1].A64,
                        c.lev[l + 1].A32, s);
    if (int rc = level_ready(l + 1)) {
      join();
      return rc;
    }
  }
  CK(cudaGetLastError());
  // coarsest level: the explicit inverse of the dense operator (blocked
  // Gauss-Jordan, kernels_coarse_inv.cu) for a bandwidth-parallel GEMV
  // inside the V-cycle
  Level &cl = c.lev[c.L - 1];
  const double *Sc = (c.L == 1) ? c.S0 : cl.S64;
  const int64_t nc = 3 * cl.nn;
  c.nc = nc;
  launch_to_dense(cl, Sc, c.Ainv, s);
  launch_coarse_inverse(nc, c.Ainv, c.Adense, c.dev_info, s);
  CK(cudaGetLastError());
  int info_h = 0, l1_fault_h = 0;
  unsigned int l1_rows_h = 0;
  CK(cudaMemcpyAsync(&info_h, c.dev_info, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (c.l1tc_ok) {
    CK(cudaMemcpyAsync(&l1_fault_h, c.l1_fault, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&l1_rows_h, c.l1_count, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  c.l1_nrows = (int)std::min<size_t>(l1_rows_h, c.l1_cap);
  if (l1_fault_h != 0) {
    c.err = "level-1 correction rows exceed their capacity";
    join();
    return TPO_E_CUDA;
  }
  if (info_h != 0) {
    c.err = "coarsest operator is not positive definite (pivot " +
            std::to_string(info_h - 1) + ")";
    join();
    return TPO_E_BREAKDOWN;
  }
  // Chebyshev bounds from the side stream
  join();
  CK(cudaMemcpyAsync(c.scal_h + SC_POWER, c.scal + SC_POWER,
                     sizeof(double) * (SC_POWER_PREV + kMaxLevels - SC_POWER),
                     cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int l = 0; l + 1 < c.L; ++l) c.lev[l].lam = power_lambda(c, l);
  c.setup_opts = o;
  c.assembled = true;
  c.setup_ms = now_ms() - t0;
  return TPO_OK;
}

}  // namespace

// FEAssemble/PCSetUp: the Galerkin hierarchy, the coarsest inverse and the
// Chebyshev bounds.  The work runs on the context's highest-priority set-up
// stream, ordered after everything already issued on c.stream, and c.stream
// waits for it on every return path.
int setup_hierarchy(Ctx &c, const tpo_solve_opts &o) {
  CK(cudaEventRecord(c.setup_ev[0], c.stream));
  CK(cudaStreamWaitEvent(c.setup_stream, c.setup_ev[0], 0));
  const int rc = setup_on(c, o, c.setup_stream);
  CK(cudaEventRecord(c.setup_ev[1], c.setup_stream));
  CK(cudaStreamWaitEvent(c.stream, c.setup_ev[1], 0));
  return rc;
}

int vcycle_apply(Ctx &c, const tpo_solve_opts &o, int precision,
                 const double *r, double *z) {
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  if (precision == TPO_PREC_FP64) {
    vcycle_rec<double>(c, 0, r, z, o, s, 1);
  } else {
    launch_d2f(n, r, c.r32, s);
    vcycle_rec<float>(c, 0, c.r32, c.z32, o, s, 1);
    launch_f2d(n, c.z32, z, s);
  }
  CK(cudaGetLastError());
  CK(c.coarse_err);
  return TPO_OK;
}

// one V-cycle and one fine apply on nb scratch columns (for timing the
// right-hand-side block size)
int vcycle_block(Ctx &c, const tpo_solve_opts &o, int precision, int nb) {
  cudaStream_t s = c.stream;
  if (precision == TPO_PREC_FP64) {
    vcycle_rec<double>(c, 0, c.r64, c.z64, o, s, nb);
    launch_apply_fine<double>(c, c.E64, c.z64, nullptr, c.q64, s, nb);
  } else {
    vcycle_rec<float>(c, 0, c.r32, c.z32, o, s, nb);
    launch_apply_fine<float>(c, c.E32, c.z32, nullptr, c.q32, s, nb);
  }
  CK(cudaGetLastError());
  CK(c.coarse_err);
  return TPO_OK;
}

int vcycle_cols(Ctx &c, const tpo_solve_opts &o, int precision, const double *r,
                double *z, int nb) {
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  if (precision == TPO_PREC_FP64) {
    vcycle_rec<double>(c, 0, r, z, o, s, nb);
  } else {
    launch_d2f(n * nb, r, c.r32, s);
    vcycle_rec<float>(c, 0, c.r32, c.z32, o, s, nb);
    launch_f2d(n * nb, c.z32, z, s);
  }
  CK(cudaGetLastError());
  CK(c.coarse_err);
  return TPO_OK;
}

// Solve K x_j = b_j for nb columns (stride 3 nn); x holds the initial
// guesses.  Column j converges at ||b_j - K x_j|| <= rtol ||b_j||.  info
// aggregates the block (iterations and outer steps summed over columns,
// the largest relative residual, the worst status); col, if given, gets
// one record per column.
int solve(Ctx &c, const tpo_solve_opts &o, const double *b, double *x,
          tpo_solve_info *info, int nb, tpo_solve_info *col) {
  const double t0 = now_ms();
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  double *sc = c.scal;
  if (nb < 1 || nb > kMaxBatch || nb > c.nb_cap) {
    c.err = "right-hand-side block exceeds the allocated columns";
    return TPO_E_ARG;
  }
  double bn[kMaxBatch], rn[kMaxBatch], target[kMaxBatch], tgt2[kMaxBatch];
  double frozen[kMaxBatch];
  int its_total[kMaxBatch], outer[kMaxBatch], status[kMaxBatch];
  int its[kMaxBatch], st[kMaxBatch];

  launch_dot<double>(c, n, b, b, sc + 4, nullptr, s, nb);
  launch_apply_fine<double>(c, c.E64, x, b, c.r64, s, nb);
  launch_dot<double>(c, n, c.r64, c.r64, sc + 5, nullptr, s, nb);
  CK(cudaGetLastError());
  if (int rc = readback(c, nb)) return rc;
  int active = 0;
  for (int j = 0; j < nb; ++j) {
    bn[j] = std::sqrt(c.scal_h[j * kColScal + 4]);
    rn[j] = std::sqrt(c.scal_h[j * kColScal + 5]);
    target[j] = o.rtol * bn[j];
    tgt2[j] = target[j] * target[j];
    its_total[j] = outer[j] = 0;
    status[j] = TPO_NOT_CONVERGED;
    frozen[j] = 0.0;
    if (bn[j] == 0.0) {
      CK(cudaMemsetAsync(x + j * n, 0, sizeof(double) * n, s));
      rn[j] = 0.0;
      status[j] = TPO_OK;
      frozen[j] = 1.0;
    } else if (rn[j] <= target[j]) {
      status[j] = TPO_OK;
      frozen[j] = 1.0;
    } else {
      ++active;
    }
  }
  if (active && o.precision == TPO_PREC_FP64) {
    // r = b - K x already in r64 and ||r||^2 in slot 5
    for (int j = 0; j < nb; ++j) c.scal_h[j * kColScal + 3] = c.scal_h[j * kColScal + 5];
    if (int rc = copy_slot(c, 3, 5, nb)) return rc;
    pcg_loop<double>(c, o, x, c.r64, c.z64, c.p64, c.q64, tgt2, o.maxit, nb,
                     frozen, its, st);
    // report the true residual
    launch_apply_fine<double>(c, c.E64, x, b, c.r64, s, nb);
    launch_dot<double>(c, n, c.r64, c.r64, sc + 5, nullptr, s, nb);
    if (int rc = readback(c, nb)) return rc;
    for (int j = 0; j < nb; ++j) {
      if (status[j] == TPO_OK) continue;   // converged before the loop
      its_total[j] = its[j];
      outer[j] = 1;
      status[j] = st[j];
      rn[j] = std::sqrt(c.scal_h[j * kColScal + 5]);
    }
  } else if (active) {
    // mixed: ONE FP32 PCG+GMG recurrence on K d_j = r_j/||r_j|| with FP64
    // residual replacement (the "reliable updates" of Sleijpen & van der
    // Vorst, 1996; residual replacement, van der Vorst & Ye, 2000).  When
    // every live column's FP32 residual has dropped by inner_rtol, or to
    // 0.7x what its target asks, x += ||r|| d in FP64, the FP64 residual
    // b - K x replaces the FP32 one (rescaled to unit norm), and the FP32
    // recurrence resumes with its search direction and rho rescaled to the
    // new units.  Restarting from p = z instead (plain defect correction)
    // would throw away the Krylov space and cost 1-2 iterations per pass.
    // Convergence is only ever decided on the FP64 residual.  Passes are
    // kept short (inner_rtol 1e-2 by default): over a long FP32 pass the
    // recursive residual drifts from the true one (K p cancels heavily in
    // FP32 for smooth p), and the old search direction then no longer fits
    // the replaced residual.  If the FP64 residual comes out more than 2x
    // above what the FP32 recurrence predicted, the next pass restarts from
    // p = z instead of resuming.
    // the FP32 residual r/||r|| has unit norm to FP32 rounding, so its
    // squared norm (the base of each pass's drop) is taken as 1 on the host
    launch_to_f32_scaled(n, c.r64, sc + 5, c.r32, s, nb);
    CK(cudaMemsetAsync(c.x32, 0, sizeof(float) * n * nb, s));
    for (int j = 0; j < nb; ++j) c.scal_h[j * kColScal + 3] = rn[j] > 0.0 ? 1.0 : 0.0;
    bool resume = false;
    int passes = 0;
    while (passes < o.max_outer) {
      double trig[kMaxBatch], inner_frozen[kMaxBatch];
      bool live[kMaxBatch];
      int nlive = 0, maxit_in = 0;
      for (int j = 0; j < nb; ++j) {
        live[j] = !(status[j] == TPO_OK || status[j] == TPO_E_BREAKDOWN ||
                    rn[j] <= target[j] || its_total[j] >= o.maxit);
        inner_frozen[j] = live[j] ? 0.0 : 1.0;
        trig[j] = 0.0;
        if (!live[j]) continue;
        ++nlive;
        const double eta = std::max(o.inner_rtol, 0.7 * target[j] / std::max(rn[j], 1e-300));
        trig[j] = eta * eta * c.scal_h[j * kColScal + 3];
        maxit_in = std::max(maxit_in, o.maxit - its_total[j]);
      }
      if (!nlive) break;
      pcg_loop<float>(c, o, c.x32, c.r32, c.z32, c.p32, c.q32, trig, maxit_in, nb,
                      inner_frozen, its, st, resume);
      ++passes;
      double predicted[kMaxBatch];   // ||r|| the FP32 recurrence ended at
      for (int j = 0; j < nb; ++j)
        predicted[j] = rn[j] * std::sqrt(std::max(c.scal_h[j * kColScal + 3], 0.0));
      // FP64 residual replacement (columns that were done before this pass
      // have a zero x32 and keep their x)
      launch_axpy_f32(n, x, c.x32, sc + 5, s, nb);
      CK(cudaMemsetAsync(c.x32, 0, sizeof(float) * n * nb, s));
      launch_apply_fine<double>(c, c.E64, x, b, c.r64, s, nb);
      launch_dot<double>(c, n, c.r64, c.r64, sc + 5, nullptr, s, nb);
      launch_to_f32_scaled(n, c.r64, sc + 5, c.r32, s, nb);
      if (int rc = readback(c, nb)) return rc;
      double f[kMaxBatch], rho[kMaxBatch];
      bool restart = false;
      for (int j = 0; j < nb; ++j) {
        const double rn_new = std::sqrt(c.scal_h[j * kColScal + 5]);
        f[j] = 1.0;
        rho[j] = c.scal_h[j * kColScal + 0];
        if (!live[j]) {
          rn[j] = rn_new;
          continue;
        }
        its_total[j] += its[j];
        ++outer[j];
        if (!std::isfinite(rn_new)) {
          status[j] = TPO_E_BREAKDOWN;
          c.err = "non-finite residual in the mixed-precision solve";
        } else if (st[j] == TPO_E_BREAKDOWN) {
          // the FP32 recurrence broke down: fatal unless it still made
          // progress, in which case the next pass restarts from p = z
          if (!(rn_new < rn[j])) status[j] = TPO_E_BREAKDOWN;
          restart = true;
        } else if (rn_new > target[j]) {
          f[j] = rn[j] / rn_new;
          // p and rho in the units of the new residual are f p and f^2 rho.
          // p is only read by the next p = z + (rho_new / rho) p, so f p
          // comes from storing f rho instead: (rho_new / (f rho)) p =
          // (rho_new / (f^2 rho)) (f p)
          rho[j] *= f[j];
          if (rn_new > 2.0 * predicted[j]) restart = true;
        }
        rn[j] = rn_new;
        c.scal_h[j * kColScal + 3] = rn_new > 0.0 ? 1.0 : 0.0;
      }
      resume = !restart;
      if (resume)
        if (int rc = upload_slot(c, 0, rho, nb)) return rc;
    }
    for (int j = 0; j < nb; ++j)
      if (status[j] != TPO_E_BREAKDOWN) status[j] = rn[j] <= target[j] ? TPO_OK : TPO_NOT_CONVERGED;
  }
  CK(cudaGetLastError());
  const double ms = now_ms() - t0;
  int worst = TPO_OK;
  tpo_solve_info acc{};
  for (int j = 0; j < nb; ++j) {
    if (status[j] < 0 ? status[j] < worst : (worst == TPO_OK && status[j] != TPO_OK))
      worst = status[j];
    const double rel = bn[j] > 0 ? rn[j] / bn[j] : 0.0;
    acc.iterations += its_total[j];
    acc.outer += outer[j];
    acc.relres = std::max(acc.relres, rel);
    if (col) {
      col[j].status = status[j];
      col[j].iterations = its_total[j];
      col[j].outer = outer[j];
      col[j].relres = rel;
      col[j].solve_ms = ms;
      col[j].setup_ms = c.setup_ms;
    }
  }
  if (info) {
    acc.status = worst;
    acc.solve_ms = ms;
    acc.setup_ms = c.setup_ms;
    *info = acc;
  }
  if (worst == TPO_NOT_CONVERGED && c.err.empty())
    c.err = "solver reached its iteration limit";
  return worst;
}

}  // namespace tpo
