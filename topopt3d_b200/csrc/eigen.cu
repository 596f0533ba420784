// Linear buckling eigenproblem: the nev largest lambda of
//   Ks phi = lambda K phi
// (Stability::Function, Buckling.cpp:63-75: target LR of (Ks, K), with the
// KUF preconditioner, Buckling.cpp:63-64).  The reference runs its own
// preconditioned eigensolver (LOPGMRES over PRINVIT, single-vector
// expansion); here the same family -- a locally optimal preconditioned
// method -- runs as BLOCK LOBPCG so every operator application is a column
// block: Ks (kernels_ks.cu) and K (the matrix-free apply) on m columns, and
// the GMG V-cycle (the solve's own preconditioner) in blocks of <= 8.
//
// Per iteration, with X the m current Ritz vectors (AX = Ks X, BX = K X):
//   R = AX - BX diag(theta);  W = mask(T R)  (T = one V-cycle)
//   Rayleigh-Ritz of (Ks, K) on span[X W P]: every Gram block in one pass
//   over the basis and its images (kernels_eig.cu), the
//   small generalized problem solved on the host by SVQB (eigen-
//   decomposition of the diagonally scaled K-Gram, directions below a
//   relative 1e-13 dropped) and Jacobi;
//   X <- [X W P] C,  P <- [0 W P] C  (images AX, BX, AP, BP updated by the
//   same coefficients, all six in one pass; recomputed from scratch every
//   20 iterations).
// Fixed degrees of freedom are masked out of every block (their rows and
// columns are zero in Ks and identity in K, i.e. lambda = 0 there).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <vector>

#include "solver.h"

namespace tpo {

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

__device__ __forceinline__ double seeded_value(uint64_t i) {
  uint64_t z = i + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// X[:, j] = seeded values on the free dofs, 0 on the fixed ones
__global__ void k_eig_start(int64_t n, int m, const uint8_t *__restrict__ fix,
                            uint64_t seed, double *X) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * m;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % n;
    const bool fixed = (fix[i / 3] >> (i % 3)) & 1u;
    X[t] = fixed ? 0.0 : seeded_value(seed * 0x100000001B3ull + (uint64_t)t);
  }
}

// AV = diag(d) V on m columns (the lumped mass of the frequency problem)
__global__ void k_diag_apply(int64_t n, int m, const double *__restrict__ d,
                             const double *__restrict__ V, double *__restrict__ AV) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * m;
       t += (int64_t)gridDim.x * blockDim.x)
    AV[t] = d[t % n] * V[t];
}

// zero the fixed dofs of m columns
__global__ void k_mask(int64_t n, int m, const uint8_t *__restrict__ fix,
                       double *X) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * m;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t % n;
    if ((fix[i / 3] >> (i % 3)) & 1u) X[t] = 0.0;
  }
}

// ---- small dense symmetric eigenproblems on the host ----------------------

// cyclic Jacobi: A (n x n, column-major, symmetric) -> eigenvalues w
// (descending) and eigenvectors V (columns)
void jacobi_eig(int n, std::vector<double> A, std::vector<double> &w,
                std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> double & { return A[(size_t)j * n + i]; };
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        tot += a(i, j) * a(i, j);
        if (i != j) off += a(i, j) * a(i, j);
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        const double app = a(p, p), aqq = a(q, q);
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0 ? 1.0 : -1.0) /
                         (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = t * cs;
        for (int k = 0; k < n; ++k) {   // A <- A J
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = cs * akp - sn * akq;
          a(k, q) = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {   // A <- J^T A
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = cs * apk - sn * aqk;
          a(q, k) = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {   // V <- V J
          const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
          V[(size_t)p * n + k] = cs * vkp - sn * vkq;
          V[(size_t)q * n + k] = sn * vkp + cs * vkq;
        }
      }
  }
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return a(x, x) > a(y, y); });
  std::vector<double> Vs((size_t)n * n);
  w.resize(n);
  for (int j = 0; j < n; ++j) {
    w[j] = a(idx[j], idx[j]);
    for (int i = 0; i < n; ++i) Vs[(size_t)j * n + i] = V[(size_t)idx[j] * n + i];
  }
  V.swap(Vs);
}

// Rayleigh-Ritz of (H, G) (k x k, column-major): C (k x m) and the m
// largest Ritz values.  Returns the rank kept, or < m on failure.
int rayleigh_ritz(int k, int m, const std::vector<double> &H,
                  const std::vector<double> &G, std::vector<double> &C,
                  std::vector<double> &theta) {
  std::vector<double> d(k);
  for (int i = 0; i < k; ++i) {
    const double g = G[(size_t)i * k + i];
    d[i] = g > 0 ? 1.0 / std::sqrt(g) : 0.0;
  }
  std::vector<double> Gs((size_t)k * k);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) Gs[(size_t)j * k + i] = d[i] * G[(size_t)j * k + i] * d[j];
  std::vector<double> gw, Q;
  jacobi_eig(k, Gs, gw, Q);
  const double gmax = gw.empty() ? 0.0 : gw[0];
  int r = 0;
  while (r < k && gw[r] > 1e-13 * gmax) ++r;
  if (r < m) return r;
  // Z = diag(d) Q_r diag(gw^-1/2)  (k x r)
  std::vector<double> Z((size_t)k * r);
  for (int j = 0; j < r; ++j) {
    const double s = 1.0 / std::sqrt(gw[j]);
    for (int i = 0; i < k; ++i) Z[(size_t)j * k + i] = d[i] * Q[(size_t)j * k + i] * s;
  }
  // Hr = Z^T H Z
  std::vector<double> HZ((size_t)k * r), Hr((size_t)r * r);
  for (int j = 0; j < r; ++j)
    for (int i = 0; i < k; ++i) {
      double s = 0;
      for (int l = 0; l < k; ++l) s += H[(size_t)l * k + i] * Z[(size_t)j * k + l];
      HZ[(size_t)j * k + i] = s;
    }
  for (int j = 0; j < r; ++j)
    for (int i = 0; i < r; ++i) {
      double s = 0;
      for (int l = 0; l < k; ++l) s += Z[(size_t)i * k + l] * HZ[(size_t)j * k + l];
      Hr[(size_t)j * r + i] = s;
    }
  for (int j = 0; j < r; ++j)      // symmetrise
    for (int i = 0; i < j; ++i) {
      const double v = 0.5 * (Hr[(size_t)j * r + i] + Hr[(size_t)i * r + j]);
      Hr[(size_t)j * r + i] = Hr[(size_t)i * r + j] = v;
    }
  std::vector<double> hw, Y;
  jacobi_eig(r, Hr, hw, Y);
  C.assign((size_t)k * m, 0.0);
  theta.assign(m, 0.0);
  for (int j = 0; j < m; ++j) {
    theta[j] = hw[j];
    for (int i = 0; i < k; ++i) {
      double s = 0;
      for (int l = 0; l < r; ++l) s += Z[(size_t)l * k + i] * Y[(size_t)j * r + l];
      C[(size_t)j * k + i] = s;
    }
  }
  return r;
}

#define CK(call)                                                       \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      c.err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return TPO_E_CUDA;                                               \
    }                                                                  \
  } while (0)

struct Blocks {
  double *X, *AX, *BX, *W, *AW, *BW, *P, *AP, *BP;
  double *Xn, *AXn, *BXn, *Pn, *APn, *BPn, *R;
};

}  // namespace

// W = T R on m columns (T = one V-cycle in the requested precision), masked
static int precondition(Ctx &c, const tpo_solve_opts &so, int precision,
                        double *R, double *W, int m) {
  const int64_t n = 3 * c.nn;
  cudaStream_t s = c.stream;
  for (int j0 = 0; j0 < m;) {
    const int nb = (m - j0) >= 8 ? 8 : (m - j0) >= 4 ? 4 : (m - j0) >= 2 ? 2 : 1;
    if (int rc = vcycle_cols(c, so, precision, R + j0 * n, W + j0 * n, nb)) return rc;
    j0 += nb;
  }
  count_launch();
  k_mask<<<grid_for(n * m, 256), 256, 0, s>>>(n, m, c.fix, W);
  return TPO_OK;
}

int buckling(Ctx &c, const tpo_eig_opts &o, double *lambda, double *phi,
             int phi_mem, tpo_eig_info *info, const double *adiag) {
  const double t0 = now_ms();
  const int64_t n = 3 * c.nn;
  const int m = o.block, nev = o.nev;
  cudaStream_t s = c.stream;
  // workspace: 16 blocks of n x m and the small Gram/coefficient matrices
  const size_t blk = (size_t)n * m;
  const size_t need = 16 * blk + 2 * (size_t)(3 * m) * (3 * m) + (size_t)(3 * m) * m + 2 * m +
                      eig_gram_scratch(3 * m);
  if (c.eig_n < need) {
    if (c.eig_buf) cudaFree(c.eig_buf);
    c.eig_buf = nullptr;
    c.eig_n = 0;
    CK(cudaMalloc(&c.eig_buf, sizeof(double) * need));
    c.eig_n = need;
  }
  double *base = c.eig_buf;
  Blocks b;
  double **slots[16] = {&b.X, &b.AX, &b.BX, &b.W, &b.AW, &b.BW, &b.P, &b.AP,
                        &b.BP, &b.Xn, &b.AXn, &b.BXn, &b.Pn, &b.APn, &b.BPn, &b.R};
  for (int i = 0; i < 16; ++i) *slots[i] = base + i * blk;
  const int K3 = 3 * m;
  double *dH = base + 16 * blk, *dG = dH + K3 * K3, *dC = dG + K3 * K3,
         *dnrm = dC + K3 * m, *dpart = dnrm + 2 * m;
  if (int rc = ensure_columns(c, kMaxBatch)) return rc;
  tpo_solve_opts so = c.setup_opts;

  auto applyAB = [&](const double *V, double *AV, double *BV) {
    if (adiag) {
      count_launch();
      k_diag_apply<<<grid_for(n * m, 256), 256, 0, s>>>(n, m, adiag, V, AV);
    } else {
      launch_ks_apply(c, V, AV, m);
    }
    for (int j0 = 0; j0 < m;) {
      const int nb = std::min(m - j0, kMaxBatch);
      launch_apply_fine<double>(c, c.E64, V + j0 * n, nullptr, BV + j0 * n, s, nb);
      j0 += nb;
    }
  };
  // Gram blocks of the basis [X W P] (first nblk of them): out (k x k)
  std::vector<double> Hh, Gh;
  auto gram = [&](int nblk) -> int {
    const EigCols cols{{b.X, b.W, b.P}, {b.AX, b.AW, b.AP}, {b.BX, b.BW, b.BP}};
    const int k = nblk * m;
    launch_eig_gram(n, m, nblk, cols, dpart, dH, dG, s);
    Hh.assign((size_t)k * k, 0.0);
    Gh.assign((size_t)k * k, 0.0);
    CK(cudaMemcpyAsync(Hh.data(), dH, sizeof(double) * k * k, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Gh.data(), dG, sizeof(double) * k * k, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int j = 0; j < k; ++j)   // symmetrise
      for (int i = 0; i < j; ++i) {
        const double hv = 0.5 * (Hh[(size_t)j * k + i] + Hh[(size_t)i * k + j]);
        const double gv = 0.5 * (Gh[(size_t)j * k + i] + Gh[(size_t)i * k + j]);
        Hh[(size_t)j * k + i] = Hh[(size_t)i * k + j] = hv;
        Gh[(size_t)j * k + i] = Gh[(size_t)i * k + j] = gv;
      }
    return TPO_OK;
  };

  // ---- start block and its Rayleigh-Ritz
  count_launch();
  k_eig_start<<<grid_for(n * m, 256), 256, 0, s>>>(n, m, c.fix, o.seed, b.X);
  applyAB(b.X, b.AX, b.BX);
  CK(cudaGetLastError());
  std::vector<double> C, theta;
  if (int rc = gram(1)) return rc;
  if (rayleigh_ritz(m, m, Hh, Gh, C, theta) < m) {
    c.err = "eigensolver start block is rank deficient";
    return TPO_E_BREAKDOWN;
  }
  CK(cudaMemcpyAsync(dC, C.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice, s));
  {
    const EigCols cols{{b.X, nullptr, nullptr}, {b.AX, nullptr, nullptr},
                       {b.BX, nullptr, nullptr}};
    const EigOut out{{b.Xn, b.AXn, b.BXn}, {nullptr, nullptr, nullptr}};
    launch_eig_combine(n, m, 1, cols, dC, out, false, s);
    std::swap(b.X, b.Xn);
    std::swap(b.AX, b.AXn);
    std::swap(b.BX, b.BXn);
  }

  int it = 0, nconv = 0, status = TPO_NOT_CONVERGED;
  bool haveP = false;
  double max_res = 0.0;
  std::vector<double> nrm(2 * m);
  for (;;) {
    // residuals and their relative norms
    EigTheta th{};
    for (int j = 0; j < m; ++j) th.v[j] = theta[j];
    launch_eig_resid_norms(n, m, b.AX, b.BX, th, b.R, dpart, dnrm, s);
    CK(cudaMemcpyAsync(nrm.data(), dnrm, sizeof(double) * 2 * m, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    nconv = 0;
    max_res = 0.0;
    for (int j = 0; j < nev; ++j) {
      const double rel = nrm[j] / std::max(std::fabs(theta[j]) * nrm[m + j], 1e-300);
      max_res = std::max(max_res, rel);
      if (rel <= o.tol && nconv == j) ++nconv;
    }
    if (nconv >= nev) {
      status = TPO_OK;
      break;
    }
    if (it >= o.maxit) break;
    ++it;
    // W = T R and its images
    if (int rc = precondition(c, so, o.precond, b.R, b.W, m)) return rc;
    applyAB(b.W, b.AW, b.BW);
    CK(cudaGetLastError());
    // Rayleigh-Ritz on [X W P] (without P if that basis is degenerate)
    int nblk = haveP ? 3 : 2;
    if (int rc = gram(nblk)) return rc;
    int r = rayleigh_ritz(nblk * m, m, Hh, Gh, C, theta);
    if (r < m && nblk == 3) {
      nblk = 2;
      if (int rc = gram(nblk)) return rc;
      r = rayleigh_ritz(nblk * m, m, Hh, Gh, C, theta);
    }
    if (r < m) {
      status = TPO_E_BREAKDOWN;
      c.err = "eigensolver basis lost rank";
      break;
    }
    const int k = nblk * m;
    CK(cudaMemcpyAsync(dC, C.data(), sizeof(double) * k * m, cudaMemcpyHostToDevice, s));
    {
      const EigCols cols{{b.X, b.W, b.P}, {b.AX, b.AW, b.AP}, {b.BX, b.BW, b.BP}};
      const EigOut out{{b.Xn, b.AXn, b.BXn}, {b.Pn, b.APn, b.BPn}};
      launch_eig_combine(n, m, nblk, cols, dC, out, true, s);
    }
    std::swap(b.X, b.Xn);
    std::swap(b.AX, b.AXn);
    std::swap(b.BX, b.BXn);
    std::swap(b.P, b.Pn);
    std::swap(b.AP, b.APn);
    std::swap(b.BP, b.BPn);
    haveP = true;
    if (it % 20 == 0) {   // refresh the images against drift
      applyAB(b.X, b.AX, b.BX);
      applyAB(b.P, b.AP, b.BP);
    }
  }
  CK(cudaGetLastError());
  for (int j = 0; j < nev; ++j) lambda[j] = theta[j];
  if (phi)
    CK(cudaMemcpyAsync(phi, b.X, sizeof(double) * n * nev,
                       phi_mem == TPO_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                 : cudaMemcpyDeviceToHost,
                       s));
  CK(cudaStreamSynchronize(s));
  if (info) {
    info->status = status;
    info->iterations = it;
    info->nconv = nconv;
    info->max_resid = max_res;
    info->solve_ms = now_ms() - t0;
  }
  if (status == TPO_NOT_CONVERGED && c.err.empty())
    c.err = "eigensolver reached its iteration limit";
  return status;
}

// The gradient of the aggregated buckling value (Stability::Function,
// Buckling.cpp:87-88 and 113-272) and its filter chain rule (P^T,
// Material_Interpolation.cpp:150-187 without a max-length filter), for nev
// K-normalised eigenpairs (lam on the host, phi nev device columns of 3 nn).
// Scratch: rhs and v (nev columns each), W (24 x nElem).  g receives the
// gradient with respect to the filtered density, dvdx the one with respect
// to the design; info aggregates the adjoint solves.
int buckling_sensitivity(Ctx &c, int nev, const double *lam, const double *phi, double p,
                         const tpo_solve_opts &o, double *rhs, double *v, double *W,
                         double *g, double *dvdx, double *value, tpo_solve_info *info) {
  cudaStream_t s = c.stream;
  const int64_t n = 3 * c.nn;
  double sum = 0.0;
  for (int k = 0; k < nev; ++k) sum += std::pow(lam[k], p);
  *value = std::pow(sum, 1.0 / p);
  // adjoint right-hand sides (:155-190)
  for (int k = 0; k < nev; ++k) launch_bk_adj_rhs(c, phi + k * n, W, rhs + k * n, s);
  CK(cudaGetLastError());
  // K v_k = rhs_k (:193-225), in blocks of right-hand sides
  CK(cudaMemsetAsync(v, 0, sizeof(double) * n * nev, s));
  tpo_solve_info acc{};
  int worst = TPO_OK;
  for (int j0 = 0; j0 < nev;) {
    int nb = 1;
    while (2 * nb <= nev - j0 && 2 * nb <= kMaxBatch) nb *= 2;
    if (int rc = ensure_columns(c, nb)) return rc;
    tpo_solve_info one{};
    const int rc = solve(c, o, rhs + j0 * n, v + j0 * n, &one, nb);
    if (rc < 0 && rc != TPO_E_BREAKDOWN) return rc;
    if (rc < 0 ? rc < worst : (worst == TPO_OK && rc != TPO_OK)) worst = rc;
    acc.iterations += one.iterations;
    acc.outer += one.outer;
    acc.relres = std::max(acc.relres, one.relres);
    acc.solve_ms += one.solve_ms;
    j0 += nb;
  }
  // element gradient (:229-265) and the filter chain rule (:267-274)
  BkCoef coef{};
  for (int k = 0; k < nev; ++k) {
    coef.a[k] = std::pow(lam[k], p - 1.0);
    coef.lam[k] = lam[k];
  }
  coef.scale = std::pow(*value, 1.0 - p);
  launch_bk_gradient(c, phi, v, n, nev, coef, g, s);
  launch_filter(c, g, dvdx, true, s);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  acc.status = worst;
  acc.setup_ms = c.setup_ms;
  if (info) *info = acc;
  return worst;
}

// Frequency::Function (Dynamic.cpp:18-171) with DiagMassFnc (:181-235):
// the lumped mass diagonal (into mdiag), the largest eigenvalues of
// M phi = lambda K phi until more than nvals have converged and the last is
// separated from the one before it by a relative 1e-5 (UNIQUE_LAST_NEV,
// EigenPeetz.cpp:310-312), value = (sum over all of them lambda^p)^(1/p)
// and, when dvdx is given, its gradient over the first nvals - 1 pairs, as
// the reference sums them (:127-160), then the filter chain rule.  phi:
// device scratch of 32 columns of 3 nn.
int frequency(Ctx &c, int nvals, double density, const double *mlump,
              const tpo_eig_opts &o_in, double p, double *lambda, int *nconv,
              double *mdiag, double *phi, double *g, double *dvdx, double *value,
              tpo_eig_info *info) {
  cudaStream_t s = c.stream;
  const double mscale = c.prm.dx[0] * c.prm.dx[1] * c.prm.dx[2] * density / 8.0 / 3.0;
  launch_lumped_mass(c, mscale, mlump, mdiag, s);
  CK(cudaGetLastError());
  tpo_eig_opts o = o_in;
  int nev = nvals + 1, rc = TPO_OK;
  tpo_eig_info one{};
  for (;;) {
    o.nev = nev;
    o.block = std::min(kMaxEigPairs, std::max(o_in.block, nev + 2));
    rc = buckling(c, o, lambda, phi, TPO_MEM_DEVICE, &one, mdiag);
    if (rc < 0 && rc != TPO_E_BREAKDOWN) return rc;
    const bool separated = std::fabs(1.0 - lambda[nev - 2] / lambda[nev - 1]) > 1e-5;
    if (separated || rc != TPO_OK || nev + 2 > kMaxEigPairs) break;
    ++nev;
  }
  *nconv = nev;
  double sum = 0.0;
  for (int k = 0; k < nev; ++k) sum += std::pow(lambda[k], p);
  *value = std::pow(sum, 1.0 / p);
  if (dvdx) {
    BkCoef coef{};
    const int nterms = std::max(0, nvals - 1);
    for (int k = 0; k < nterms; ++k) {
      coef.a[k] = std::pow(lambda[k], p - 1.0);
      coef.lam[k] = lambda[k];
    }
    coef.scale = std::pow(*value, 1.0 - p);
    launch_freq_gradient(c, phi, 3 * c.nn, nterms, mscale, coef, g, s);
    launch_filter(c, g, dvdx, true, s);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s));
  if (info) *info = one;
  return rc;
}

}  // namespace tpo
