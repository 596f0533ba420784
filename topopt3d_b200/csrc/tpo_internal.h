// Internal declarations of the B200 TopOpt3D FE library: the context, the
// per-level state and the kernel launchers.  Nothing here is part of the
// C ABI (include/topopt_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/topopt_b200.h"

namespace tpo {

// ---------------------------------------------------------------------------
// The element stiffness in the 2x2x2 Hadamard (modal) basis.
//
// Nodal values of one element in lexicographic corner order l = bx+2by+4bz
// are transformed per component by the unnormalised butterfly
//   uh[q] = sum_l s(l,q) u[l],  s(l,q) = prod_{d in q} (bit d of l ? +1 : -1)
// (q = mode bitmask over x,y,z).  With Kh = T K0 T^T / 64 the element matvec
// is y = T^T Kh T u.  Kh couples only these blocks of (mode q, component c)
// pairs (true for any box element and isotropic D); the 45 constants are
// stored block by block, row-major:
//   0: 3x3 {(1,0),(2,1),(4,2)}   normal strains
//   1: 2x2 {(1,1),(2,0)}         shear xy
//   2: 2x2 {(1,2),(4,0)}         shear xz
//   3: 2x2 {(2,2),(4,1)}         shear yz
//   4: 2x2 {(3,0),(6,2)}         bilinear modes
//   5: 2x2 {(3,1),(5,2)}
//   6: 2x2 {(6,1),(5,0)}
//   7: 3x3 {(3,2),(6,0),(5,1)}
//   8: 3 x 1x1 {(7,0)},{(7,1)},{(7,2)}
// ---------------------------------------------------------------------------
constexpr int kNumKh = 45;

template <typename T>
struct Kh {
  T v[kNumKh];
};

// diagonal of K0 in lexicographic corner order (24 values) for the Jacobi
// diagonal of the fine operator
template <typename T>
struct K0Diag {
  T v[24];
};

// stress-stiffness constants: shape-function gradients g[q][a][l] =
// dN_l/dx_a at Gauss point q (corners l in lexicographic order), the
// isotropic D entries (t1 = (1-nu) c, t3 = nu c, t2 = shear modulus) and
// detJ (FEAnalysis.cpp:869-1050, RecMesh.cpp:453-462)
struct KsConst {
  double g[8][3][8];
  double t1, t2, t3, detJ;
};

// density filter template: offsets and raw weights 1 - d/R (Filter.cpp:43-52)
constexpr int kMaxFilterTaps = 512;

struct FilterTaps {
  int n;
  int8_t off[kMaxFilterTaps][3];
  double w[kMaxFilterTaps];
};

struct Level {
  int dims[3] = {0, 0, 0};
  int64_t nn = 0;
  // Galerkin operator as a 27-point 3x3-block stencil, SoA:
  // S[(nb*9 + 3r + s) * nn + node], nb = (dk+1)*9 + (dj+1)*3 + (di+1)
  double *S64 = nullptr;
  float *S32 = nullptr;
  // node-major copies A[n*243 + (3r + s)*27 + nb] for the persistent kernel
  double *A64 = nullptr;
  float *A32 = nullptr;
  // symmetric half (centre + 13 forward blocks) for the levels between the
  // finest and the persistent kernel: H[(h*9 + 3r + s) * nn + n]
  double *H64 = nullptr;
  float *H32 = nullptr;
  double *dinv64 = nullptr;
  float *dinv32 = nullptr;
  double lam = 0.0;
  // V-cycle work vectors (3*nn per column, Ctx::nb_cap columns); e = second
  // Chebyshev direction and w = pre-smoothed iterate of the levels run by
  // the persistent kernel
  double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr, *d64 = nullptr,
         *a64 = nullptr, *e64 = nullptr, *w64 = nullptr;
  float *b32 = nullptr, *x32 = nullptr, *r32 = nullptr, *d32 = nullptr,
        *a32 = nullptr, *e32 = nullptr, *w32 = nullptr;
};

// side streams of the set-up (per-level power iterations)
constexpr int kAuxStreams = 4;
// GMG levels of one context
constexpr int kMaxLevels = 16;

struct Ctx {
  tpo_mesh_params prm{};
  int nel[3] = {0, 0, 0};
  int64_t ne = 0, nn = 0;
  int L = 0;
  int ps = 0;   // first level run by the persistent coarse-cycle kernel
  int nb_cap = 1;   // columns the level and solver work vectors hold
  int rhs_block_tuned = 0;   // autotuned right-hand-side block (0: not yet)
  cudaError_t coarse_err = cudaSuccess;   // last cooperative launch status
  std::vector<Level> lev;
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  // set-up side streams (the Chebyshev bound estimates of the levels
  // overlap the Galerkin chain and one another; level l runs on side
  // stream l % kAuxStreams) and their events
  cudaStream_t aux_stream[kAuxStreams] = {};
  cudaEvent_t lev_ev[kMaxLevels] = {};
  cudaEvent_t aux_ev[kAuxStreams] = {};
  // the set-up's critical chain (Galerkin products, coarse factorisation
  // and inverse) runs on a highest-priority stream forked from `stream`, so
  // the side streams' power iterations fill in around it
  cudaStream_t setup_stream = nullptr;
  cudaEvent_t setup_ev[2] = {};
  std::string err;

  // element constants
  double K0[576];
  Kh<double> kh64{};
  Kh<float> kh32{};
  K0Diag<double> kd64{};

  // host-side boundary conditions
  std::vector<uint8_t> fix_h;
  std::vector<double> F_h;
  // the Set_BC lists (Inputs.cpp:145-170) MeshOut writes: nodes in the
  // order selected, with per node 3 support flags / 3 load values
  std::vector<int64_t> supp_node, load_node;
  std::vector<uint8_t> supp_val;
  std::vector<double> load_val;
  bool initialized = false;
  bool have_material = false;
  bool assembled = false;
  tpo_solve_opts setup_opts{};
  double setup_ms = 0.0;

  // device state
  uint8_t *fix = nullptr;   // per-node fixed-component bitmask
  // identity-row mask of the fine operator: fix | non-positive diagonal
  // (kernels_apply.cu, k_identity_mask); refreshed whenever E or fix change
  uint8_t *idm = nullptr;
  double *F = nullptr, *U = nullptr;
  double *x = nullptr, *rho = nullptr, *E64 = nullptr, *dEdz = nullptr;
  double *Es64 = nullptr;   // rho^p without E_min (stress stiffness)
  double *dEsdz64 = nullptr;   // d Es / d rho (Material_Interpolation.cpp:67-70)
  float *E32 = nullptr;
  double *S0 = nullptr;     // fine-level assembled stencil (setup only)
  double *K0lex = nullptr;  // K0 in lexicographic corner order (576)
  // level-1 Galerkin blocks of interior fine elements, [i][ln][lm][9]
  // (element.cpp, build_galerkin_blocks), and the per-coarse-element
  // general-path flags
  double *GMi = nullptr;
  double GMi_h[8 * 8 * 8 * 9];
  // general-path coarse elements of the level-1 Galerkin product: slot per
  // coarse element (-1: fast path), the element of each slot, the count,
  // and the 64 blocks of 9 per slot
  int *gk_slot = nullptr, *gk_elem = nullptr;
  unsigned int *gk_count = nullptr;
  double *gk_G = nullptr;
  size_t gk_cap = 0;
  // level 1 in FP32 on the tensor cores (kernels_l1tc.cu): the form
  // requested (0 automatic, 1 always the stored stencil), whether the
  // context qualifies (even element counts, level 1 above the persistent
  // levels), the operand image of the 8 blocks G_i (hi and lo TF32 parts),
  // the correction rows of the nodes next to general-path coarse elements
  // (node of each row, rows of 243 values, capacity in rows), C u on those
  // rows as a dense level-1 vector, the CTAs holding such nodes, the row
  // count and the overflow flag
  int l1_form = 0;
  bool l1tc_ok = false;
  bool l1_bimg_ready = false;
  float *l1_B = nullptr;
  int *l1_rows = nullptr;
  float *l1_C = nullptr;
  size_t l1_cap = 0;
  float *l1_cval = nullptr;
  uint8_t *l1_cflag = nullptr;
  unsigned int *l1_count = nullptr;
  int l1_nrows = 0;   // host copy of the row count (read at the end of set-up)
  int *l1_fault = nullptr;
  // scratch of the dimension-by-dimension Galerkin products (levels >= 1)
  double *gd_tmp = nullptr;
  double *Ainv = nullptr;   // dense inverse of the coarsest operator
  int64_t nc = 0;

  // filter
  FilterTaps taps{};
  FilterTaps *taps_d = nullptr;
  double *finv = nullptr;   // 1 / row sum per element

  // solver work (fine level, FP64 and FP32; r, z, p, q and x32 hold
  // nb_cap columns, w64 one)
  double *r64 = nullptr, *z64 = nullptr, *p64 = nullptr, *q64 = nullptr,
         *w64 = nullptr;
  float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *q32 = nullptr,
        *x32 = nullptr;
  double *scal = nullptr;   // device scalars
  double *scal_h = nullptr; // pinned host mirror
  double *part = nullptr;   // reduction partials
  unsigned int *ticket = nullptr;
  unsigned int *gbar = nullptr;  // grid-barrier counter of the persistent
                                 // coarse-grid kernel (kernels_coarse.cu)
  double *tmpe = nullptr, *tmpe2 = nullptr;   // element-sized scratch
  double *io_a = nullptr, *io_b = nullptr;    // staging for host buffers
  double *io_ba = nullptr, *io_bb = nullptr;  // the same for column blocks
  double *oc_ws = nullptr;                    // OC update workspace (6 nElem)
  size_t io_bytes = 0;

  // coarsest inverse
  double *Adense = nullptr;     // workspace of the coarsest inversion
  int *dev_info = nullptr;

  // stress stiffness: 27-point scalar stencil S[d * nn + n] and the
  // per-element scratch (36 x ne) it is gathered from
  KsConst ksc{};
  double *ks_S = nullptr, *ks_H = nullptr;
  bool ks_ready = false;
  // eigensolver block workspace
  double *eig_buf = nullptr;
  size_t eig_n = 0;
  double *bk_buf = nullptr;   // buckling-sensitivity workspace
  size_t bk_n = 0;
  double *fq_buf = nullptr;   // frequency workspace
  size_t fq_n = 0;
  double *mma_buf = nullptr;  // MMA workspace (device) and partials mirror
  size_t mma_n = 0;
  int mma_steps = 0;   // dual Newton steps of the last tpo_mma_update
  double *mma_h = nullptr;

  // CUDA graphs of the CG iteration loop (a device-side while loop around
  // the iteration body), keyed on (x, columns)
  cudaGraphExec_t graph64 = nullptr, graph32 = nullptr;
  const void *graph64_x = nullptr, *graph32_x = nullptr;
  int graph64_nb = 0, graph32_nb = 0;
  long long graph64_nodes = 0, graph32_nodes = 0;
};

// --------------------------- kernel launchers ------------------------------

// process-wide count of kernel launches (tpo_kernel_launches)
extern std::atomic<long long> g_launches;
inline void count_launch(long long n = 1) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
}

constexpr int kRedBlocks = 592;   // 4 x 148 SMs: fixed grid for reductions

// Right-hand sides are processed in blocks of up to kMaxBatch columns:
// column j of a block vector lives at offset j * (3 * nn_level).  Each
// column has kColScal device scalars at scal + j * kColScal:
//   0 rho = r.z, 1 rho of the previous iteration, 2 p.q, 3 r.r (current
//   PCG), 4 b.b, 5 r.r of the FP64 residual, 6 frozen flag (non-zero: the
//   column has converged and its CG updates are skipped), 7 (column 0
//   only) fault flag of the persistent coarse-grid kernel: non-zero when a
//   grid-barrier wait ran out (read with the other scalars by readback).
// Scalars of the design-side calls follow the column block at kScalMisc;
// the power iteration of level l leaves its last two squared norms in
// SC_POWER + l and SC_POWER_PREV + l.
constexpr int kMaxBatch = 8;
constexpr int kColScal = 8;
constexpr int kScalMisc = kMaxBatch * kColScal;   // 64
enum { SC_COMPLIANCE = kScalMisc, SC_VOLUME, SC_OC_DG, SC_OC_CHANGE, SC_POWER };
constexpr int SC_POWER_PREV = SC_POWER + kMaxLevels;
// blocks that passed every barrier of tpo_barrier_selftest
constexpr int SC_SELFTEST = SC_POWER_PREV + kMaxLevels;
// the device-resident PCG loop (solver.cu): per column the target r.r,
// the iteration count and the status (0 running, 1 converged, -1
// breakdown); the iterations done and the iteration limit
constexpr int SC_LOOP_TARGET = SC_SELFTEST + 1;
constexpr int SC_LOOP_ITS = SC_LOOP_TARGET + kMaxBatch;
constexpr int SC_LOOP_STATUS = SC_LOOP_ITS + kMaxBatch;
constexpr int SC_LOOP_K = SC_LOOP_STATUS + kMaxBatch;
constexpr int SC_LOOP_MAXIT = SC_LOOP_K + 1;
constexpr int kScalCount = SC_LOOP_MAXIT + 1;
constexpr int kSlotFault = 7;

// fixed reduction grid (blocks per column) for a block of nb columns
inline int red_grid(int nb) {
  return nb <= 1 ? kRedBlocks : (kRedBlocks / nb < 148 ? 148 : kRedBlocks / nb);
}
// reduction scratch: red_grid(nb) * nb <= kAuxPart partials on the main
// stream; set-up side stream i uses part + kAuxPart + i * kRedBlocks and
// ticket + kMaxBatch + i
constexpr int kAuxPart = 2048;
constexpr int kPartCount = kAuxPart + kAuxStreams * kRedBlocks;

// fine matrix-free operator: y = M K M u + (1-M) u, or y = b - (that)
template <typename T>
void launch_apply_fine(const Ctx &c, const T *E, const T *u, const T *b, T *y,
                       cudaStream_t s, int nb = 1);

// fused fine-level variants: how the input is formed and what the epilogue
// writes (kernels_apply_staged.cu, finish_dof)
enum { IN_U = 0, IN_CHEB = 1 };
enum { OUT_Y = 0, OUT_RESID = 1, OUT_CHEB2 = 2, OUT_POST0 = 3, OUT_POST1 = 4 };

// u, b, y, y2 are per column (stride ld); dinv is shared by the columns
template <typename T>
struct ApplyArgs {
  const T *u, *b, *dinv;
  T *y, *y2;
  T invtheta, theta, c1, c2;
  int64_t ld;    // column stride (3 * nn), set by the launcher
  int nchunk;    // z chunks per column, set by the launcher
};

template <typename T>
void launch_apply_fused(const Ctx &c, const T *E, int in, int out,
                        const ApplyArgs<T> &args, cudaStream_t s, int nb = 1);
void launch_fine_diag(const Ctx &c, double *dinv64, float *dinv32,
                      cudaStream_t s);
void launch_fine_stencil(const Ctx &c, double *S, cudaStream_t s);
void launch_identity_mask(const Ctx &c, cudaStream_t s);

// stencil levels
template <typename T>
void launch_apply_stencil(const Level &v, const T *S, const T *u, const T *b,
                          T *y, cudaStream_t s);
template <typename T>
void launch_apply_stencil_sym(const Level &v, const T *H, const T *u,
                              const T *b, T *y, cudaStream_t s, int nb = 1);
// the symmetric-half stencil of one column with the fused Chebyshev(2)
// input/epilogue modes of the fine level (ApplyArgs: u, b, dinv, y, y2)
template <typename T>
void launch_apply_sym_fused(const Level &v, const T *H, int in, int out,
                            const ApplyArgs<T> &a, cudaStream_t s);
void launch_stencil_to_half(int64_t nn, const double *S, double *H64,
                            float *H32, cudaStream_t s);
// level 1 on the tensor cores (kernels_l1tc.cu)
// true when the FP32 level-1 operator runs on the tensor-core kernel
inline bool l1_tensor(const Ctx &c) { return c.l1tc_ok && c.l1_form == 0; }
// per-context operand image and per-assembly correction rows; syncs the
// stream once when the correction capacity has to grow
int l1tc_prepare(Ctx &c, const double *Sc, int nslots, cudaStream_t s);
// y = A_1 u (OUT_Y), b - A_1 u (OUT_RESID) or the fused Chebyshev(2)
// forms, one column (two launches: the correction rows, then the apply,
// which starts while the first runs)
void launch_l1tc(const Ctx &c, int in, int out, const ApplyArgs<float> &a, cudaStream_t s);
// the grid of the kernel: x tiles, y tiles, node planes per CTA, z chunks
void l1tc_grid(const Level &v, int *tx, int *ty, int *zchunk, int *nz);
// the same product one dimension at a time (three launches through tmp,
// galerkin_dims_scratch doubles)
void launch_galerkin_dims(const Level &fine, const double *Sf, double *Sc,
                          double *tmp, cudaStream_t s);
size_t galerkin_dims_scratch(const Level &fine);
// level 1 = P^T A_0 P from the element moduli (no fine stencil); syncs
// the stream once (the general-path element count)
int launch_galerkin_fine(Ctx &c, double *Sc, cudaStream_t s);
void launch_stencil_diag(const Level &v, const double *S, double *dinv64,
                         float *dinv32, cudaStream_t s);
template <typename T>
void launch_restrict(const Level &fine, const Level &coarse, const T *rf,
                     T *bc, cudaStream_t s, int nb = 1);
template <typename T>
void launch_prolong_add(const Level &fine, const Level &coarse, const T *xc,
                        T *xf, cudaStream_t s, int nb = 1);
void launch_to_dense(const Level &v, const double *S, double *A,
                     cudaStream_t s);
// stencil SoA S[(nb*9 + 3r+s)*nn + n] -> node-major A[n*243 + (3r+s)*27 + nb]
// (FP64 and an FP32 copy)
void launch_soa_to_aos(int64_t nn, const double *S, double *A64, float *A32,
                       cudaStream_t s);
// A (n x n, column-major, SPD) <- A^-1 in place by blocked Gauss-Jordan
// (kernels_coarse_inv.cu); work holds coarse_inverse_work(n) doubles; *info
// becomes the global index + 1 of the first pivot that is not positive
size_t coarse_inverse_work(int64_t n);
void launch_coarse_inverse(int64_t n, double *A, double *work, int *info, cudaStream_t s);
template <typename T>
void launch_coarse_gemv(int64_t n, const double *Ainv, const T *b, T *x,
                        cudaStream_t s, int nb = 1);

// Chebyshev smoother pieces
template <typename T>
void launch_cheb_init(int64_t n, const T *dinv, const T *b, T *r, T *d, T *x,
                      double inv_theta, bool zero_guess, cudaStream_t s,
                      int nb = 1);
template <typename T>
void launch_cheb_step(int64_t n, const T *dinv, const T *Ad, T *r, T *d, T *x,
                      double c1, double c2, cudaStream_t s, int nb = 1);

// vectors and reductions (FP64 accumulation; results in device scalars).
// With nb columns, n is the length of one column and the scalars of column
// j are at (pointer) + j * kColScal.
// part/ticket: reduction scratch other than the context's (for a reduction
// that runs concurrently with others); null = the context's
template <typename T>
void launch_dot(const Ctx &c, int64_t n, const T *a, const T *b, double *out,
                double *shift_to, cudaStream_t s, int nb = 1,
                double *part = nullptr, unsigned int *ticket = nullptr);
// CG rho = r.z per column into slot 0, the previous rho into slot 1; a
// frozen column (slot 6 set) keeps both, so a resumed recurrence finds the
// rho of its last active iteration
template <typename T>
void launch_rho_dot(const Ctx &c, int64_t n, const T *r, const T *z, cudaStream_t s,
                    int nb);
template <typename T>
void launch_cg_p(int64_t n, const T *z, T *p, const double *scal, bool first,
                 cudaStream_t s, int nb = 1);
template <typename T>
void launch_cg_update(const Ctx &c, int64_t n, T *x, T *r, const T *p,
                      const T *q, const double *scal, double *rr,
                      cudaStream_t s, int nb = 1);
template <typename T>
void launch_power_start(int64_t n, T *a, cudaStream_t s);
// w *= dinv and its squared norm (FP64 sums) into *out (the previous *out
// into *shift_to), one pass; reduction scratch as launch_dot's
template <typename T>
void launch_scale_diag_dot(const Ctx &c, int64_t n, T *w, const T *dinv, double *out,
                           double *shift_to, cudaStream_t s, double *part,
                           unsigned int *ticket);
void launch_to_f32_scaled(int64_t n, const double *a, const double *scal,
                          float *b, cudaStream_t s, int nb = 1);
void launch_axpy_f32(int64_t n, double *U, const float *d, const double *scal,
                     cudaStream_t s, int nb = 1);
void launch_d2f(int64_t n, const double *a, float *b, cudaStream_t s);
void launch_f2d(int64_t n, const float *a, double *b, cudaStream_t s);
void launch_fill(int64_t n, double *a, double v, cudaStream_t s);

// design-side kernels
void launch_filter_rowsum(const Ctx &c, cudaStream_t s);
void launch_filter(const Ctx &c, const double *in, double *out, bool transpose,
                   cudaStream_t s);
// P^T applied to the constant vector `value`
void launch_filter_adj_uniform(const Ctx &c, double value, double *out,
                               cudaStream_t s);
void launch_simp(const Ctx &c, double penal, double eps, cudaStream_t s);
// stress stiffness from c.U and c.Es64 (kernels_ks.cu)
void launch_ks_assemble(const Ctx &c, cudaStream_t s);
// buckling sensitivities (kernels_ks.cu): per eigenpair k, a_k = lam_k^(p-1);
// scale = value^(1-p)
constexpr int kMaxEigPairs = 32;
struct BkCoef {
  double a[kMaxEigPairs];
  double lam[kMaxEigPairs];
  double scale;
};
// adjoint right-hand side of one eigenvector phi: rhs = sum_e Es_e
// d(phi^T ks_e phi)/du_e (W: 24 x nElem scratch), zero at fixed dofs
void launch_bk_adj_rhs(const Ctx &c, const double *phi, double *W, double *rhs,
                       cudaStream_t s);
// block eigensolver kernels (kernels_eig.cu).  A basis of nblk blocks of m
// columns (n rows, column-major): L[b] the vectors, A[b] and B[b] their
// two operator images
struct EigCols {
  const double *L[3], *A[3], *B[3];
};
struct EigOut {
  double *X[3], *P[3];   // per image group (vectors, A, B)
};
struct EigTheta {
  double v[kMaxEigPairs];
};
// doubles of partial sums launch_eig_gram and launch_eig_resid_norms need
// for a basis of k columns
size_t eig_gram_scratch(int k);
// H = L^T A and G = L^T B over all k = nblk m columns (k x k, column-major)
void launch_eig_gram(int64_t n, int m, int nblk, const EigCols &cols, double *part, double *H,
                     double *G, cudaStream_t s);
// out.X[g] = [group g blocks] C (C: k x m) and, with want_p, out.P[g] the
// same without block 0
void launch_eig_combine(int64_t n, int m, int nblk, const EigCols &cols, const double *C,
                        const EigOut &out, bool want_p, cudaStream_t s);
// R = AX - BX diag(theta), nrm[j] = ||R_j||, nrm[m + j] = ||BX_j||
void launch_eig_resid_norms(int64_t n, int m, const double *AX, const double *BX,
                            const EigTheta &th, double *R, double *part, double *nrm,
                            cudaStream_t s);
// frequency (kernels_ks.cu): the lumped mass diagonal m (3 nn) from c.rho,
// and the gradient g_e from nterms eigenvector columns (stride ld)
void launch_lumped_mass(const Ctx &c, double scale, const double *mlump, double *m,
                        cudaStream_t s);
void launch_freq_gradient(const Ctx &c, const double *phi, int64_t ld, int nterms,
                          double mscale, const BkCoef &coef, double *g, cudaStream_t s);
// g_e, the gradient before the filter chain rule, from c.U and nev columns
// of phi and the adjoint solutions v (stride ld)
void launch_bk_gradient(const Ctx &c, const double *phi, const double *v, int64_t ld,
                        int nev, const BkCoef &coef, double *g, cudaStream_t s);
// y = Ks u for nb columns (stride 3 nn), on c.stream
void launch_ks_apply(const Ctx &c, const double *u, double *y, int nb);
void launch_sensitivity(const Ctx &c, const double *U, double *dc,
                        cudaStream_t s);
void launch_oc_step(const Ctx &c, int64_t n, double *x, const double *xold,
                    const double *xmin, const double *xmax, const double *dfdx,
                    const double *dgdx, double move, double lmid, double *out,
                    cudaStream_t s);
void launch_oc_clip(int64_t n, double *dfdx, cudaStream_t s);
// MMA for m >= 2 constraints (kernels_design.cu): MMAsub, DualSolve and
// Change in one cooperative launch
constexpr int kMmaMaxM = 8;
struct MmaConst {
  double move, asyinit, asyincr, asydecr, albefa, raa0;
};
struct MmaSolveArgs {
  int64_t n;
  int m, fresh;
  MmaConst k;
  double epsimin;
  double g[kMmaMaxM];
  double *x, *x1, *x2, *low, *upp;             // in/out design state
  const double *xmin, *xmax, *dfdx, *dgdx;     // dgdx n x m column-major
  double *alfa, *beta, *p0, *q0, *P, *Q;       // n, n, n, n, n*m, n*m scratch
  double *part;       // 2 * (m + m(m+1)/2) * kRedBlocks doubles
  double *out;        // [0] Change (zeroed by the launcher), [1] Newton
                      // steps, [2] status (0 ok, 1 singular Newton system)
  unsigned int *bar;  // grid barrier counter (c.gbar)
  double *fault;      // set when a grid-barrier wait runs out
};
// false when no block of the kernel fits on an SM (nothing launched)
bool launch_mma_solve(MmaSolveArgs &a, cudaStream_t s, cudaError_t *err);
// the whole OC bisection in one cooperative launch of kRedBlocks CTAs (uses
// c.part, c.gbar and the fault slot); false when the device cannot hold
// them all at once, and the caller runs the per-trial launches instead
bool launch_oc_bisect(const Ctx &c, int64_t n, double *x, const double *xold,
                      const double *xmin, const double *xmax, const double *dfdx,
                      const double *dgdx, double move, double g, cudaStream_t s,
                      cudaError_t *err);
void launch_oc_finish(const Ctx &c, int64_t n, double *x, const double *xold,
                      const double *xmin, const double *xmax, double *out,
                      cudaStream_t s);
// the grid-barrier self-test (selftest.cu): `blocks` co-resident CTAs cross
// `phases` barriers on c.gbar, block `skip` (if in range) leaves before its
// first arrival, waits give up after max_polls polls; the count of blocks
// that passed every barrier goes to c.scal[SC_SELFTEST]
cudaError_t launch_barrier_selftest(const Ctx &c, int blocks, int phases, int skip,
                                    int max_polls, cudaStream_t s);

// host-side element constants (element.cpp)
int build_element_constants(Ctx &c);
bool build_filter_taps(const int nel[3], const double dx[3], double R,
                       FilterTaps &taps);

}  // namespace tpo
