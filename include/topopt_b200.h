/*
 * topopt_b200.h -- C ABI of the B200-native TopOpt3D finite-element path.
 *
 * One context (tpo_ctx) holds one structured hex8 problem on one GPU: the
 * mesh, boundary conditions, density filter, SIMP material, the geometric
 * multigrid hierarchy and the solution vectors, all resident in HBM.  Every
 * entry point returns an int status: 0 = success, > 0 = the solver stopped
 * without converging (iterations and residual are still reported),
 * < 0 = error (see TPO_E_*); tpo_last_error() gives the message.  No entry
 * point aborts the process.  A context is bound to the device that was
 * current at tpo_create and must not be used from two host threads at once.
 *
 * Vectors use the reference numbering: element e = i + j*nx + k*nx*ny,
 * node n = i + j*(nx+1) + k*(nx+1)*(ny+1), dof = 3*n + component.  Buffers
 * are FP64 and caller-owned; `mem` selects host (TPO_MEM_HOST) or device
 * (TPO_MEM_DEVICE) pointers.  Host buffers are copied inside the call.
 *
 * Each declaration names the darinpeetz/TopOpt3D member it replaces
 * (file:line in that tree).
 */
#ifndef TOPOPT_B200_H
#define TOPOPT_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define TPO_API __attribute__((visibility("default")))
#else
#define TPO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define TPO_OK 0
#define TPO_NOT_CONVERGED 1
#define TPO_E_ARG (-1)      /* invalid argument or call order */
#define TPO_E_CUDA (-2)     /* CUDA runtime / library error */
#define TPO_E_BREAKDOWN (-3)/* CG breakdown, non-finite residual, indefinite */
#define TPO_E_UNSUPPORTED (-4)

#define TPO_MEM_HOST 0
#define TPO_MEM_DEVICE 1

#define TPO_PREC_FP64 0     /* FP64 apply, smoother, transfers, CG */
#define TPO_PREC_MIXED 1    /* FP32 PCG+GMG with FP64 residual replacement */

#define TPO_BC_SUPPORT 0
#define TPO_BC_LOAD 1

typedef struct tpo_ctx tpo_ctx;

typedef struct {
  int32_t nel[3];     /* elements per dimension (NEL) */
  double dx[3];       /* element edge lengths (Dimensions / NEL) */
  double E0, nu;      /* Young's modulus and Poisson ratio (E0, Nu0) */
  double rmin;        /* density-filter radius, absolute (RMin) */
  int32_t mg_levels;  /* GMG levels incl. the finest (-kuf_pc_mg_levels);
                         <= 0 selects floor(log2(min nel)) as the reference */
} tpo_mesh_params;

typedef struct {
  double rtol;        /* ||F - K U|| <= rtol * ||F|| (KSP rtol 1e-8) */
  int32_t maxit;      /* CG iterations (inner iterations in mixed form) */
  int32_t precision;  /* TPO_PREC_FP64 or TPO_PREC_MIXED */
  int32_t cheb_degree;/* Chebyshev steps per smoothing (2) */
  double cheb_lo;     /* smoothing interval [lo, hi] * lambda_max(D^-1 A) */
  double cheb_hi;
  int32_t power_its;  /* power iterations for lambda_max at setup (15) */
  double inner_rtol;  /* mixed form: relative drop of the FP32 residual
                         between two FP64 residual replacements (1e-2); the
                         last pass asks for 0.7 rtol instead when that is
                         less of a drop */
  int32_t max_outer;  /* mixed form: FP64 residual replacements (10) */
  int32_t use_graph;  /* capture the V-cycle/CG iteration in a CUDA graph */
  int32_t rhs_block;  /* tpo_solve: right-hand sides solved together as one
                         block (1, 2, 4 or 8); 0 = autotuned between 4 and 8
                         once per context (default) */
} tpo_solve_opts;

typedef struct {
  int32_t status;     /* as the return code */
  int32_t iterations; /* CG iterations (FP32 iterations when mixed) */
  int32_t outer;      /* FP64 residual replacements (1 in FP64 form) */
  double relres;      /* final ||F - K U|| / ||F||, FP64 */
  double solve_ms;    /* host wall time of the solve phase */
  double setup_ms;    /* host wall time of the last FEAssemble/PCSetUp */
} tpo_solve_info;

/* fills the defaults used throughout (rtol 1e-8, maxit 500, FP64, Chebyshev
 * degree 2 on [0.1, 1.1] * lambda, 15 power iterations, inner_rtol 1e-2,
 * max_outer 10, graphs on, autotuned right-hand-side blocks) */
TPO_API void tpo_default_solve_opts(tpo_solve_opts *opts);

/* TopOpt::CreateMesh (RecMesh.cpp:426-728) on one device: structured box
 * mesh, density filter (Filter.cpp:21-150), GMG level layout
 * (Interpolation.cpp:31-169) and the element stiffness K0
 * (FEAnalysis.cpp:869-1050). */
TPO_API int tpo_create(const tpo_mesh_params *params, tpo_ctx **out);
/* TopOpt::Clear (TopOpt.cpp:59-89) */
TPO_API int tpo_destroy(tpo_ctx *ctx);
TPO_API const char *tpo_last_error(const tpo_ctx *ctx);

/* sizes: elements, nodes, levels actually built */
TPO_API int tpo_sizes(const tpo_ctx *ctx, int64_t *n_elem, int64_t *n_node,
              int32_t *n_levels);
/* GMG level l (0 = finest): nodes per dimension */
TPO_API int tpo_level_dims(const tpo_ctx *ctx, int32_t level, int32_t dims[3]);

/* TopOpt::Set_BC (Inputs.cpp:105-223) for SUPPORT and LOAD: selects every
 * node with sum_d ((x_d-c_d)/r_d)^2 <= 1 inside limits [lo0,hi0,lo1,hi1,
 * lo2,hi2]; a support fixes each component whose value is non-zero, a load
 * adds `values` to every selected node.  *n_selected receives the count. */
TPO_API int tpo_add_bc(tpo_ctx *ctx, int32_t type, const double center[3],
               const double radius[3], const double limits[6],
               const double values[3], int64_t *n_selected);
/* direct form: per-node fixed-component bitmask (bit c fixes component c)
 * and load vector F (3*nNode); either may be NULL to keep the current one */
TPO_API int tpo_set_bc(tpo_ctx *ctx, const uint8_t *fixmask, const double *F, int mem);
TPO_API int tpo_get_bc(const tpo_ctx *ctx, uint8_t *fixmask, double *F, int mem);

/* TopOpt::FEInitialize (FEAnalysis.cpp:215-424): freezes the BCs, uploads
 * the fixed mask and F, allocates the solver state (U = 0). */
TPO_API int tpo_fe_initialize(tpo_ctx *ctx);

/* TopOpt::MatIntFnc (Material_Interpolation.cpp:20-140) with vdMin <= 0:
 * rho = P x, E = eps + (1-eps) rho^p, dEdz = (1-eps) p rho^(p-1).
 * The reference hard-codes eps = 1e-10 (:28). */
TPO_API int tpo_mat_int_fnc(tpo_ctx *ctx, const double *x, double penal, double eps,
                    int mem);
/* set E (and optionally dEdz) directly, bypassing filter and SIMP */
TPO_API int tpo_set_moduli(tpo_ctx *ctx, const double *E, const double *dEdz, int mem);

/* TopOpt::FEAssemble + PCSetUp (FEAnalysis.cpp:432-490, :541-573): the
 * matrix-free fine operator with the Dirichlet fixes, Galerkin coarse
 * operators P^T A P on every level, Jacobi diagonals, Chebyshev bounds and
 * the coarsest-level Cholesky factor. */
TPO_API int tpo_fe_assemble(tpo_ctx *ctx, const tpo_solve_opts *opts);

/* TopOpt::FESolve (FEAnalysis.cpp:507-732): PCG + GMG on K U = F from the
 * context's current U (nonzero initial guess, :389). */
TPO_API int tpo_fe_solve(tpo_ctx *ctx, const tpo_solve_opts *opts,
                 tpo_solve_info *info);

/* solve K U = b for nrhs right-hand sides (column-major, 3*nNode each);
 * U holds the initial guesses and receives the solutions.  The right-hand
 * sides run in blocks of opts->rhs_block columns (power-of-two remainders):
 * one block shares every operator read, V-cycle launch and grid barrier,
 * with per-column CG scalars and convergence.  info: iterations and outer
 * passes summed over the right-hand sides, the largest relative residual,
 * the worst status.  (The reference solves its load cases one KSPSolve at
 * a time, FEAnalysis.cpp:673.) */
TPO_API int tpo_solve(tpo_ctx *ctx, const double *b, double *U, int32_t nrhs,
              int mem, const tpo_solve_opts *opts, tpo_solve_info *info);

/* y = K(rho) u on the finest level (the reference MatMult(K), with the
 * MatZeroRowsColumns identity rows, FEAnalysis.cpp:473), nrhs columns;
 * precision TPO_PREC_FP64 or TPO_PREC_MIXED (FP32 arithmetic). */
TPO_API int tpo_apply(tpo_ctx *ctx, const double *u, double *y, int32_t nrhs,
              int32_t precision, int mem);
/* FP32 form of tpo_apply on device buffers only (3*nNode floats each): the
 * matrix-free kernel alone, as used inside the mixed-precision solve. */
TPO_API int tpo_apply_f32(tpo_ctx *ctx, const float *u, float *y);
/* y = A_l u on GMG level l with the assembled Galerkin operator (l >= 1) */
TPO_API int tpo_apply_level(tpo_ctx *ctx, int32_t level, const double *u, double *y,
                    int mem);
/* tpo_apply_level in a chosen precision: TPO_PREC_FP64 as tpo_apply_level,
 * TPO_PREC_MIXED runs the FP32 operator the mixed-precision V-cycle uses on
 * that level (u rounded to FP32, y widened back); levels 0 .. the last one
 * above the persistent coarse levels. */
TPO_API int tpo_apply_level_prec(tpo_ctx *ctx, int32_t level, const double *u, double *y,
                                 int32_t precision, int mem);
/* Form of the FP32 level-1 operator (the reference's Galerkin PCMG level,
 * FEAnalysis.cpp:410-416): 0 automatic = the tensor-core matrix-free form
 * sum_E sum_i E_i G_i u_E whenever every element count is even and level 1
 * lies above the persistent coarse levels, else the stored stencil; 1 = the
 * stored half stencil always.  *tensor (optional) receives 1 when the
 * tensor-core form is in use.  Takes effect at the next apply or solve. */
TPO_API int tpo_set_level1_form(tpo_ctx *ctx, int32_t form, int32_t *tensor);
/* one application of the GMG V-cycle preconditioner z = M r (finest) */
TPO_API int tpo_vcycle(tpo_ctx *ctx, const double *r, double *z, int32_t precision,
               int mem);
/* lambda_max(D^-1 A_l) estimate used by the Chebyshev smoother */
TPO_API int tpo_level_lambda(const tpo_ctx *ctx, int32_t level, double *lambda);

/* ---- linear buckling (Stability, Buckling.cpp:15-414) ------------------- */

typedef struct {
  int32_t nev;        /* eigenvalues wanted: the largest of Ks phi = lambda K phi
                         (target LR, Buckling.cpp:69-70) (6) */
  int32_t block;      /* block size, nev <= block <= 32 (12) */
  int32_t maxit;      /* iterations (500, Buckling.cpp:71) */
  double tol;         /* converged when ||Ks x - lambda K x|| <= tol |lambda|
                         ||K x|| for the nev leading pairs (1e-6) */
  int32_t precond;    /* preconditioner: one GMG V-cycle in TPO_PREC_FP64 or
                         TPO_PREC_MIXED (FP32) arithmetic (FP64) */
  uint64_t seed;      /* start block seed (1) */
} tpo_eig_opts;

typedef struct {
  int32_t status;     /* TPO_OK, TPO_NOT_CONVERGED or TPO_E_BREAKDOWN */
  int32_t iterations;
  int32_t nconv;      /* leading pairs within tol */
  double max_resid;   /* largest relative residual of the nev pairs */
  double solve_ms;    /* host wall time of the eigensolve */
} tpo_eig_info;

TPO_API void tpo_default_eig_opts(tpo_eig_opts *opts);

/* Stability::StressFnc (Buckling.cpp:291-361) and the Dirichlet fix of
 * Buckling.cpp:29-30: Ks = sum_e -Es_e ks_e(U) from the context's current
 * U (after tpo_fe_solve) and Es = rho^p of the last tpo_mat_int_fnc (E
 * itself after tpo_set_moduli), fixed rows and columns zero. */
TPO_API int tpo_ks_assemble(tpo_ctx *ctx);
/* y = Ks u, nrhs columns (the reference MatMult(Ks)) */
TPO_API int tpo_ks_apply(tpo_ctx *ctx, const double *u, double *y, int32_t nrhs,
                 int mem);
/* the opts->nev largest eigenvalues of Ks phi = lambda K phi, descending,
 * in lambda[nev] (host); phi (optional, 3*nNode x nev column-major,
 * K-orthonormal, in `mem`) the eigenvectors.  Replaces the LOPGMRES call of
 * Stability::Function (Buckling.cpp:58-86) by block LOBPCG preconditioned
 * with the GMG V-cycle of tpo_fe_assemble.  Needs tpo_fe_assemble and
 * tpo_ks_assemble. */
TPO_API int tpo_buckling(tpo_ctx *ctx, const tpo_eig_opts *opts, double *lambda,
                 double *phi, int mem, tpo_eig_info *info);
/* The gradient of Stability::Function (Buckling.cpp:87-88, 113-272) with
 * TopOpt::Chain_Filter (Material_Interpolation.cpp:150-187): value = (sum
 * lambda_i^p)^(1/p) over nev <= 32 eigenpairs (lambda on the host; phi
 * 3*nNode x nev column-major and K-normalised, in `mem`, as tpo_buckling
 * returns them) and its gradient dvdx (nElem, in `mem`) with respect to the
 * design x; dvdrho (optional) is the gradient with respect to the filtered
 * density before the filter chain rule.  The nev adjoint systems
 * K v_i = d(phi_i^T Ks phi_i)/dU (:155-225) are solved as blocks of
 * right-hand sides with opts (NULL = defaults); info (optional) aggregates
 * them.  Needs tpo_fe_assemble, and tpo_ks_assemble from the current U. */
TPO_API int tpo_buckling_sensitivity(tpo_ctx *ctx, int32_t nev, const double *lambda,
                             const double *phi, double p, const tpo_solve_opts *opts,
                             double *value, double *dvdx, double *dvdrho, int mem,
                             tpo_solve_info *info);

/* Frequency::Function (Dynamic.cpp:18-171) with DiagMassFnc (:181-235):
 * the lumped mass M (element volume x density / 24 per node component
 * from the filtered density, plus mlump, optional per-dof point masses in
 * `mem`; 1e-8 at fixed dofs), then the largest eigenvalues of
 * M phi = lambda K phi (lambda = 1/omega^2, the lowest frequencies) until
 * more than nvals have converged and the last is separated from the one
 * before it by a relative 1e-5 (UNIQUE_LAST_NEV), by the block eigensolver
 * of tpo_buckling with opts (NULL = defaults; nev and block are set here).
 * lambda (host, room for 32) receives them descending and *nconv their
 * count; *value = (sum lambda^p)^(1/p) over all of them; dvdx (nElem in
 * `mem`, optional) its design gradient, summed over the first nvals - 1
 * eigenpairs as the reference does (:127-160), with the filter chain rule.
 * Needs tpo_fe_assemble; 1 <= nvals <= 29. */
TPO_API int tpo_frequency(tpo_ctx *ctx, int32_t nvals, double density, const double *mlump,
                  const tpo_eig_opts *opts, double p, double *lambda, int32_t *nconv,
                  double *value, double *dvdx, int mem, tpo_eig_info *info);

/* ---- MMA for two or more constraints (MMA.cpp:185-595) ----------------- */

typedef struct {
  double move;        /* step limit (0.5) */
  double asyinit;     /* asymptote parameters (0.5, 1.2, 0.7) */
  double asyincr;
  double asydecr;
  double albefa;      /* move-limit factor towards the asymptotes (0.1) */
  double raa0;        /* objective regularisation (1e-5) */
  double epsimin;     /* smallest epsilon of the dual Newton loop (1e-7) */
} tpo_mma_opts;

/* the defaults of MMA::Set_Defaults (MMA.h:21-23) */
TPO_API void tpo_default_mma_opts(tpo_mma_opts *opts);
/* MMA::MMAsub (MMA.cpp:185-343) with MMA::DualSolve (:353-595), the branch
 * MMA::Update takes for m >= 2 constraints, over nElem design variables:
 * asymptotes from x, xold1, xold2 (fresh while *fresh_start and iter < 3;
 * *fresh_start is cleared once not), the convex approximation, the dual
 * Newton iteration on the m multipliers (the whole update in one persistent
 * GPU launch), then xold2 <- xold1 <- x, x <- the subproblem
 * solution, *change = max |x - xold1| / (xmax - xmin).  x, xold1, xold2,
 * low and upp are the caller's state, updated in place; xmin, xmax, dfdx
 * (nElem) and dgdx (nElem x m, column-major) are read, all in `mem`; g (m)
 * on the host.  The constants are Set_m's (a0 = b0 = 1, a = 0, c = 1000,
 * d = 1); 1 <= m <= 8. */
TPO_API int tpo_mma_update(tpo_ctx *ctx, const tpo_mma_opts *opts, int32_t iter,
                   int32_t *fresh_start, int32_t m, double *x, double *xold1,
                   double *xold2, double *low, double *upp, const double *xmin,
                   const double *xmax, const double *dfdx, const double *g,
                   const double *dgdx, double *change, int mem);
/* the number of dual Newton steps (SearchDir solves) the last successful
 * tpo_mma_update took */
TPO_API int tpo_mma_last_info(const tpo_ctx *ctx, int32_t *newton_steps);

/* U, F, x, rho, E, dEdz, Es accessors: which = "U","F","x","rho","E","dEdz","Es" */
TPO_API int tpo_get_vector(const tpo_ctx *ctx, const char *which, double *out, int mem);
TPO_API int tpo_set_vector(tpo_ctx *ctx, const char *which, const double *in, int mem);

/* Compliance::Function (Compliance.cpp:15-57) on the context's U:
 * C = U.F and dC/dx = P^T(-dEdz .* u_e^T K0 u_e) (Chain_Filter,
 * Material_Interpolation.cpp:150-187).  dCdx / dCdrho may be NULL. */
TPO_API int tpo_compliance(tpo_ctx *ctx, double *C, double *dCdx, double *dCdrho,
                   int mem);
/* Volume::Function (Volume.cpp:15-41): V = sum(rho)/nElem, dV/dx */
TPO_API int tpo_volume(tpo_ctx *ctx, double *V, double *dVdx, int mem);
/* MatMult(P) (transpose = 0) or MatMultTranspose(P) (transpose = 1) */
TPO_API int tpo_filter(tpo_ctx *ctx, const double *in, double *out, int32_t transpose,
               int mem);

/* MMA::OCsub (MMA.cpp:103-180) on the GPU, OCeta = 0.5: x (nElem) is
 * updated in place; dfdx is clipped to <= 0 in place; returns Change. */
TPO_API int tpo_oc_update(tpo_ctx *ctx, double *x, const double *xmin,
                  const double *xmax, double *dfdx, double g,
                  const double *dgdx, double move, double *change, int mem);

/* block until all work of the context is done */
TPO_API int tpo_sync(tpo_ctx *ctx);

/* run the context's work on a caller stream (a cudaStream_t passed as
 * void*); NULL restores the context's own stream.  No reference
 * counterpart: it lets a host framework order and time the kernels. */
TPO_API int tpo_set_stream(tpo_ctx *ctx, void *stream);

/* number of kernels this library has launched in the process (graph
 * launches count their kernel nodes).  No reference counterpart. */
TPO_API int64_t tpo_kernel_launches(void);

/* ---- the reference's output and restart files (TopOpt.cpp:97-508,
 * RecMesh.cpp:34-412) ---------------------------------------------------
 * index_bytes is sizeof(PetscInt) of the PETSc build the files belong to
 * (4 by default, 8 with 64-bit indices).  Raw arrays are native-endian as
 * the reference writes them with ofstream / MPI-IO; the PETSc binary
 * viewer encoding is big-endian.  One process: the distributions are
 * [0, nElem] and [0, nNode].  No .info side files are written.  Writers
 * expect `folder` to exist (the reference writes into the working
 * directory).  Calls without a context report errors through
 * tpo_last_error(NULL). */

/* VecView / VecLoad on a binary viewer: [1211214, n] as PetscInt, then n
 * doubles.  tpo_read_vec_bin with v = NULL returns the length only. */
TPO_API int tpo_write_vec_bin(const char *path, const double *v, int64_t n,
                              int32_t index_bytes);
TPO_API int tpo_read_vec_bin(const char *path, double *v, int64_t cap, int64_t *n,
                             int32_t index_bytes);
/* MatView / MatLoad of an AIJ matrix: [1211216, M, N, nnz], the M row
 * lengths, the column indices, the values; rowptr has M + 1 entries.
 * tpo_read_mat_bin with rowptr = NULL returns the sizes only. */
TPO_API int tpo_write_mat_bin(const char *path, int64_t M, int64_t N, const int64_t *rowptr,
                              const int64_t *col, const double *val, int32_t index_bytes);
TPO_API int tpo_read_mat_bin(const char *path, int64_t *M, int64_t *N, int64_t *nnz,
                             int64_t *rowptr, int64_t *col, double *val, int64_t cap_rows,
                             int64_t cap_nnz, int32_t index_bytes);
/* TopOpt::MeshOut (TopOpt.cpp:97-359) into `folder`: Element_/Node_
 * Distribution, elements, nodes, the load and support lists (eigen
 * supports, springs and masses empty), Filter.bin (the density filter P),
 * Max_Filter.bin and Void_Edge_Volume.bin (the max-length-scale filter of
 * radius rmax, unscaled, and max(rowsum) - rowsum), active.bin and the
 * interpolations P<l>.bin with P<l>.bin.split. */
TPO_API int tpo_mesh_out(tpo_ctx *ctx, const char *folder, double rmax, int32_t index_bytes);
/* TopOpt::PrintVals (TopOpt.cpp:445-508): U, x, V (the filtered density),
 * Es, E as <name><name_suffix>.bin, and the mode shapes phiB (nB columns)
 * and phiD (nD columns) of 3*nNode host doubles each as
 * phiB<suffix>_mode<i>.bin and phiD_<suffix>_mode<i>.bin. */
TPO_API int tpo_print_vals(tpo_ctx *ctx, const char *folder, const char *name_suffix,
                           const double *phiB, int32_t nB, const double *phiD, int32_t nD,
                           int32_t index_bytes);
/* TopOpt::LoadMesh (RecMesh.cpp:34-412) for a structured hex8 box: a new
 * context from a MeshOut folder.  nel and dx come from the files (params
 * supplies E0, nu, rmin and mg_levels; mg_levels <= 0 takes one more than
 * the P<l>.bin files present); the support and load lists become the BCs.
 * A Filter.bin that is not the radius-rmin filter of the mesh, springs,
 * eigen-only supports or passive elements are refused. */
TPO_API int tpo_load_mesh(const char *folder, const tpo_mesh_params *params,
                          int32_t index_bytes, tpo_ctx **out);
/* The design part of LoadMesh (RecMesh.cpp:391-404) with Main.cpp:52-56:
 * x (nElem) = 0.5, then x_pen<p>.bin for each penalty in turn until one is
 * missing.  *penal (in: the current penalty, out: the penalty reached) and
 * *start (the index of the first penalty still to run) may be NULL. */
TPO_API int tpo_load_design(tpo_ctx *ctx, const char *folder, const double *penalties,
                            int32_t npen, double *x, double *penal, int32_t *start,
                            int32_t index_bytes);
/* massNodes.bin / masses.bin (RecMesh.cpp:147-180) as the 3*nNode point
 * mass vector tpo_frequency takes (summed where a node repeats). */
TPO_API int tpo_load_point_masses(tpo_ctx *ctx, const char *folder, double *mlump,
                                  int32_t index_bytes);

/* Self-test of the failure detection of the persistent kernels.  It has no
 * counterpart in the reference, whose only failure reporting is the solver
 * status (FEAnalysis.cpp:677-684).  The coarse-grid V-cycle, the OC
 * bisection and the MMA update each run as one cooperative launch whose
 * phases are separated by a grid barrier with a bounded wait; a wait that
 * runs out sets a fault flag, every block returns, and the next read-back
 * reports TPO_E_CUDA and resets the barrier.  This call runs that
 * machinery on its own: `blocks` (1..64) co-resident blocks cross `phases`
 * (1..1024) barriers; when skip_block is in [0, blocks) that block leaves
 * before its first arrival, so the other blocks' waits run out after
 * max_polls (1..2^22) polls each.  *completed (optional) receives the
 * number of blocks that passed every barrier.  Returns TPO_OK when all
 * arrived, TPO_E_CUDA with a message after a wait ran out (the counter and
 * the flag are reset, the context stays usable). */
TPO_API int tpo_barrier_selftest(tpo_ctx *ctx, int32_t blocks, int32_t phases,
                                 int32_t skip_block, int32_t max_polls,
                                 int32_t *completed);

/* Filtered compliance sensitivity that allocates nothing.  It has no
 * counterpart in the reference.  It serves callers that may not call
 * cudaMalloc: a plugin whose host framework owns all device memory through
 * its own pool, code running while a CUDA graph is being captured, or a
 * process that fixes its device memory budget up front.  They cannot create
 * a context (tpo_create allocates), so this call needs none:
 *   dCdx = P^T(-dEdz .* u_e^T K0 u_e)   (Compliance.cpp:37-51)
 * for the mesh nel/dx, material E0/nu and filter radius rmin, on caller
 * device buffers U (3*nNode), dEdz (nElem) and dCdx (nElem), issued on
 * `stream` (a cudaStream_t; NULL is the legacy default stream).
 * Its per-element intermediate lives in a fixed device array of
 * TPO_NOALLOC_MAX_ELEMS doubles (8 MiB) inside the library; every GPU that
 * loads the library holds that array until the process exits.  Meshes with
 * more elements are rejected with TPO_E_ARG and a message.  The first call
 * on a device looks the array's address up with that device current, so
 * make that first call before any stream capture.  Every call shares the
 * one array: calls whose kernels overlap on the same GPU race on it, so
 * order them (one stream, or events).  `msg` (optional, msg_len bytes)
 * receives an error description. */
#define TPO_NOALLOC_MAX_ELEMS (1 << 20)
TPO_API int tpo_sensitivity_noalloc(const int32_t nel[3], const double dx[3],
                                    double E0, double nu, double rmin,
                                    const double *U, const double *dEdz,
                                    double *dCdx, void *stream, char *msg,
                                    int32_t msg_len);

#ifdef __cplusplus
}
#endif
#endif /* TOPOPT_B200_H */
