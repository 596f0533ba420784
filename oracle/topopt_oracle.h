/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the TopOpt3D finite-element
 * hot path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load this library, and only as the checker / CPU baseline; the
 * product (topopt3d_b200) never links or calls it.
 *
 * Plain C (C11 + optional OpenMP), FP64 throughout.  Every routine restates
 * the reference algorithm and names the reference file:line it follows
 * (paths are relative to the darinpeetz/TopOpt3D tree).  The solver
 * arithmetic that the reference delegates to PETSc (CG, PCMG with Galerkin
 * coarse operators, Chebyshev/Jacobi smoothing, direct coarse solve) is
 * restated from the published algorithms; the reference pins no PETSc
 * version and ships no tests or golden vectors, so parity against the
 * reference itself is UNPINNED -- the oracle is pinned by mathematical
 * known-answer tests and by an independent scipy sparse direct solve.
 */
#ifndef TOPOPT_ORACLE_H
#define TOPOPT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- mesh, element, constitutive -------------------------------------- */

/* D (6x6, row-major, Voigt [xx,yy,zz,xy,yz,xz]); RecMesh.cpp:453-462 */
void tor_constitutive(double E0, double nu, double D[36]);

/* K0 (24x24 row-major, dof = 3*local_node + comp) of a dx*dy*dz box element,
 * 2x2x2 Gauss at +-1/sqrt(3), W = 1; FEAnalysis.cpp:869-1050 */
void tor_element_stiffness(const double dx[3], double E0, double nu,
                           double K0[576]);

/* the 8 global node numbers of element e; RecMesh.cpp:486-512 */
void tor_element_nodes(const int nel[3], int64_t e, int64_t nodes[8]);

/* node coordinates (Eigen LinSpaced semantics); RecMesh.cpp:565-597 */
void tor_node_coords(const int nel[3], const double dx[3],
                     const double origin[3], int64_t n, double xyz[3]);

/* Set_BC node selection (Inputs.cpp:105-124): writes the selected node
 * numbers in increasing order into out (may be NULL), returns the count. */
int64_t tor_select_nodes(const int nel[3], const double dx[3],
                         const double origin[3], const double center[3],
                         const double radius[3], const double limits[6],
                         int64_t *out);

/* ---- density filter (Filter.cpp:21-150) -------------------------------- */

/* nnz of the radius-R filter (pass NULL arrays to query), else fills the
 * row-normalised CSR (rowptr[nElem+1], col, val). */
int64_t tor_filter_build(const int nel[3], const double dx[3], double R,
                         int64_t *rowptr, int32_t *col, double *val);
void tor_csr_mult(int64_t nrow, const int64_t *rowptr, const int32_t *col,
                  const double *val, const double *x, double *y);
void tor_csr_mult_t(int64_t nrow, int64_t ncol, const int64_t *rowptr,
                    const int32_t *col, const double *val, const double *x,
                    double *y);

/* PETSc VecPow special cases, used by MatIntFnc */
double tor_vecpow(double v, double p);

/* MatIntFnc with vdMin <= 0 (Material_Interpolation.cpp:20-75):
 * from filtered densities rho -> E, dEdz, Es, dEsdz (SIMP). */
void tor_simp(int64_t ne, const double *rho, double penal, double eps,
              double *E, double *dEdz, double *Es, double *dEsdz);

/* ---- the oracle problem object ----------------------------------------- */

typedef struct tor_problem tor_problem;

typedef struct {
  int    nel[3];
  double dx[3];
  double E0, nu;
  double rmin;        /* density filter radius (absolute) */
  int    mg_levels;   /* total GMG levels including the finest */
} tor_params;

typedef struct {
  double rtol;        /* relative to ||b||, unpreconditioned norm */
  int    maxit;
  int    cheb_degree; /* smoothing steps per level (pre and post) */
  double cheb_lo, cheb_hi; /* interval = [lo, hi] * lambda_max estimate */
  int    power_its;   /* power iterations for lambda_max(D^-1 A) */
} tor_solve_opts;

tor_problem *tor_create(const tor_params *p);
void tor_destroy(tor_problem *P);
int64_t tor_n_nodes(const tor_problem *P);
int64_t tor_n_elems(const tor_problem *P);

/* boundary conditions: fixed-component mask per node (bit c = comp c fixed)
 * and the load vector (3*nNode).  Either set them directly or add Set_BC
 * regions (type 0 = support, 1 = load). */
void tor_set_bc_arrays(tor_problem *P, const uint8_t *fixmask, const double *F);
int64_t tor_add_bc(tor_problem *P, int type, const double center[3],
                   const double radius[3], const double limits[6],
                   const double values[3]);
void tor_get_bc(const tor_problem *P, uint8_t *fixmask, double *F);

/* MatIntFnc: x -> rho = P x -> E, dEdz (vdMin <= 0 path) */
void tor_set_design(tor_problem *P, const double *x, double penal, double eps);
void tor_get_material(const tor_problem *P, double *rho, double *E,
                      double *dEdz);
/* set the element moduli directly (bypasses the filter) */
void tor_set_moduli(tor_problem *P, const double *E, const double *dEdz);

/* FEAssemble + PCSetUp: assembled K with the BC fixes, the Galerkin
 * hierarchy, diagonals, lambda estimates and the coarse Cholesky factor. */
int tor_assemble(tor_problem *P, const tor_solve_opts *o);

/* y = K u with the assembled fine matrix */
void tor_apply(const tor_problem *P, const double *u, double *y);
/* y = A_l u on GMG level l (0 = finest) */
void tor_apply_level(const tor_problem *P, int level, const double *u,
                     double *y);
int64_t tor_level_nodes(const tor_problem *P, int level, int dims[3]);
/* dense 3x3 block (row node i, col node j) of A_l, 0 if absent */
int tor_level_block(const tor_problem *P, int level, int64_t i, int64_t j,
                    double blk[9]);
double tor_level_lambda(const tor_problem *P, int level);
/* fine -> coarse prolongation weights of level l (fine node f, coarse c) */
double tor_prolong_weight(const tor_problem *P, int level, int64_t f,
                          int64_t c);
/* one V-cycle preconditioner application z = M r on the finest level */
void tor_vcycle(tor_problem *P, const double *r, double *z);

/* FESolve: PCG + GMG on K U = F (U holds the initial guess).  Returns
 * 0 converged, 1 max-it, -1 breakdown / non-finite.  its, relres out. */
int tor_solve(tor_problem *P, const tor_solve_opts *o, double *U, int *its,
              double *relres);
/* solve with an arbitrary right-hand side b */
int tor_solve_rhs(tor_problem *P, const tor_solve_opts *o, const double *b,
                  double *U, int *its, double *relres);

/* Compliance::Function (Compliance.cpp:15-57): C = U.F,
 * dCdx = P^T( -dEdz .* (u_e^T K0 u_e) ) */
void tor_compliance(const tor_problem *P, const double *U, double *C,
                    double *dCdx, double *dCdrho);
/* Volume::Function (Volume.cpp:15-41) */
void tor_volume(const tor_problem *P, double *V, double *dVdx);
/* filter forward (rho = P x) or transpose (P^T g) */
void tor_filter(const tor_problem *P, const double *in, double *out,
                int transpose);

/* MMA::OCsub (MMA.cpp:103-180), OCeta = 0.5: updates x in place and
 * returns Change. */
double tor_oc_update(int64_t n, double *x, const double *xmin,
                     const double *xmax, double *dfdx, double g,
                     const double *dgdx, double move);


/* ---- buckling ------------------------------------------------------------ */
/* element stress stiffness ks (24x24, row-major, reference local node order)
 * for element displacements u (Buckling.cpp:313-327) */
void tor_stress_stiffness_element(const double dx[3], double E0, double nu,
                                  const double u[24], double ks[576]);
/* Ks = sum_e -Es_e ks_e(U) with the Dirichlet rows/columns zeroed
 * (Buckling.cpp:22-30, 291-361) */
void tor_ks_assemble(tor_problem *P, const double *U);
void tor_ks_apply(const tor_problem *P, const double *u, double *y);
void tor_get_es(const tor_problem *P, double *Es);

#ifdef __cplusplus
}
#endif
#endif
