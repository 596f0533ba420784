/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the TopOpt3D FE hot path.
 * See topopt_oracle.h for the scope statement.  Reference citations are
 * file:line in the darinpeetz/TopOpt3D tree.
 *
 * Storage: the assembled stiffness and every Galerkin level are 3x3-block
 * CSR matrices over nodes (the reference assembles K with block size 3,
 * FEAnalysis.cpp:329); the prolongations are node-level scalar CSR
 * matrices (each reference entry is weight * I3, Interpolation.cpp:323).
 */
#include "topopt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* constitutive matrix and element stiffness                                 */
/* ------------------------------------------------------------------------ */

void tor_constitutive(double E0, double nu, double D[36])
{
  /* RecMesh.cpp:453-462 */
  double c = E0 / ((1 + nu) * (1 - 2 * nu));
  double G = E0 / (2 * (1 + nu));
  double t1 = (1 - nu) * c, t2 = G, t3 = nu * c;
  memset(D, 0, 36 * sizeof(double));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[6 * i + j] = (i == j) ? t1 : t3;
  D[6 * 3 + 3] = D[6 * 4 + 4] = D[6 * 5 + 5] = t2;
}

/* parent-coordinate shape derivative signs, node order of dN
 * (FEAnalysis.cpp:955-986) */
static const int kNodeSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1},
                                    {-1, 1, -1},  {-1, -1, 1}, {1, -1, 1},
                                    {1, 1, 1},    {-1, 1, 1}};

static double det3(const double a[9])
{
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

static void inv3(const double a[9], double r[9])
{
  double d = det3(a);
  r[0] = (a[4] * a[8] - a[5] * a[7]) / d;
  r[1] = (a[2] * a[7] - a[1] * a[8]) / d;
  r[2] = (a[1] * a[5] - a[2] * a[4]) / d;
  r[3] = (a[5] * a[6] - a[3] * a[8]) / d;
  r[4] = (a[0] * a[8] - a[2] * a[6]) / d;
  r[5] = (a[2] * a[3] - a[0] * a[5]) / d;
  r[6] = (a[3] * a[7] - a[4] * a[6]) / d;
  r[7] = (a[1] * a[6] - a[0] * a[7]) / d;
  r[8] = (a[0] * a[4] - a[1] * a[3]) / d;
}

void tor_element_stiffness(const double dx[3], double E0, double nu,
                           double K0[576])
{
  /* LocalK (FEAnalysis.cpp:869-892) with GaussPoints (900-926), dN
   * (936-990) and AssignB (1024-1046). */
  double D[36];
  tor_constitutive(E0, nu, D);
  double coords[8][3];
  for (int n = 0; n < 8; n++)
    for (int d = 0; d < 3; d++)
      coords[n][d] = kNodeSign[n][d] > 0 ? dx[d] : 0.0;
  memset(K0, 0, 576 * sizeof(double));
  const double g = 1.0 / sqrt(3.0);
  for (int q = 0; q < 8; q++) {
    double xi = kNodeSign[q][0] * g, eta = kNodeSign[q][1] * g,
           zeta = kNodeSign[q][2] * g;
    double dNdxi[3][8];
    for (int n = 0; n < 8; n++) {
      double a = kNodeSign[n][0], b = kNodeSign[n][1], c = kNodeSign[n][2];
      dNdxi[0][n] = a * (1 + b * eta) * (1 + c * zeta) / 8.0;
      dNdxi[1][n] = b * (1 + a * xi) * (1 + c * zeta) / 8.0;
      dNdxi[2][n] = c * (1 + a * xi) * (1 + b * eta) / 8.0;
    }
    double J[9] = {0}, iJ[9];
    for (int r = 0; r < 3; r++)
      for (int cc = 0; cc < 3; cc++)
        for (int n = 0; n < 8; n++) J[3 * r + cc] += dNdxi[r][n] * coords[n][cc];
    double detJ = det3(J);
    inv3(J, iJ);
    double dNdx[3][8];
    for (int r = 0; r < 3; r++)
      for (int n = 0; n < 8; n++) {
        double s = 0;
        for (int k = 0; k < 3; k++) s += iJ[3 * r + k] * dNdxi[k][n];
        dNdx[r][n] = s;
      }
    double B[6][24];
    memset(B, 0, sizeof(B));
    for (int n = 0; n < 8; n++) {
      B[0][3 * n] = dNdx[0][n];
      B[1][3 * n + 1] = dNdx[1][n];
      B[2][3 * n + 2] = dNdx[2][n];
      B[3][3 * n] = dNdx[1][n];
      B[3][3 * n + 1] = dNdx[0][n];
      B[4][3 * n + 1] = dNdx[2][n];
      B[4][3 * n + 2] = dNdx[1][n];
      B[5][3 * n] = dNdx[2][n];
      B[5][3 * n + 2] = dNdx[0][n];
    }
    double DB[6][24];
    for (int r = 0; r < 6; r++)
      for (int cc = 0; cc < 24; cc++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += D[6 * r + k] * B[k][cc];
        DB[r][cc] = s;
      }
    for (int r = 0; r < 24; r++)
      for (int cc = 0; cc < 24; cc++) {
        double s = 0;
        for (int k = 0; k < 6; k++) s += B[k][r] * DB[k][cc];
        K0[24 * r + cc] += s * detJ;   /* W[q] = 1 */
      }
  }
}

void tor_element_nodes(const int nel[3], int64_t e, int64_t nodes[8])
{
  /* RecMesh.cpp:486-512 */
  int64_t Nx = nel[0] + 1, Ny = nel[1] + 1;
  int64_t i = e % nel[0], j = (e / nel[0]) % nel[1], k = e / ((int64_t)nel[0] * nel[1]);
  int64_t n0 = i + j * Nx + k * Nx * Ny;
  nodes[0] = n0;
  nodes[1] = n0 + 1;
  nodes[2] = n0 + 1 + Nx;
  nodes[3] = n0 + Nx;
  for (int a = 0; a < 4; a++) nodes[4 + a] = nodes[a] + Nx * Ny;
}

static double linspaced(double lo, double hi, int64_t n, int64_t i)
{
  /* Eigen 3.3 LinSpaced for floating point (non-flipped branch) */
  if (n == 1) return hi;
  double step = (hi - lo) / (double)(n - 1);
  if (fabs(hi) < fabs(lo))
    return (i == 0) ? lo : hi - (double)(n - 1 - i) * step;
  return (i == n - 1) ? hi : lo + (double)i * step;
}

void tor_node_coords(const int nel[3], const double dx[3],
                     const double origin[3], int64_t n, double xyz[3])
{
  /* RecMesh.cpp:582-597 on one rank: node.col(d) = LinSpaced(Nnd(d),
   * origin, dx*nel + origin) replicated lexicographically */
  int64_t N[3] = {nel[0] + 1, nel[1] + 1, nel[2] + 1};
  int64_t idx[3] = {n % N[0], (n / N[0]) % N[1], n / (N[0] * N[1])};
  for (int d = 0; d < 3; d++)
    xyz[d] = linspaced(origin[d], dx[d] * nel[d] + origin[d], N[d], idx[d]);
}

int64_t tor_select_nodes(const int nel[3], const double dx[3],
                         const double origin[3], const double center[3],
                         const double radius[3], const double limits[6],
                         int64_t *out)
{
  /* Inputs.cpp:116-124: distance test <= 1 inside the limits */
  int64_t nn = (int64_t)(nel[0] + 1) * (nel[1] + 1) * (nel[2] + 1), cnt = 0;
  for (int64_t n = 0; n < nn; n++) {
    double xyz[3], dist = 0;
    int valid = 1;
    tor_node_coords(nel, dx, origin, n, xyz);
    for (int d = 0; d < 3; d++) {
      double t = (xyz[d] - center[d]) / radius[d];
      dist += t * t;
      valid = valid && (xyz[d] >= limits[2 * d]) && (xyz[d] <= limits[2 * d + 1]);
    }
    if (valid && dist <= 1) {
      if (out) out[cnt] = n;
      cnt++;
    }
  }
  return cnt;
}

/* ------------------------------------------------------------------------ */
/* density filter                                                            */
/* ------------------------------------------------------------------------ */

int64_t tor_filter_build(const int nel[3], const double dx[3], double R,
                         int64_t *rowptr, int32_t *col, double *val)
{
  /* RecFilter (Filter.cpp:21-94) + Assemble_Filter row scaling (136-147) */
  short N[3];
  for (int d = 0; d < 3; d++) N[d] = (short)(R / dx[d]);
  int T = (2 * N[0] + 1) * (2 * N[1] + 1) * (2 * N[2] + 1);
  double *dist = (double *)malloc(sizeof(double) * T);
  char *in = (char *)malloc(T);
  for (int k = -N[2]; k <= N[2]; k++)
    for (int j = -N[1]; j <= N[1]; j++)
      for (int i = -N[0]; i <= N[0]; i++) {
        int ind = i + N[0] + (j + N[1]) * (2 * N[0] + 1) +
                  (k + N[2]) * (2 * N[0] + 1) * (2 * N[1] + 1);
        dist[ind] = sqrt(pow(i * dx[0], 2) + pow(j * dx[1], 2) + pow(k * dx[2], 2));
        in[ind] = dist[ind] < R;
      }
  int64_t ne = (int64_t)nel[0] * nel[1] * nel[2], nnz = 0;
  if (rowptr) rowptr[0] = 0;
  for (int64_t el = 0; el < ne; el++) {
    int eli = (int)(el % nel[0]), elj = (int)((el / nel[0]) % nel[1]),
        elk = (int)(el / ((int64_t)nel[0] * nel[1]));
    int64_t start = nnz;
    double rs = 0;
    for (int k = -N[2]; k <= N[2]; k++)
      for (int j = -N[1]; j <= N[1]; j++)
        for (int i = -N[0]; i <= N[0]; i++) {
          int ind = i + N[0] + (j + N[1]) * (2 * N[0] + 1) +
                    (k + N[2]) * (2 * N[0] + 1) * (2 * N[1] + 1);
          int valid = in[ind] && i + eli >= 0 && i + eli < nel[0] &&
                      j + elj >= 0 && j + elj < nel[1] && k + elk >= 0 &&
                      k + elk < nel[2];
          if (!valid) continue;
          if (col) {
            col[nnz] = (int32_t)(el + i + (int64_t)j * nel[0] +
                                 (int64_t)k * nel[0] * nel[1]);
            val[nnz] = 1 - dist[ind] / R;
            rs += val[nnz];
          }
          nnz++;
        }
    if (val) {
      double inv = 1.0 / rs;   /* VecPointwiseDivide(Ones, rowSum) */
      for (int64_t t = start; t < nnz; t++) val[t] *= inv;
    }
    if (rowptr) rowptr[el + 1] = nnz;
  }
  free(dist);
  free(in);
  return nnz;
}

void tor_csr_mult(int64_t nrow, const int64_t *rowptr, const int32_t *col,
                  const double *val, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < nrow; r++) {
    double s = 0;
    for (int64_t t = rowptr[r]; t < rowptr[r + 1]; t++) s += val[t] * x[col[t]];
    y[r] = s;
  }
}

void tor_csr_mult_t(int64_t nrow, int64_t ncol, const int64_t *rowptr,
                    const int32_t *col, const double *val, const double *x,
                    double *y)
{
  memset(y, 0, sizeof(double) * ncol);
  for (int64_t r = 0; r < nrow; r++)
    for (int64_t t = rowptr[r]; t < rowptr[r + 1]; t++) y[col[t]] += val[t] * x[r];
}

double tor_vecpow(double v, double p)
{
  /* PETSc VecPow special cases */
  if (p == 1.0) return v;
  if (p == -1.0) return 1.0 / v;
  if (p == 0.0) return (v == v) ? 1.0 : v;
  if (p == 0.5) return v >= 0 ? sqrt(v) : INFINITY;
  if (p == -0.5) return v >= 0 ? 1.0 / sqrt(v) : INFINITY;
  if (p == 2.0) return v * v;
  if (p == -2.0) return 1.0 / (v * v);
  return v >= 0 ? pow(v, p) : INFINITY;
}

void tor_simp(int64_t ne, const double *rho, double penal, double eps,
              double *E, double *dEdz, double *Es, double *dEsdz)
{
  /* Material_Interpolation.cpp:40-75 with vdMin <= 0: y = 1, z = rho */
  for (int64_t e = 0; e < ne; e++) {
    double z = rho[e];
    double d = tor_vecpow(z, penal - 1);    /* :67-68 */
    double es = d * z;                      /* :69 */
    d = d * penal;                          /* :70 */
    if (Es) Es[e] = es;
    if (dEsdz) dEsdz[e] = d;
    dEdz[e] = d * (1 - eps);                /* :72-73 */
    E[e] = eps + (1 - eps) * es;            /* :74-75 */
  }
}

/* ------------------------------------------------------------------------ */
/* block sparse matrices                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  int64_t n;        /* block rows (nodes) */
  int64_t *rowptr;
  int32_t *col;
  double *val;      /* 9 per block, row-major */
} bsr3;

typedef struct {    /* node-level scalar CSR, nrow x ncol */
  int64_t nrow, ncol;
  int64_t *rowptr;
  int32_t *col;
  double *val;
} csr;

static void bsr_free(bsr3 *A)
{
  free(A->rowptr); free(A->col); free(A->val);
  memset(A, 0, sizeof(*A));
}

static void csr_free(csr *A)
{
  free(A->rowptr); free(A->col); free(A->val);
  memset(A, 0, sizeof(*A));
}

static void bsr_mult(const bsr3 *A, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < A->n; r++) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t t = A->rowptr[r]; t < A->rowptr[r + 1]; t++) {
      const double *b = A->val + 9 * t;
      const double *xx = x + 3 * (int64_t)A->col[t];
      s0 += b[0] * xx[0] + b[1] * xx[1] + b[2] * xx[2];
      s1 += b[3] * xx[0] + b[4] * xx[1] + b[5] * xx[2];
      s2 += b[6] * xx[0] + b[7] * xx[1] + b[8] * xx[2];
    }
    y[3 * r] = s0; y[3 * r + 1] = s1; y[3 * r + 2] = s2;
  }
}

static const double *bsr_find(const bsr3 *A, int64_t r, int64_t c)
{
  int64_t lo = A->rowptr[r], hi = A->rowptr[r + 1] - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) / 2;
    if (A->col[mid] == c) return A->val + 9 * mid;
    if (A->col[mid] < c) lo = mid + 1; else hi = mid - 1;
  }
  return NULL;
}

/* ------------------------------------------------------------------------ */
/* problem object                                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  int dims[3];        /* nodes per dimension */
  int64_t nn;         /* nodes */
  bsr3 A;
  double *dinv;       /* 1 / diag(A), 3*nn */
  double lam;         /* lambda_max(D^-1 A) estimate */
  csr P;              /* prolongation from level+1 (rows = this level) */
  csr PT;             /* its transpose */
  double *b, *x, *r, *t1, *t2; /* V-cycle work vectors */
} level_t;

struct tor_problem {
  tor_params prm;
  int64_t ne, nn;
  double K0[576];
  uint8_t *fix;       /* per-node fixed-component bitmask */
  double *F;
  /* filter */
  int64_t fnnz;
  int64_t *frow;
  int32_t *fcol;
  double *fval;
  /* material */
  double *x, *rho, *E, *dEdz;
  double *Es;         /* rho^p without E_min (Material_Interpolation.cpp:69) */
  bsr3 Ks;            /* stress stiffness (Buckling.cpp:291-361) */
  /* hierarchy */
  int L;
  level_t *lev;
  double *chol;       /* dense Cholesky factor of the coarsest level */
  int64_t nc;         /* coarsest dof count */
  tor_solve_opts opts;
  int assembled;
};

tor_problem *tor_create(const tor_params *p)
{
  tor_problem *P = (tor_problem *)calloc(1, sizeof(tor_problem));
  P->prm = *p;
  P->ne = (int64_t)p->nel[0] * p->nel[1] * p->nel[2];
  P->nn = (int64_t)(p->nel[0] + 1) * (p->nel[1] + 1) * (p->nel[2] + 1);
  tor_element_stiffness(p->dx, p->E0, p->nu, P->K0);
  P->fix = (uint8_t *)calloc(P->nn, 1);
  P->F = (double *)calloc(3 * P->nn, sizeof(double));
  P->fnnz = tor_filter_build(p->nel, p->dx, p->rmin, NULL, NULL, NULL);
  P->frow = (int64_t *)malloc(sizeof(int64_t) * (P->ne + 1));
  P->fcol = (int32_t *)malloc(sizeof(int32_t) * P->fnnz);
  P->fval = (double *)malloc(sizeof(double) * P->fnnz);
  tor_filter_build(p->nel, p->dx, p->rmin, P->frow, P->fcol, P->fval);
  P->x = (double *)calloc(P->ne, sizeof(double));
  P->rho = (double *)calloc(P->ne, sizeof(double));
  P->E = (double *)calloc(P->ne, sizeof(double));
  P->dEdz = (double *)calloc(P->ne, sizeof(double));
  P->Es = (double *)calloc(P->ne, sizeof(double));
  P->L = p->mg_levels < 1 ? 1 : p->mg_levels;
  P->lev = (level_t *)calloc(P->L, sizeof(level_t));
  return P;
}

static void free_levels(tor_problem *P)
{
  for (int l = 0; l < P->L; l++) {
    level_t *v = &P->lev[l];
    bsr_free(&v->A);
    csr_free(&v->P);
    csr_free(&v->PT);
    free(v->dinv); free(v->b); free(v->x); free(v->r); free(v->t1); free(v->t2);
    v->dinv = v->b = v->x = v->r = v->t1 = v->t2 = NULL;
  }
  free(P->chol);
  P->chol = NULL;
  P->assembled = 0;
}

void tor_destroy(tor_problem *P)
{
  if (!P) return;
  free_levels(P);
  free(P->lev);
  free(P->fix); free(P->F);
  free(P->frow); free(P->fcol); free(P->fval);
  free(P->x); free(P->rho); free(P->E); free(P->dEdz); free(P->Es);
  bsr_free(&P->Ks);
  free(P);
}

int64_t tor_n_nodes(const tor_problem *P) { return P->nn; }
int64_t tor_n_elems(const tor_problem *P) { return P->ne; }

void tor_set_bc_arrays(tor_problem *P, const uint8_t *fixmask, const double *F)
{
  if (fixmask) memcpy(P->fix, fixmask, P->nn);
  if (F) memcpy(P->F, F, sizeof(double) * 3 * P->nn);
}

int64_t tor_add_bc(tor_problem *P, int type, const double center[3],
                   const double radius[3], const double limits[6],
                   const double values[3])
{
  /* Set_BC (Inputs.cpp:105-223): SUPPORT sets the fixed components of every
   * selected node (fixedDof, FEAnalysis.cpp:236-246); LOAD adds the full
   * value vector to every selected node (FEAnalysis.cpp:352-355). */
  static const double origin[3] = {0, 0, 0};
  int64_t cnt = tor_select_nodes(P->prm.nel, P->prm.dx, origin, center, radius,
                                 limits, NULL);
  int64_t *sel = (int64_t *)malloc(sizeof(int64_t) * (cnt ? cnt : 1));
  tor_select_nodes(P->prm.nel, P->prm.dx, origin, center, radius, limits, sel);
  for (int64_t s = 0; s < cnt; s++) {
    int64_t n = sel[s];
    for (int c = 0; c < 3; c++) {
      if (type == 0) {
        if (values[c] != 0) P->fix[n] |= (uint8_t)(1u << c);
      } else {
        P->F[3 * n + c] += values[c];
      }
    }
  }
  free(sel);
  return cnt;
}

void tor_get_bc(const tor_problem *P, uint8_t *fixmask, double *F)
{
  if (fixmask) memcpy(fixmask, P->fix, P->nn);
  if (F) memcpy(F, P->F, sizeof(double) * 3 * P->nn);
}

void tor_set_design(tor_problem *P, const double *x, double penal, double eps)
{
  /* MatIntFnc (Material_Interpolation.cpp:20-75), vdMin <= 0 */
  memcpy(P->x, x, sizeof(double) * P->ne);
  tor_csr_mult(P->ne, P->frow, P->fcol, P->fval, P->x, P->rho);   /* :35 */
  tor_simp(P->ne, P->rho, penal, eps, P->E, P->dEdz, P->Es, NULL);
}

void tor_get_material(const tor_problem *P, double *rho, double *E, double *dEdz)
{
  if (rho) memcpy(rho, P->rho, sizeof(double) * P->ne);
  if (E) memcpy(E, P->E, sizeof(double) * P->ne);
  if (dEdz) memcpy(dEdz, P->dEdz, sizeof(double) * P->ne);
}

void tor_set_moduli(tor_problem *P, const double *E, const double *dEdz)
{
  memcpy(P->E, E, sizeof(double) * P->ne);
  if (dEdz) memcpy(P->dEdz, dEdz, sizeof(double) * P->ne);
}

void tor_filter(const tor_problem *P, const double *in, double *out, int transpose)
{
  if (transpose)
    tor_csr_mult_t(P->ne, P->ne, P->frow, P->fcol, P->fval, in, out);
  else
    tor_csr_mult(P->ne, P->frow, P->fcol, P->fval, in, out);
}

/* ---- FEAssemble ---------------------------------------------------------- */

static void assemble_fine(tor_problem *P, bsr3 *A)
{
  /* K = sum_e E_e K0 (FEAnalysis.cpp:443-468), summed per block in element
   * order as ADD_VALUES does; then MatZeroRowsColumns(fixed, 1.0) (:473) and
   * the non-positive diagonal fix (:476-484). */
  const int *nel = P->prm.nel;
  int64_t Nx = nel[0] + 1, Ny = nel[1] + 1, Nz = nel[2] + 1, nn = P->nn;
  A->n = nn;
  A->rowptr = (int64_t *)malloc(sizeof(int64_t) * (nn + 1));
  A->rowptr[0] = 0;
  for (int64_t n = 0; n < nn; n++) {
    int64_t i = n % Nx, j = (n / Nx) % Ny, k = n / (Nx * Ny);
    int cx = 1 + (i > 0) + (i < Nx - 1), cy = 1 + (j > 0) + (j < Ny - 1),
        cz = 1 + (k > 0) + (k < Nz - 1);
    A->rowptr[n + 1] = A->rowptr[n] + cx * cy * cz;
  }
  int64_t nb = A->rowptr[nn];
  A->col = (int32_t *)malloc(sizeof(int32_t) * nb);
  A->val = (double *)calloc(9 * nb, sizeof(double));
  const double *K0 = P->K0;
#pragma omp parallel for schedule(static)
  for (int64_t n = 0; n < nn; n++) {
    int64_t i = n % Nx, j = (n / Nx) % Ny, k = n / (Nx * Ny);
    int64_t t = A->rowptr[n];
    for (int dk = -1; dk <= 1; dk++)
      for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++) {
          int64_t mi = i + di, mj = j + dj, mk = k + dk;
          if (mi < 0 || mi >= Nx || mj < 0 || mj >= Ny || mk < 0 || mk >= Nz)
            continue;
          int64_t m = mi + mj * Nx + mk * Nx * Ny;
          A->col[t] = (int32_t)m;
          double *blk = A->val + 9 * t;
          /* elements containing both n and m, in increasing element order */
          for (int64_t ek = (k > mk ? k : mk) - 1; ek <= (k < mk ? k : mk); ek++)
            for (int64_t ej = (j > mj ? j : mj) - 1; ej <= (j < mj ? j : mj); ej++)
              for (int64_t ei = (i > mi ? i : mi) - 1; ei <= (i < mi ? i : mi); ei++) {
                if (ei < 0 || ej < 0 || ek < 0 || ei >= nel[0] || ej >= nel[1] ||
                    ek >= nel[2])
                  continue;
                int64_t e = ei + ej * nel[0] + ek * (int64_t)nel[0] * nel[1];
                int ln = (int)((i - ei) + 2 * (j - ej) + 4 * (k - ek));
                int lm = (int)((mi - ei) + 2 * (mj - ej) + 4 * (mk - ek));
                /* lexicographic corner -> reference local node number */
                static const int lex2loc[8] = {0, 1, 3, 2, 4, 5, 7, 6};
                int a = lex2loc[ln], b = lex2loc[lm];
                double Ee = P->E[e];
                for (int r = 0; r < 3; r++)
                  for (int c = 0; c < 3; c++)
                    blk[3 * r + c] += Ee * K0[24 * (3 * a + r) + 3 * b + c];
              }
          t++;
        }
  }
  /* Dirichlet rows and columns -> identity */
#pragma omp parallel for schedule(static)
  for (int64_t n = 0; n < nn; n++) {
    for (int64_t t = A->rowptr[n]; t < A->rowptr[n + 1]; t++) {
      int64_t m = A->col[t];
      double *blk = A->val + 9 * t;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
          int fr = (P->fix[n] >> r) & 1, fc = (P->fix[m] >> c) & 1;
          if (fr || fc) blk[3 * r + c] = (m == n && r == c) ? 1.0 : 0.0;
        }
      if (m == n)
        for (int r = 0; r < 3; r++)
          if (!(blk[4 * r] > 0)) blk[4 * r] = 1.0;
    }
  }
}

/* ---- GMG hierarchy -------------------------------------------------------- */

static void build_prolongation(const int fd[3], const int cd[3], csr *P)
{
  /* Create_Interpolation (Interpolation.cpp:123-169): coarse node at every
   * even fine index, weights (0.5, 1, 0.5)^3; row-normalised
   * (Interpolation.cpp:330-347).  Coarse numbering is lexicographic over the
   * coarse grid (the sort at Interpolation.cpp:210-214 on one rank). */
  int64_t nf = (int64_t)fd[0] * fd[1] * fd[2], nc = (int64_t)cd[0] * cd[1] * cd[2];
  P->nrow = nf;
  P->ncol = nc;
  P->rowptr = (int64_t *)malloc(sizeof(int64_t) * (nf + 1));
  P->col = (int32_t *)malloc(sizeof(int32_t) * nf * 8);
  P->val = (double *)malloc(sizeof(double) * nf * 8);
  int64_t t = 0;
  P->rowptr[0] = 0;
  for (int64_t f = 0; f < nf; f++) {
    int fi[3] = {(int)(f % fd[0]), (int)((f / fd[0]) % fd[1]),
                 (int)(f / ((int64_t)fd[0] * fd[1]))};
    int cand[3][2], nc1[3];
    double w1[3][2];
    for (int d = 0; d < 3; d++) {
      nc1[d] = 0;
      /* coarse nodes 2c within distance 1 of fi */
      for (int c = (fi[d] - 1 + 1) / 2; 2 * c <= fi[d] + 1; c++) {
        if (c < 0 || c >= cd[d] || 2 * c > fd[d] - 1) continue;
        if (2 * c < fi[d] - 1) continue;
        cand[d][nc1[d]] = c;
        w1[d][nc1[d]] = (2 * c == fi[d]) ? 1.0 : 0.5;
        nc1[d]++;
      }
    }
    double rs = 0;
    int64_t start = t;
    for (int a = 0; a < nc1[2]; a++)
      for (int b = 0; b < nc1[1]; b++)
        for (int c = 0; c < nc1[0]; c++) {
          P->col[t] = (int32_t)(cand[0][c] + (int64_t)cand[1][b] * cd[0] +
                                (int64_t)cand[2][a] * cd[0] * cd[1]);
          P->val[t] = w1[0][c] * w1[1][b] * w1[2][a];
          rs += P->val[t];
          t++;
        }
    double inv = 1.0 / rs;
    for (int64_t s = start; s < t; s++) P->val[s] *= inv;
    P->rowptr[f + 1] = t;
  }
}

static void csr_transpose(const csr *A, csr *T)
{
  T->nrow = A->ncol;
  T->ncol = A->nrow;
  int64_t nnz = A->rowptr[A->nrow];
  T->rowptr = (int64_t *)calloc(T->nrow + 1, sizeof(int64_t));
  T->col = (int32_t *)malloc(sizeof(int32_t) * nnz);
  T->val = (double *)malloc(sizeof(double) * nnz);
  for (int64_t t = 0; t < nnz; t++) T->rowptr[A->col[t] + 1]++;
  for (int64_t r = 0; r < T->nrow; r++) T->rowptr[r + 1] += T->rowptr[r];
  int64_t *pos = (int64_t *)malloc(sizeof(int64_t) * T->nrow);
  memcpy(pos, T->rowptr, sizeof(int64_t) * T->nrow);
  for (int64_t r = 0; r < A->nrow; r++)
    for (int64_t t = A->rowptr[r]; t < A->rowptr[r + 1]; t++) {
      int64_t p = pos[A->col[t]]++;
      T->col[p] = (int32_t)r;
      T->val[p] = A->val[t];
    }
  free(pos);
}

static int cmp_i32(const void *a, const void *b)
{
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* Ac = P^T A P (PCMG Galerkin, FEAnalysis.cpp:412); Gustavson row-wise with
 * a dense marker per thread. */
static void galerkin(const bsr3 *A, const csr *P, const csr *PT, bsr3 *Ac)
{
  int64_t nc = P->ncol;
  Ac->n = nc;
  Ac->rowptr = (int64_t *)calloc(nc + 1, sizeof(int64_t));
  int32_t **rc = (int32_t **)malloc(sizeof(int32_t *) * nc);
  double **rv = (double **)malloc(sizeof(double *) * nc);
  int *rn = (int *)calloc(nc, sizeof(int));
#pragma omp parallel
  {
    int64_t *mark = (int64_t *)malloc(sizeof(int64_t) * nc);
    for (int64_t q = 0; q < nc; q++) mark[q] = -1;
    int32_t cols[512];
    double acc[512 * 9];
#pragma omp for schedule(dynamic, 64)
    for (int64_t I = 0; I < nc; I++) {
      int cnt = 0;
      for (int64_t s = PT->rowptr[I]; s < PT->rowptr[I + 1]; s++) {
        int64_t f = PT->col[s];
        double wf = PT->val[s];
        for (int64_t t = A->rowptr[f]; t < A->rowptr[f + 1]; t++) {
          int64_t g = A->col[t];
          const double *blk = A->val + 9 * t;
          for (int64_t u = P->rowptr[g]; u < P->rowptr[g + 1]; u++) {
            int64_t J = P->col[u];
            double w = wf * P->val[u];
            int64_t slot = mark[J];
            if (slot < 0 || slot >= cnt || cols[slot] != J) {
              slot = cnt++;
              mark[J] = slot;
              cols[slot] = (int32_t)J;
              memset(acc + 9 * slot, 0, 9 * sizeof(double));
            }
            for (int q = 0; q < 9; q++) acc[9 * slot + q] += w * blk[q];
          }
        }
      }
      /* sort the row by column */
      int32_t sorted[512];
      memcpy(sorted, cols, sizeof(int32_t) * cnt);
      qsort(sorted, cnt, sizeof(int32_t), cmp_i32);
      rc[I] = (int32_t *)malloc(sizeof(int32_t) * cnt);
      rv[I] = (double *)malloc(sizeof(double) * 9 * cnt);
      for (int q = 0; q < cnt; q++) {
        int32_t J = sorted[q];
        rc[I][q] = J;
        memcpy(rv[I] + 9 * q, acc + 9 * mark[J], 9 * sizeof(double));
      }
      rn[I] = cnt;
      for (int q = 0; q < cnt; q++) mark[cols[q]] = -1;
    }
    free(mark);
  }
  for (int64_t I = 0; I < nc; I++) Ac->rowptr[I + 1] = Ac->rowptr[I] + rn[I];
  int64_t nb = Ac->rowptr[nc];
  Ac->col = (int32_t *)malloc(sizeof(int32_t) * nb);
  Ac->val = (double *)malloc(sizeof(double) * 9 * nb);
  for (int64_t I = 0; I < nc; I++) {
    memcpy(Ac->col + Ac->rowptr[I], rc[I], sizeof(int32_t) * rn[I]);
    memcpy(Ac->val + 9 * Ac->rowptr[I], rv[I], sizeof(double) * 9 * rn[I]);
    free(rc[I]);
    free(rv[I]);
  }
  free(rc); free(rv); free(rn);
}

static double vdot(int64_t n, const double *a, const double *b)
{
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* deterministic start vector for the power iteration: splitmix64 of the
 * dof index mapped to [-1, 1) */
static double start_value(uint64_t i)
{
  uint64_t z = i + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

static double estimate_lambda(const level_t *v, int its)
{
  int64_t n = 3 * v->nn;
  double *a = (double *)malloc(sizeof(double) * n);
  double *w = (double *)malloc(sizeof(double) * n);
  for (int64_t i = 0; i < n; i++) a[i] = start_value((uint64_t)i);
  double nrm = sqrt(vdot(n, a, a));
  for (int64_t i = 0; i < n; i++) a[i] /= nrm;
  double lam = 0;
  for (int k = 0; k < its; k++) {
    bsr_mult(&v->A, a, w);
    for (int64_t i = 0; i < n; i++) w[i] *= v->dinv[i];
    lam = sqrt(vdot(n, w, w));
    for (int64_t i = 0; i < n; i++) a[i] = w[i] / lam;
  }
  free(a);
  free(w);
  return lam;
}

int tor_assemble(tor_problem *P, const tor_solve_opts *o)
{
  free_levels(P);
  P->opts = *o;
  int L = P->L;
  int dims[3] = {P->prm.nel[0] + 1, P->prm.nel[1] + 1, P->prm.nel[2] + 1};
  for (int l = 0; l < L; l++) {
    level_t *v = &P->lev[l];
    memcpy(v->dims, dims, sizeof(dims));
    v->nn = (int64_t)dims[0] * dims[1] * dims[2];
    for (int d = 0; d < 3; d++) dims[d] = (dims[d] + 1) / 2;
  }
  assemble_fine(P, &P->lev[0].A);
  for (int l = 0; l + 1 < L; l++) {
    build_prolongation(P->lev[l].dims, P->lev[l + 1].dims, &P->lev[l].P);
    csr_transpose(&P->lev[l].P, &P->lev[l].PT);
    galerkin(&P->lev[l].A, &P->lev[l].P, &P->lev[l].PT, &P->lev[l + 1].A);
  }
  for (int l = 0; l < L; l++) {
    level_t *v = &P->lev[l];
    int64_t n = 3 * v->nn;
    v->dinv = (double *)malloc(sizeof(double) * n);
    for (int64_t r = 0; r < v->nn; r++) {
      const double *d = bsr_find(&v->A, r, r);
      for (int c = 0; c < 3; c++) v->dinv[3 * r + c] = 1.0 / d[4 * c];
    }
    v->b = (double *)calloc(n, sizeof(double));
    v->x = (double *)calloc(n, sizeof(double));
    v->r = (double *)calloc(n, sizeof(double));
    v->t1 = (double *)calloc(n, sizeof(double));
    v->t2 = (double *)calloc(n, sizeof(double));
    if (l + 1 < L) v->lam = estimate_lambda(v, o->power_its);
  }
  /* coarsest: dense Cholesky (the reference uses BJacobi + LU,
   * FEAnalysis.cpp:555-573; the operator is SPD) */
  level_t *c = &P->lev[L - 1];
  int64_t nc = 3 * c->nn;
  P->nc = nc;
  P->chol = (double *)calloc(nc * nc, sizeof(double));
  for (int64_t r = 0; r < c->nn; r++)
    for (int64_t t = c->A.rowptr[r]; t < c->A.rowptr[r + 1]; t++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          P->chol[(3 * r + a) * nc + 3 * (int64_t)c->A.col[t] + b] =
              c->A.val[9 * t + 3 * a + b];
  double *Lm = P->chol;
  for (int64_t j = 0; j < nc; j++) {
    double s = Lm[j * nc + j];
    for (int64_t k = 0; k < j; k++) s -= Lm[j * nc + k] * Lm[j * nc + k];
    if (!(s > 0)) return -1;
    double d = sqrt(s);
    Lm[j * nc + j] = d;
#pragma omp parallel for schedule(static)
    for (int64_t i = j + 1; i < nc; i++) {
      double t = Lm[i * nc + j];
      for (int64_t k = 0; k < j; k++) t -= Lm[i * nc + k] * Lm[j * nc + k];
      Lm[i * nc + j] = t / d;
    }
  }
  P->assembled = 1;
  return 0;
}

void tor_apply(const tor_problem *P, const double *u, double *y)
{
  bsr_mult(&P->lev[0].A, u, y);
}

void tor_apply_level(const tor_problem *P, int level, const double *u, double *y)
{
  bsr_mult(&P->lev[level].A, u, y);
}

int64_t tor_level_nodes(const tor_problem *P, int level, int dims[3])
{
  if (dims) memcpy(dims, P->lev[level].dims, 3 * sizeof(int));
  return P->lev[level].nn;
}

int tor_level_block(const tor_problem *P, int level, int64_t i, int64_t j,
                    double blk[9])
{
  const double *b = bsr_find(&P->lev[level].A, i, j);
  if (!b) { memset(blk, 0, 9 * sizeof(double)); return 0; }
  memcpy(blk, b, 9 * sizeof(double));
  return 1;
}

double tor_level_lambda(const tor_problem *P, int level)
{
  return P->lev[level].lam;
}

double tor_prolong_weight(const tor_problem *P, int level, int64_t f, int64_t c)
{
  const csr *A = &P->lev[level].P;
  for (int64_t t = A->rowptr[f]; t < A->rowptr[f + 1]; t++)
    if (A->col[t] == c) return A->val[t];
  return 0.0;
}

/* ---- smoother, V-cycle, PCG ----------------------------------------------- */

static void coarse_solve(const tor_problem *P, const double *b, double *x)
{
  int64_t n = P->nc;
  const double *Lm = P->chol;
  for (int64_t i = 0; i < n; i++) {
    double s = b[i];
    for (int64_t k = 0; k < i; k++) s -= Lm[i * n + k] * x[k];
    x[i] = s / Lm[i * n + i];
  }
  for (int64_t i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int64_t k = i + 1; k < n; k++) s -= Lm[k * n + i] * x[k];
    x[i] = s / Lm[i * n + i];
  }
}

/* Chebyshev semi-iteration with Jacobi preconditioning (Saad, Iterative
 * Methods for Sparse Linear Systems, Alg. 12.1), interval [lo, hi]*lambda.
 * x holds the initial guess; zero_guess skips the first residual apply. */
static void chebyshev(level_t *v, const tor_solve_opts *o, const double *b,
                      double *x, int zero_guess)
{
  int64_t n = 3 * v->nn;
  double a = o->cheb_lo * v->lam, bb = o->cheb_hi * v->lam;
  double theta = 0.5 * (bb + a), delta = 0.5 * (bb - a), sigma = theta / delta;
  double rho = 1.0 / sigma;
  double *r = v->t1, *d = v->t2, *Ad = v->r;
  if (zero_guess) {
    for (int64_t i = 0; i < n; i++) { x[i] = 0; r[i] = v->dinv[i] * b[i]; }
  } else {
    bsr_mult(&v->A, x, Ad);
    for (int64_t i = 0; i < n; i++) r[i] = v->dinv[i] * (b[i] - Ad[i]);
  }
  for (int64_t i = 0; i < n; i++) d[i] = r[i] / theta;
  for (int k = 0; k < o->cheb_degree; k++) {
    for (int64_t i = 0; i < n; i++) x[i] += d[i];
    if (k + 1 == o->cheb_degree) break;
    bsr_mult(&v->A, d, Ad);
    double rn = 1.0 / (2.0 * sigma - rho);
    for (int64_t i = 0; i < n; i++) {
      r[i] -= v->dinv[i] * Ad[i];
      d[i] = rn * rho * d[i] + (2.0 * rn / delta) * r[i];
    }
    rho = rn;
  }
}

static void vcycle(tor_problem *P, int l, const double *b, double *x)
{
  level_t *v = &P->lev[l];
  if (l == P->L - 1) { coarse_solve(P, b, x); return; }
  int64_t n = 3 * v->nn;
  level_t *c = &P->lev[l + 1];
  chebyshev(v, &P->opts, b, x, 1);                       /* pre-smooth */
  double *res = v->r;
  bsr_mult(&v->A, x, res);
  for (int64_t i = 0; i < n; i++) res[i] = b[i] - res[i];
  /* restrict: b_c = P^T r (MatRestrict) */
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < c->nn; I++) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t t = v->PT.rowptr[I]; t < v->PT.rowptr[I + 1]; t++) {
      int64_t f = v->PT.col[t];
      double w = v->PT.val[t];
      s0 += w * res[3 * f]; s1 += w * res[3 * f + 1]; s2 += w * res[3 * f + 2];
    }
    c->b[3 * I] = s0; c->b[3 * I + 1] = s1; c->b[3 * I + 2] = s2;
  }
  vcycle(P, l + 1, c->b, c->x);
  /* prolong-add: x += P x_c (MatInterpolateAdd) */
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < v->nn; f++) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t t = v->P.rowptr[f]; t < v->P.rowptr[f + 1]; t++) {
      int64_t I = v->P.col[t];
      double w = v->P.val[t];
      s0 += w * c->x[3 * I]; s1 += w * c->x[3 * I + 1]; s2 += w * c->x[3 * I + 2];
    }
    x[3 * f] += s0; x[3 * f + 1] += s1; x[3 * f + 2] += s2;
  }
  chebyshev(v, &P->opts, b, x, 0);                       /* post-smooth */
}

void tor_vcycle(tor_problem *P, const double *r, double *z)
{
  vcycle(P, 0, r, z);
}

int tor_solve_rhs(tor_problem *P, const tor_solve_opts *o, const double *b,
                  double *U, int *its, double *relres)
{
  /* KSPCG with KSP_NORM_UNPRECONDITIONED and a nonzero initial guess
   * (FEAnalysis.cpp:387-395), converged when ||r|| <= rtol ||b||. */
  P->opts.maxit = o->maxit;
  P->opts.rtol = o->rtol;
  int64_t n = 3 * P->nn;
  double *r = (double *)malloc(sizeof(double) * n);
  double *z = (double *)malloc(sizeof(double) * n);
  double *p = (double *)malloc(sizeof(double) * n);
  double *q = (double *)malloc(sizeof(double) * n);
  double bn = sqrt(vdot(n, b, b));
  int status = 1, k = 0;
  double rn = 0, rho_old = 0;
  if (bn == 0) {
    memset(U, 0, sizeof(double) * n);
    status = 0;
    goto done;
  }
  bsr_mult(&P->lev[0].A, U, r);
  for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
  rn = sqrt(vdot(n, r, r));
  if (rn <= o->rtol * bn) { status = 0; goto done; }
  for (k = 0; k < o->maxit;) {
    vcycle(P, 0, r, z);
    double rho = vdot(n, r, z);
    if (!(rho > 0)) { status = -1; break; }
    if (k == 0) memcpy(p, z, sizeof(double) * n);
    else {
      double beta = rho / rho_old;
      for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    rho_old = rho;
    bsr_mult(&P->lev[0].A, p, q);
    double pq = vdot(n, p, q);
    if (!(pq > 0)) { status = -1; break; }
    double alpha = rho / pq;
    for (int64_t i = 0; i < n; i++) { U[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
    k++;
    rn = sqrt(vdot(n, r, r));
    if (!isfinite(rn)) { status = -1; break; }
    if (rn <= o->rtol * bn) { status = 0; break; }
  }
done:
  if (its) *its = k;
  if (relres) *relres = bn > 0 ? rn / bn : 0.0;
  free(r); free(z); free(p); free(q);
  return status;
}

int tor_solve(tor_problem *P, const tor_solve_opts *o, double *U, int *its,
              double *relres)
{
  return tor_solve_rhs(P, o, P->F, U, its, relres);
}

/* ---- functions -------------------------------------------------------------- */

void tor_compliance(const tor_problem *P, const double *U, double *C,
                    double *dCdx, double *dCdrho)
{
  /* Compliance.cpp:19 and :37-46, then Chain_Filter (:51) with vdMin <= 0,
   * which reduces to P^T (Material_Interpolation.cpp:165-181). */
  int64_t n = 3 * P->nn;
  double c = 0;
  for (int64_t i = 0; i < n; i++) c += U[i] * P->F[i];
  if (C) *C = c;
  if (!dCdx && !dCdrho) return;
  double *g = (double *)malloc(sizeof(double) * P->ne);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < P->ne; e++) {
    int64_t nodes[8];
    double ue[24], s = 0;
    tor_element_nodes(P->prm.nel, e, nodes);
    for (int a = 0; a < 8; a++)
      for (int d = 0; d < 3; d++) ue[3 * a + d] = U[3 * nodes[a] + d];
    for (int r = 0; r < 24; r++) {
      double t = 0;
      for (int q = 0; q < 24; q++) t += P->K0[24 * r + q] * ue[q];
      s += ue[r] * t;
    }
    g[e] = -P->dEdz[e] * s;
  }
  if (dCdrho) memcpy(dCdrho, g, sizeof(double) * P->ne);
  if (dCdx) tor_csr_mult_t(P->ne, P->ne, P->frow, P->fcol, P->fval, g, dCdx);
  free(g);
}

void tor_volume(const tor_problem *P, double *V, double *dVdx)
{
  /* Volume.cpp:75-91: V = sum(rho)/nElem, dV = P^T (dVdrho / nElem) */
  double s = 0;
  for (int64_t e = 0; e < P->ne; e++) s += P->rho[e];
  if (V) *V = s / (double)P->ne;
  if (dVdx) {
    double *g = (double *)malloc(sizeof(double) * P->ne);
    for (int64_t e = 0; e < P->ne; e++) g[e] = 1.0 * (1.0 / (double)P->ne);
    tor_csr_mult_t(P->ne, P->ne, P->frow, P->fcol, P->fval, g, dVdx);
    free(g);
  }
}

double tor_oc_update(int64_t n, double *x, const double *xmin, const double *xmax,
                     double *dfdx, double g, const double *dgdx, double move)
{
  /* MMA::OCsub (MMA.cpp:103-180) with OCeta = 0.5 (MMA.cpp:87-90) */
  double *xold = (double *)malloc(sizeof(double) * n);
  memcpy(xold, x, sizeof(double) * n);
  double l1 = 0, l2 = 1e6;
  while (l2 - l1 > 1e-4) {
    double lmid = 0.5 * (l1 + l2);
    double dg = 0;
    for (int64_t i = 0; i < n; i++) {
      if (dfdx[i] > 0) dfdx[i] = 0;
      double B = pow(-dfdx[i] / dgdx[i] / lmid, 0.5);
      double xc = xmin[i] + (xold[i] - xmin[i]) * B;
      double step = move * (xmax[i] - xmin[i]);
      double v = xc;
      if (v > xold[i] + step) v = xold[i] + step;
      if (v > xmax[i]) v = xmax[i];
      if (v < xold[i] - step) v = xold[i] - step;
      if (v < xmin[i]) v = xmin[i];
      x[i] = v;
      dg += dgdx[i] * (v - xold[i]);
    }
    if (g + dg > 0) l1 = lmid; else l2 = lmid;
  }
  /* small values are zeroed before Change is measured (MMA.cpp:166-173) */
  for (int64_t i = 0; i < n; i++)
    if (x[i] < 1e-6) x[i] = 0;
  double change = 0;
  for (int64_t i = 0; i < n; i++) {
    double c = fabs((x[i] - xold[i]) / (xmax[i] - xmin[i]));
    if (c > change) change = c;
  }
  free(xold);
  return change;
}

/* ------------------------------------------------------------------------ */
/* stress stiffness (buckling)                                               */
/* ------------------------------------------------------------------------ */

void tor_stress_stiffness_element(const double dx[3], double E0, double nu,
                                  const double u[24], double ks[576])
{
  /* Stability::StressFnc (Buckling.cpp:313-327): ks = sum_q W_q G_q^T
   * sigtos(d B_q u) G_q detJ, with G from TopOpt::AssignG
   * (FEAnalysis.cpp:1062-1081): row 3i + j, column 3n + i holds dN_n/dx_j,
   * i.e. G u stacks the gradients of the three displacement components;
   * sigtos (Buckling.cpp:371-414) repeats the 3x3 stress tensor of the
   * Voigt vector [xx, yy, zz, xy, yz, xz] on the diagonal.  u is in the
   * reference's local node order (dN, FEAnalysis.cpp:955-986). */
  double D[36];
  tor_constitutive(E0, nu, D);
  double coords[8][3];
  for (int n = 0; n < 8; n++)
    for (int d = 0; d < 3; d++) coords[n][d] = kNodeSign[n][d] > 0 ? dx[d] : 0.0;
  memset(ks, 0, 576 * sizeof(double));
  const double g = 1.0 / sqrt(3.0);
  for (int q = 0; q < 8; q++) {
    double xi = kNodeSign[q][0] * g, eta = kNodeSign[q][1] * g,
           zeta = kNodeSign[q][2] * g;
    double dNdxi[3][8];
    for (int n = 0; n < 8; n++) {
      double a = kNodeSign[n][0], b = kNodeSign[n][1], c = kNodeSign[n][2];
      dNdxi[0][n] = a * (1 + b * eta) * (1 + c * zeta) / 8.0;
      dNdxi[1][n] = b * (1 + a * xi) * (1 + c * zeta) / 8.0;
      dNdxi[2][n] = c * (1 + a * xi) * (1 + b * eta) / 8.0;
    }
    double J[9] = {0}, iJ[9];
    for (int r = 0; r < 3; r++)
      for (int cc = 0; cc < 3; cc++)
        for (int n = 0; n < 8; n++) J[3 * r + cc] += dNdxi[r][n] * coords[n][cc];
    double detJ = det3(J);
    inv3(J, iJ);
    double dNdx[3][8];
    for (int r = 0; r < 3; r++)
      for (int n = 0; n < 8; n++) {
        double t = 0;
        for (int k = 0; k < 3; k++) t += iJ[3 * r + k] * dNdxi[k][n];
        dNdx[r][n] = t;
      }
    /* B (AssignB, FEAnalysis.cpp:1024-1046) and sigma = d B u */
    double B[6][24];
    memset(B, 0, sizeof(B));
    for (int n = 0; n < 8; n++) {
      B[0][3 * n] = dNdx[0][n];
      B[1][3 * n + 1] = dNdx[1][n];
      B[2][3 * n + 2] = dNdx[2][n];
      B[3][3 * n] = dNdx[1][n];
      B[3][3 * n + 1] = dNdx[0][n];
      B[4][3 * n + 1] = dNdx[2][n];
      B[4][3 * n + 2] = dNdx[1][n];
      B[5][3 * n] = dNdx[2][n];
      B[5][3 * n + 2] = dNdx[0][n];
    }
    double eps_v[6], sig[6];
    for (int r = 0; r < 6; r++) {
      double t = 0;
      for (int c = 0; c < 24; c++) t += B[r][c] * u[c];
      eps_v[r] = t;
    }
    for (int r = 0; r < 6; r++) {
      double t = 0;
      for (int k = 0; k < 6; k++) t += D[6 * r + k] * eps_v[k];
      sig[r] = t;
    }
    /* sigtos */
    double S[9][9];
    memset(S, 0, sizeof(S));
    double s3[3][3] = {{sig[0], sig[3], sig[5]},
                       {sig[3], sig[1], sig[4]},
                       {sig[5], sig[4], sig[2]}};
    for (int b = 0; b < 3; b++)
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) S[3 * b + r][3 * b + c] = s3[r][c];
    /* G (AssignG) */
    double G[9][24];
    memset(G, 0, sizeof(G));
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int n = 0; n < 8; n++) G[3 * i + j][3 * n + i] = dNdx[j][n];
    double SG[9][24];
    for (int r = 0; r < 9; r++)
      for (int c = 0; c < 24; c++) {
        double t = 0;
        for (int k = 0; k < 9; k++) t += S[r][k] * G[k][c];
        SG[r][c] = t;
      }
    for (int r = 0; r < 24; r++)
      for (int c = 0; c < 24; c++) {
        double t = 0;
        for (int k = 0; k < 9; k++) t += G[k][r] * SG[k][c];
        ks[24 * r + c] += t * detJ;   /* W[q] = 1 */
      }
  }
}

void tor_ks_assemble(tor_problem *P, const double *U)
{
  /* Ks = sum_e -Es_e ks_e (Buckling.cpp:329-352, Es without E_min, :343),
   * then MatZeroRowsColumns(Ks, fixedDof, 0.0) (:29-30).  Same block
   * pattern as K; elements are visited in 8 parity classes so that the
   * elements of one class touch disjoint blocks (parallel without races). */
  const int *nel = P->prm.nel;
  int64_t Nx = nel[0] + 1, Ny = nel[1] + 1, Nz = nel[2] + 1, nn = P->nn;
  bsr3 *A = &P->Ks;
  bsr_free(A);
  A->n = nn;
  A->rowptr = (int64_t *)malloc(sizeof(int64_t) * (nn + 1));
  A->rowptr[0] = 0;
  for (int64_t n = 0; n < nn; n++) {
    int64_t i = n % Nx, j = (n / Nx) % Ny, k = n / (Nx * Ny);
    int cx = 1 + (i > 0) + (i < Nx - 1), cy = 1 + (j > 0) + (j < Ny - 1),
        cz = 1 + (k > 0) + (k < Nz - 1);
    A->rowptr[n + 1] = A->rowptr[n] + cx * cy * cz;
  }
  A->col = (int32_t *)malloc(sizeof(int32_t) * A->rowptr[nn]);
  A->val = (double *)calloc(9 * (size_t)A->rowptr[nn], sizeof(double));
  for (int64_t n = 0; n < nn; n++) {
    int64_t i = n % Nx, j = (n / Nx) % Ny, k = n / (Nx * Ny);
    int64_t t = A->rowptr[n];
    for (int dk = -1; dk <= 1; dk++)
      for (int dj = -1; dj <= 1; dj++)
        for (int di = -1; di <= 1; di++) {
          int64_t mi = i + di, mj = j + dj, mk = k + dk;
          if (mi < 0 || mi >= Nx || mj < 0 || mj >= Ny || mk < 0 || mk >= Nz)
            continue;
          A->col[t++] = (int32_t)(mi + mj * Nx + mk * Nx * Ny);
        }
  }
  for (int color = 0; color < 8; color++) {
    int pi = color & 1, pj = (color >> 1) & 1, pk = (color >> 2) & 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ek = pk; ek < nel[2]; ek += 2)
      for (int64_t ej = pj; ej < nel[1]; ej += 2)
        for (int64_t ei = pi; ei < nel[0]; ei += 2) {
          int64_t e = ei + ej * nel[0] + ek * (int64_t)nel[0] * nel[1];
          int64_t nodes[8];
          tor_element_nodes(nel, e, nodes);
          double u[24], ks[576];
          for (int a = 0; a < 8; a++)
            for (int d = 0; d < 3; d++) u[3 * a + d] = U[3 * nodes[a] + d];
          tor_stress_stiffness_element(P->prm.dx, P->prm.E0, P->prm.nu, u, ks);
          double w = -P->Es[e];
          for (int a = 0; a < 8; a++)
            for (int b = 0; b < 8; b++) {
              double *blk = (double *)bsr_find(A, nodes[a], nodes[b]);
              for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++)
                  blk[3 * r + c] += w * ks[24 * (3 * a + r) + 3 * b + c];
            }
        }
  }
#pragma omp parallel for schedule(static)
  for (int64_t n = 0; n < nn; n++)
    for (int64_t t = A->rowptr[n]; t < A->rowptr[n + 1]; t++) {
      int64_t m = A->col[t];
      double *blk = A->val + 9 * t;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
          if (((P->fix[n] >> r) & 1) || ((P->fix[m] >> c) & 1)) blk[3 * r + c] = 0.0;
    }
}

void tor_ks_apply(const tor_problem *P, const double *u, double *y)
{
  bsr_mult(&P->Ks, u, y);
}

void tor_get_es(const tor_problem *P, double *Es)
{
  memcpy(Es, P->Es, sizeof(double) * P->ne);
}
