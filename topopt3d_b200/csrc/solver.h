// Host-side solver entry points shared by the C ABI layer.
#pragma once

#include "tpo_internal.h"

namespace tpo {

void invalidate_graphs(Ctx &c);
int estimate_lambda(Ctx &c, int level, int its, double *lam);
int setup_hierarchy(Ctx &c, const tpo_solve_opts &o);
int vcycle_apply(Ctx &c, const tpo_solve_opts &o, int precision,
                 const double *r, double *z);
int vcycle_block(Ctx &c, const tpo_solve_opts &o, int precision, int nb);
// z = V-cycle(r) on nb <= kMaxBatch columns (FP64 or FP32 arithmetic)
int vcycle_cols(Ctx &c, const tpo_solve_opts &o, int precision, const double *r,
                double *z, int nb);
// room for nb columns in the level and solver work vectors (capi.cu)
int ensure_columns(Ctx &c, int nb);
// the nev largest eigenvalues of A phi = lambda K phi (eigen.cu): A = Ks,
// or diag(adiag) when adiag (3 nn, device) is given
int buckling(Ctx &c, const tpo_eig_opts &o, double *lambda, double *phi,
             int phi_mem, tpo_eig_info *info, const double *adiag = nullptr);
// Frequency::Function: lumped mass, eigenpairs, value and gradient (eigen.cu)
int frequency(Ctx &c, int nvals, double density, const double *mlump,
              const tpo_eig_opts &o, double p, double *lambda, int *nconv,
              double *mdiag, double *phi, double *g, double *dvdx, double *value,
              tpo_eig_info *info);
// gradient of the aggregated buckling value (eigen.cu)
int buckling_sensitivity(Ctx &c, int nev, const double *lam, const double *phi, double p,
                         const tpo_solve_opts &o, double *rhs, double *v, double *W,
                         double *g, double *dvdx, double *value, tpo_solve_info *info);
int solve(Ctx &c, const tpo_solve_opts &o, const double *b, double *x,
          tpo_solve_info *info, int nb = 1, tpo_solve_info *col = nullptr);

}  // namespace tpo
