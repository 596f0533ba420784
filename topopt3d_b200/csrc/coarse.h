// Parameters of the persistent coarse-grid V-cycle kernel (kernels_coarse.cu).
#pragma once

#include "tpo_internal.h"

namespace tpo {

constexpr int kCoarseThreads = 256;
constexpr int kMaxChebDegree = 8;
constexpr int kMaxCoarseLevels = 8;
// levels with at most this many nodes run inside the persistent kernel
constexpr int64_t kPersistentMaxNodes = 65536;

// Every vector below holds `nb` columns (CoarseCycle::nb), column j at
// offset j * 3 * nn; A and dinv are shared by the columns.
template <typename T>
struct CoarseLevel {
  int dims[3];
  int64_t nn;
  const T *A;      // the Galerkin stencil, node-major: A[n*243 + (3r+s)*27 + nb]
  const T *dinv;   // 1 / diag
  T *b;            // right-hand side (restricted residual of the parent)
  T *xpre;         // pre-smoothed iterate, then + P x_child
  T *xout;         // post-smoothed result (read by the parent)
  T *r, *d0, *d1;  // Chebyshev residual and ping-pong directions
  T *res;          // b - A xpre
  T inv_theta;
  T c1[kMaxChebDegree], c2[kMaxChebDegree];
  int deg;
};

template <typename T>
struct CoarseCycle {
  int nlev;                          // stencil levels handled in the kernel
  int nb;                            // columns (1, 2, 4 or 8)
  CoarseLevel<T> lev[kMaxCoarseLevels];
  const double *Ainv;                // dense inverse of the coarsest operator
  int64_t nc;                        // coarsest dof count
  int cdims[3];                      // coarsest nodes per dimension
  T *bc, *xc;                        // coarsest right-hand side / solution
                                     // (column stride nc)
  unsigned int *bar;                 // grid-barrier counter (zero between
                                     // launches)
  double *fault;                     // set to 1 when a barrier wait runs out
};

template <typename T>
cudaError_t launch_coarse_cycle(const CoarseCycle<T> &P, cudaStream_t s);

}  // namespace tpo
