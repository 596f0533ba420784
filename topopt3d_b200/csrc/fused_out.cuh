// Input and epilogue forms shared by the level-1 operator kernels (the
// half-stored stencil, kernels_mg.cu; the tensor-core form, kernels_l1tc.cu).
// They match the fine-level kernel's (kernels_apply_staged.cu, finish_dof):
// IN_U reads u, IN_CHEB forms the Chebyshev start invtheta D^-1 b on the
// fly; OUT_Y / OUT_RESID / OUT_CHEB2 / OUT_POST0 / OUT_POST1 write Au,
// b - Au or the fused Chebyshev(2) updates.
#pragma once

#include "tpo_internal.h"

namespace tpo {

template <typename T, int IN>
__device__ __forceinline__ T sym_in(const ApplyArgs<T> &a, int i) {
  if (IN == IN_CHEB) return a.invtheta * (a.dinv[i] * a.b[i]);
  return a.u[i];
}

// the epilogue on values already loaded: bi = b[i], di = dinv[i],
// y2i = y2[i] (each read only by the forms that use it)
template <typename T, int OUT>
__device__ __forceinline__ void sym_out_v(const ApplyArgs<T> &a, int i, T Au, T u, T bi,
                                          T di, T y2i) {
  if (OUT == OUT_Y) {
    a.y[i] = Au;
  } else if (OUT == OUT_RESID) {
    a.y[i] = bi - Au;
  } else if (OUT == OUT_CHEB2) {
    const T r1 = di * bi - di * Au;
    a.y[i] = u + (a.c1 * u + a.c2 * r1);
  } else if (OUT == OUT_POST0) {
    const T d0 = a.invtheta * (di * (bi - Au));
    a.y[i] = d0;
    a.y2[i] = u + d0;
  } else {   // OUT_POST1
    const T r1 = a.theta * u - di * Au;
    a.y[i] = y2i + (a.c1 * u + a.c2 * r1);
  }
}

template <int OUT>
struct OutNeeds {
  static constexpr bool b = OUT == OUT_RESID || OUT == OUT_CHEB2 || OUT == OUT_POST0;
  static constexpr bool dinv = OUT == OUT_CHEB2 || OUT == OUT_POST0 || OUT == OUT_POST1;
  static constexpr bool y2 = OUT == OUT_POST1;
};

template <typename T, int OUT>
__device__ __forceinline__ void sym_out(const ApplyArgs<T> &a, int i, T Au, T u) {
  sym_out_v<T, OUT>(a, i, Au, u, OutNeeds<OUT>::b ? a.b[i] : T(0),
                    OutNeeds<OUT>::dinv ? a.dinv[i] : T(0), OutNeeds<OUT>::y2 ? a.y2[i] : T(0));
}

}  // namespace tpo
