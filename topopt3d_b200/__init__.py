"""B200-native finite-element hot path of darinpeetz/TopOpt3D.

The GPU library (``libtopopt_b200.so``, C ABI in ``include/topopt_b200.h``)
implements the SIMP hex8 stiffness apply, the GMG-preconditioned CG solve
(FP64 and mixed FP32/FP64), the compliance sensitivity and the density
filter.  ``TopOpt`` mirrors the reference's call surface.
"""
from ._lib import (BC_LOAD, BC_SUPPORT, MEM_DEVICE, MEM_HOST, PREC_FP64,
                   PREC_MIXED, EigInfo, EigOpts, SolveInfo, SolveOpts,
                   default_eig_opts, default_opts, load)
from .topopt import (MMA, OC, Compliance, Frequency, Function_Base, Stability, TopOpt,
                     TopOptError, Volume, optimize)

__all__ = ["TopOpt", "TopOptError", "MMA", "Compliance", "Volume", "Frequency", "Function_Base",
           "OC", "optimize", "Stability", "EigOpts", "EigInfo",
           "default_eig_opts", "SolveOpts", "SolveInfo", "default_opts", "load",
           "PREC_FP64", "PREC_MIXED", "MEM_HOST", "MEM_DEVICE", "BC_SUPPORT",
           "BC_LOAD"]
