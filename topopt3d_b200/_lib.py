"""ctypes binding of the C ABI in include/topopt_b200.h.

The shared library is built in-tree (``topopt3d_b200/libtopopt_b200.so``);
there is no fallback: a missing library or a missing GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtopopt_b200.so")

TPO_OK = 0
TPO_NOT_CONVERGED = 1
TPO_E_ARG = -1
TPO_E_CUDA = -2
TPO_E_BREAKDOWN = -3
TPO_E_UNSUPPORTED = -4
MEM_HOST = 0
MEM_DEVICE = 1
PREC_FP64 = 0
PREC_MIXED = 1
BC_SUPPORT = 0
BC_LOAD = 1

# every symbol include/topopt_b200.h declares
EXPORTS = (
    "tpo_default_solve_opts", "tpo_create", "tpo_destroy", "tpo_last_error",
    "tpo_sizes", "tpo_level_dims", "tpo_add_bc", "tpo_set_bc", "tpo_get_bc",
    "tpo_fe_initialize", "tpo_mat_int_fnc", "tpo_set_moduli",
    "tpo_fe_assemble", "tpo_fe_solve", "tpo_solve", "tpo_apply", "tpo_apply_f32",
    "tpo_apply_level", "tpo_apply_level_prec", "tpo_set_level1_form", "tpo_vcycle", "tpo_level_lambda", "tpo_get_vector",
    "tpo_set_vector", "tpo_compliance", "tpo_volume", "tpo_filter",
    "tpo_oc_update", "tpo_sync", "tpo_set_stream", "tpo_kernel_launches",
    "tpo_sensitivity_noalloc", "tpo_default_eig_opts", "tpo_ks_assemble",
    "tpo_ks_apply", "tpo_buckling", "tpo_buckling_sensitivity", "tpo_frequency",
    "tpo_default_mma_opts", "tpo_mma_update", "tpo_mma_last_info",
    "tpo_write_vec_bin", "tpo_read_vec_bin", "tpo_write_mat_bin", "tpo_read_mat_bin",
    "tpo_mesh_out", "tpo_print_vals", "tpo_load_mesh", "tpo_load_design",
    "tpo_load_point_masses", "tpo_barrier_selftest",
)
NOALLOC_MAX_ELEMS = 1 << 20


class MeshParams(C.Structure):
    _fields_ = [("nel", C.c_int32 * 3), ("dx", C.c_double * 3),
                ("E0", C.c_double), ("nu", C.c_double), ("rmin", C.c_double),
                ("mg_levels", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("maxit", C.c_int32),
                ("precision", C.c_int32), ("cheb_degree", C.c_int32),
                ("cheb_lo", C.c_double), ("cheb_hi", C.c_double),
                ("power_its", C.c_int32), ("inner_rtol", C.c_double),
                ("max_outer", C.c_int32), ("use_graph", C.c_int32),
                ("rhs_block", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32),
                ("outer", C.c_int32), ("relres", C.c_double),
                ("solve_ms", C.c_double), ("setup_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EigOpts(C.Structure):
    _fields_ = [("nev", C.c_int32), ("block", C.c_int32), ("maxit", C.c_int32),
                ("tol", C.c_double), ("precond", C.c_int32), ("seed", C.c_uint64)]


class MmaOpts(C.Structure):
    _fields_ = [("move", C.c_double), ("asyinit", C.c_double), ("asyincr", C.c_double),
                ("asydecr", C.c_double), ("albefa", C.c_double), ("raa0", C.c_double),
                ("epsimin", C.c_double)]


class EigInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32),
                ("nconv", C.c_int32), ("max_resid", C.c_double),
                ("solve_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(path: str | None = None):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m topopt3d_b200.build`")
    lib = C.CDLL(p)
    vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    dp = C.POINTER(C.c_double)
    sig = {
        "tpo_default_solve_opts": (None, [C.POINTER(SolveOpts)]),
        "tpo_create": (C.c_int, [C.POINTER(MeshParams), C.POINTER(vp)]),
        "tpo_destroy": (C.c_int, [vp]),
        "tpo_last_error": (C.c_char_p, [vp]),
        "tpo_sizes": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32)]),
        "tpo_level_dims": (C.c_int, [vp, i32, C.POINTER(i32)]),
        "tpo_add_bc": (C.c_int, [vp, i32, dp, dp, dp, dp, C.POINTER(i64)]),
        "tpo_set_bc": (C.c_int, [vp, vp, vp, C.c_int]),
        "tpo_get_bc": (C.c_int, [vp, vp, vp, C.c_int]),
        "tpo_fe_initialize": (C.c_int, [vp]),
        "tpo_mat_int_fnc": (C.c_int, [vp, vp, d, d, C.c_int]),
        "tpo_set_moduli": (C.c_int, [vp, vp, vp, C.c_int]),
        "tpo_fe_assemble": (C.c_int, [vp, C.POINTER(SolveOpts)]),
        "tpo_fe_solve": (C.c_int, [vp, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
        "tpo_solve": (C.c_int, [vp, vp, vp, i32, C.c_int, C.POINTER(SolveOpts),
                                C.POINTER(SolveInfo)]),
        "tpo_apply": (C.c_int, [vp, vp, vp, i32, i32, C.c_int]),
        "tpo_apply_f32": (C.c_int, [vp, vp, vp]),
        "tpo_apply_level": (C.c_int, [vp, i32, vp, vp, C.c_int]),
        "tpo_apply_level_prec": (C.c_int, [vp, i32, vp, vp, i32, C.c_int]),
        "tpo_set_level1_form": (C.c_int, [vp, i32, C.POINTER(i32)]),
        "tpo_vcycle": (C.c_int, [vp, vp, vp, i32, C.c_int]),
        "tpo_level_lambda": (C.c_int, [vp, i32, dp]),
        "tpo_get_vector": (C.c_int, [vp, C.c_char_p, vp, C.c_int]),
        "tpo_set_vector": (C.c_int, [vp, C.c_char_p, vp, C.c_int]),
        "tpo_compliance": (C.c_int, [vp, dp, vp, vp, C.c_int]),
        "tpo_volume": (C.c_int, [vp, dp, vp, C.c_int]),
        "tpo_filter": (C.c_int, [vp, vp, vp, i32, C.c_int]),
        "tpo_oc_update": (C.c_int, [vp, vp, vp, vp, vp, d, vp, d, dp, C.c_int]),
        "tpo_sync": (C.c_int, [vp]),
        "tpo_barrier_selftest": (C.c_int, [vp, i32, i32, i32, i32, C.POINTER(i32)]),
        "tpo_set_stream": (C.c_int, [vp, vp]),
        "tpo_kernel_launches": (C.c_int64, []),
        "tpo_sensitivity_noalloc": (C.c_int, [C.POINTER(i32), dp, d, d, d, vp, vp,
                                              vp, vp, C.c_char_p, i32]),
        "tpo_default_eig_opts": (None, [C.POINTER(EigOpts)]),
        "tpo_ks_assemble": (C.c_int, [vp]),
        "tpo_ks_apply": (C.c_int, [vp, vp, vp, i32, C.c_int]),
        "tpo_buckling": (C.c_int, [vp, C.POINTER(EigOpts), dp, vp, C.c_int,
                                   C.POINTER(EigInfo)]),
        "tpo_buckling_sensitivity": (C.c_int, [vp, i32, dp, vp, d, C.POINTER(SolveOpts),
                                               dp, vp, vp, C.c_int,
                                               C.POINTER(SolveInfo)]),
        "tpo_frequency": (C.c_int, [vp, i32, d, vp, C.POINTER(EigOpts), d, dp,
                                    C.POINTER(i32), dp, vp, C.c_int, C.POINTER(EigInfo)]),
        "tpo_default_mma_opts": (None, [C.POINTER(MmaOpts)]),
        "tpo_mma_update": (C.c_int, [vp, C.POINTER(MmaOpts), i32, C.POINTER(i32), i32,
                                     vp, vp, vp, vp, vp, vp, vp, vp, dp, vp, dp, C.c_int]),
        "tpo_mma_last_info": (C.c_int, [vp, C.POINTER(i32)]),
        "tpo_write_vec_bin": (C.c_int, [C.c_char_p, dp, C.c_int64, i32]),
        "tpo_read_vec_bin": (C.c_int, [C.c_char_p, dp, C.c_int64,
                                       C.POINTER(C.c_int64), i32]),
        "tpo_write_mat_bin": (C.c_int, [C.c_char_p, C.c_int64, C.c_int64,
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int64), dp,
                                        i32]),
        "tpo_read_mat_bin": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64), dp,
                                       C.c_int64, C.c_int64, i32]),
        "tpo_mesh_out": (C.c_int, [vp, C.c_char_p, d, i32]),
        "tpo_print_vals": (C.c_int, [vp, C.c_char_p, C.c_char_p, dp, i32, dp, i32, i32]),
        "tpo_load_mesh": (C.c_int, [C.c_char_p, C.POINTER(MeshParams), i32,
                                    C.POINTER(vp)]),
        "tpo_load_design": (C.c_int, [vp, C.c_char_p, dp, i32, dp, dp, C.POINTER(i32),
                                      i32]),
        "tpo_load_point_masses": (C.c_int, [vp, C.c_char_p, dp, i32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def default_opts(**kw) -> SolveOpts:
    o = SolveOpts()
    load().tpo_default_solve_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def default_mma_opts(**kw) -> MmaOpts:
    o = MmaOpts()
    load().tpo_default_mma_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o


def default_eig_opts(**kw) -> EigOpts:
    o = EigOpts()
    load().tpo_default_eig_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise AttributeError(k)
        setattr(o, k, v)
    return o
