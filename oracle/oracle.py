"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker or the CPU baseline.  The
product package (``topopt3d_b200``) never imports it.

The oracle is an FP64 C restatement of the darinpeetz/TopOpt3D FE path
(see topopt_oracle.h).  Parity against the reference itself is unpinned: the
reference has no tests or golden vectors and cannot be built here (PETSc,
SLEPc, ParMETIS, MPI and Eigen are absent); the oracle is pinned by
mathematical known-answer tests and an independent scipy sparse solve.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libtopopt_oracle.so")
_lib = None


def build() -> str:
    """Compile the oracle shared library (make, system gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "topopt_oracle.c")
        if (not os.path.exists(_LIB_PATH)
                or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class Params(C.Structure):
    _fields_ = [("nel", C.c_int * 3), ("dx", C.c_double * 3), ("E0", C.c_double),
                ("nu", C.c_double), ("rmin", C.c_double), ("mg_levels", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("maxit", C.c_int), ("cheb_degree", C.c_int),
                ("cheb_lo", C.c_double), ("cheb_hi", C.c_double),
                ("power_its", C.c_int)]


def _declare(L):
    vp = C.c_void_p
    L.tor_constitutive.argtypes = [C.c_double, C.c_double, _dp]
    L.tor_element_stiffness.argtypes = [_dp, C.c_double, C.c_double, _dp]
    L.tor_element_nodes.argtypes = [C.POINTER(C.c_int), C.c_int64, _i64]
    L.tor_node_coords.argtypes = [C.POINTER(C.c_int), _dp, _dp, C.c_int64, _dp]
    L.tor_select_nodes.restype = C.c_int64
    L.tor_select_nodes.argtypes = [C.POINTER(C.c_int), _dp, _dp, _dp, _dp, _dp, vp]
    L.tor_filter_build.restype = C.c_int64
    L.tor_filter_build.argtypes = [C.POINTER(C.c_int), _dp, C.c_double, vp, vp, vp]
    L.tor_vecpow.restype = C.c_double
    L.tor_vecpow.argtypes = [C.c_double, C.c_double]
    L.tor_create.restype = vp
    L.tor_create.argtypes = [C.POINTER(Params)]
    L.tor_destroy.argtypes = [vp]
    L.tor_n_nodes.restype = C.c_int64
    L.tor_n_nodes.argtypes = [vp]
    L.tor_n_elems.restype = C.c_int64
    L.tor_n_elems.argtypes = [vp]
    L.tor_set_bc_arrays.argtypes = [vp, vp, vp]
    L.tor_add_bc.restype = C.c_int64
    L.tor_add_bc.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp]
    L.tor_get_bc.argtypes = [vp, _u8, _dp]
    L.tor_set_design.argtypes = [vp, _dp, C.c_double, C.c_double]
    L.tor_get_material.argtypes = [vp, vp, vp, vp]
    L.tor_set_moduli.argtypes = [vp, _dp, vp]
    L.tor_assemble.restype = C.c_int
    L.tor_assemble.argtypes = [vp, C.POINTER(SolveOpts)]
    L.tor_apply.argtypes = [vp, _dp, _dp]
    L.tor_apply_level.argtypes = [vp, C.c_int, _dp, _dp]
    L.tor_level_nodes.restype = C.c_int64
    L.tor_level_nodes.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
    L.tor_level_block.restype = C.c_int
    L.tor_level_block.argtypes = [vp, C.c_int, C.c_int64, C.c_int64, _dp]
    L.tor_level_lambda.restype = C.c_double
    L.tor_level_lambda.argtypes = [vp, C.c_int]
    L.tor_prolong_weight.restype = C.c_double
    L.tor_prolong_weight.argtypes = [vp, C.c_int, C.c_int64, C.c_int64]
    L.tor_vcycle.argtypes = [vp, _dp, _dp]
    L.tor_solve.restype = C.c_int
    L.tor_solve.argtypes = [vp, C.POINTER(SolveOpts), _dp, C.POINTER(C.c_int),
                            C.POINTER(C.c_double)]
    L.tor_solve_rhs.restype = C.c_int
    L.tor_solve_rhs.argtypes = [vp, C.POINTER(SolveOpts), _dp, _dp,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.tor_compliance.argtypes = [vp, _dp, C.POINTER(C.c_double), vp, vp]
    L.tor_volume.argtypes = [vp, C.POINTER(C.c_double), vp]
    L.tor_filter.argtypes = [vp, _dp, _dp, C.c_int]
    L.tor_oc_update.restype = C.c_double
    L.tor_oc_update.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, _dp,
                                C.c_double]
    L.tor_stress_stiffness_element.argtypes = [_dp, C.c_double, C.c_double, _dp,
                                               _dp]
    L.tor_ks_assemble.argtypes = [vp, _dp]
    L.tor_ks_apply.argtypes = [vp, _dp, _dp]
    L.tor_get_es.argtypes = [vp, _dp]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _ivec3(v):
    return (C.c_int * 3)(*[int(t) for t in v])


def element_stiffness(dx=(1.0, 1.0, 1.0), E0=1.0, nu=0.3) -> np.ndarray:
    K = np.zeros(576)
    lib().tor_element_stiffness(np.asarray(dx, float), E0, nu, K)
    return K.reshape(24, 24)


def element_nodes(nel, e) -> np.ndarray:
    out = np.zeros(8, np.int64)
    lib().tor_element_nodes(_ivec3(nel), int(e), out)
    return out


def node_coords(nel, dx, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
    """all node coordinates (nNode x 3, RecMesh.cpp:582-597)"""
    L = lib()
    nn = int(np.prod([n + 1 for n in nel]))
    out = np.zeros((nn, 3))
    xyz = np.zeros(3)
    dxa, oa = np.asarray(dx, float), np.asarray(origin, float)
    for n in range(nn):
        L.tor_node_coords(_ivec3(nel), dxa, oa, n, xyz)
        out[n] = xyz
    return out


def select_nodes(nel, dx, center, radius, limits, origin=(0.0, 0.0, 0.0)):
    L = lib()
    args = [_ivec3(nel), np.asarray(dx, float), np.asarray(origin, float),
            np.asarray(center, float), np.asarray(radius, float),
            np.asarray(limits, float)]
    n = L.tor_select_nodes(*args, None)
    out = np.zeros(max(n, 1), np.int64)
    L.tor_select_nodes(*args, _ptr(out))
    return out[:n]


def filter_csr(nel, dx, R):
    L = lib()
    nel3, dx3 = _ivec3(nel), np.asarray(dx, float)
    nnz = L.tor_filter_build(nel3, dx3, float(R), None, None, None)
    ne = int(np.prod(nel))
    rp = np.zeros(ne + 1, np.int64)
    col = np.zeros(nnz, np.int32)
    val = np.zeros(nnz)
    L.tor_filter_build(nel3, dx3, float(R), _ptr(rp), _ptr(col), _ptr(val))
    return rp, col, val


def vecpow(v, p):
    return lib().tor_vecpow(float(v), float(p))


def default_opts(rtol=1e-8, maxit=500, cheb_degree=2, cheb_lo=0.1, cheb_hi=1.1,
                 power_its=15) -> SolveOpts:
    return SolveOpts(rtol, maxit, cheb_degree, cheb_lo, cheb_hi, power_its)


class Problem:
    """One oracle TopOpt problem: mesh, filter, BCs, material, hierarchy."""

    def __init__(self, nel, dx=(1.0, 1.0, 1.0), E0=1.0, nu=0.3, rmin=1.5,
                 mg_levels=3):
        self.L = lib()
        self.params = Params(_ivec3(nel), (C.c_double * 3)(*dx), E0, nu, rmin,
                             mg_levels)
        self.h = self.L.tor_create(C.byref(self.params))
        self.nel = tuple(int(t) for t in nel)
        self.nn = self.L.tor_n_nodes(self.h)
        self.ne = self.L.tor_n_elems(self.h)
        self.mg_levels = mg_levels

    def __del__(self):
        if getattr(self, "h", None):
            self.L.tor_destroy(self.h)
            self.h = None

    # boundary conditions
    def add_bc(self, kind, center, radius, limits, values) -> int:
        t = {"support": 0, "load": 1}[kind]
        return self.L.tor_add_bc(self.h, t, np.asarray(center, float),
                                 np.asarray(radius, float),
                                 np.asarray(limits, float),
                                 np.asarray(values, float))

    def set_bc(self, fixmask=None, F=None):
        fm = None if fixmask is None else np.ascontiguousarray(fixmask, np.uint8)
        ff = None if F is None else np.ascontiguousarray(F, np.float64)
        self.L.tor_set_bc_arrays(self.h, _ptr(fm), _ptr(ff))

    def get_bc(self):
        fm = np.zeros(self.nn, np.uint8)
        F = np.zeros(3 * self.nn)
        self.L.tor_get_bc(self.h, fm, F)
        return fm, F

    # material
    def set_design(self, x, penal=3.0, eps=1e-10):
        self.L.tor_set_design(self.h, np.ascontiguousarray(x, np.float64),
                              float(penal), float(eps))

    def set_moduli(self, E, dEdz=None):
        d = None if dEdz is None else np.ascontiguousarray(dEdz, np.float64)
        self.L.tor_set_moduli(self.h, np.ascontiguousarray(E, np.float64), _ptr(d))

    def material(self):
        rho, E, dEdz = np.zeros(self.ne), np.zeros(self.ne), np.zeros(self.ne)
        self.L.tor_get_material(self.h, _ptr(rho), _ptr(E), _ptr(dEdz))
        return rho, E, dEdz

    # FE
    def assemble(self, opts=None):
        self.opts = opts or default_opts()
        rc = self.L.tor_assemble(self.h, C.byref(self.opts))
        if rc != 0:
            raise RuntimeError("oracle coarse Cholesky failed")

    def apply(self, u):
        y = np.zeros(3 * self.nn)
        self.L.tor_apply(self.h, np.ascontiguousarray(u, np.float64), y)
        return y

    def apply_level(self, level, u):
        n = self.level_nodes(level)[0]
        y = np.zeros(3 * n)
        self.L.tor_apply_level(self.h, level, np.ascontiguousarray(u, np.float64), y)
        return y

    def level_nodes(self, level):
        dims = (C.c_int * 3)()
        n = self.L.tor_level_nodes(self.h, level, dims)
        return n, tuple(dims)

    def level_block(self, level, i, j):
        b = np.zeros(9)
        self.L.tor_level_block(self.h, level, int(i), int(j), b)
        return b.reshape(3, 3)

    def level_lambda(self, level):
        return self.L.tor_level_lambda(self.h, level)

    def prolong_weight(self, level, f, c):
        return self.L.tor_prolong_weight(self.h, level, int(f), int(c))

    def vcycle(self, r):
        z = np.zeros(3 * self.nn)
        self.L.tor_vcycle(self.h, np.ascontiguousarray(r, np.float64), z)
        return z

    def solve(self, U0=None, b=None, opts=None):
        o = opts or self.opts
        U = np.zeros(3 * self.nn) if U0 is None else np.array(U0, np.float64)
        its, rr = C.c_int(0), C.c_double(0)
        if b is None:
            st = self.L.tor_solve(self.h, C.byref(o), U, C.byref(its), C.byref(rr))
        else:
            st = self.L.tor_solve_rhs(self.h, C.byref(o),
                                      np.ascontiguousarray(b, np.float64), U,
                                      C.byref(its), C.byref(rr))
        return U, st, its.value, rr.value

    def compliance(self, U):
        c = C.c_double(0)
        dx, dr = np.zeros(self.ne), np.zeros(self.ne)
        self.L.tor_compliance(self.h, np.ascontiguousarray(U, np.float64),
                              C.byref(c), _ptr(dx), _ptr(dr))
        return c.value, dx, dr

    # buckling (Buckling.cpp:15-361)
    def ks_assemble(self, U):
        self.L.tor_ks_assemble(self.h, np.ascontiguousarray(U, np.float64))

    def ks_apply(self, u):
        y = np.zeros(3 * self.nn)
        self.L.tor_ks_apply(self.h, np.ascontiguousarray(u, np.float64), y)
        return y

    def es(self):
        out = np.zeros(self.ne)
        self.L.tor_get_es(self.h, out)
        return out

    def volume(self):
        v = C.c_double(0)
        dv = np.zeros(self.ne)
        self.L.tor_volume(self.h, C.byref(v), _ptr(dv))
        return v.value, dv

    def filter(self, v, transpose=False):
        out = np.zeros(self.ne)
        self.L.tor_filter(self.h, np.ascontiguousarray(v, np.float64), out,
                          int(bool(transpose)))
        return out


def stress_stiffness_element(u, dx=(1.0, 1.0, 1.0), E0=1.0, nu=0.3):
    """ks (24x24) of one element for its displacements u (24, reference
    local node order), Buckling.cpp:313-327."""
    ks = np.zeros(576)
    lib().tor_stress_stiffness_element(np.asarray(dx, np.float64), E0, nu,
                                       np.ascontiguousarray(u, np.float64), ks)
    return ks.reshape(24, 24)


def dense(apply, n):
    """Dense matrix of a linear operator on R^n by columns (small n)."""
    A = np.zeros((n, n))
    e = np.zeros(n)
    for j in range(n):
        e[j] = 1.0
        A[:, j] = apply(e)
        e[j] = 0.0
    return A


def buckling(pb, nev=6, ncv=None, tol=1e-12, solve_rtol=1e-13, v0_seed=0):
    """The nev largest eigenvalues of Ks phi = lambda K phi (the target LR
    of Buckling.cpp:63-70) for an assembled problem whose Ks has been built
    (ks_assemble).  Independent of the CUDA path's eigensolver: ARPACK
    Lanczos (scipy eigsh, generalized mode with M = K) whose M^-1 is the
    oracle's PCG + GMG solve to solve_rtol.  Returns (lambda descending,
    phi as rows, K-normalised)."""
    import scipy.sparse.linalg as spl
    n = 3 * pb.nn
    o = default_opts(rtol=solve_rtol, maxit=5000)
    A = spl.LinearOperator((n, n), matvec=pb.ks_apply, dtype=np.float64)
    M = spl.LinearOperator((n, n), matvec=pb.apply, dtype=np.float64)

    def minv(b):
        U, st, _, _ = pb.solve(b=np.ascontiguousarray(b, np.float64).ravel(), opts=o)
        if st != 0:
            raise RuntimeError(f"oracle solve failed (status {st})")
        return U

    Minv = spl.LinearOperator((n, n), matvec=minv, dtype=np.float64)
    v0 = np.random.default_rng(v0_seed).standard_normal(n)
    lam, phi = spl.eigsh(A, k=nev, M=M, Minv=Minv, which="LA", tol=tol,
                         ncv=ncv or max(2 * nev + 1, 20), v0=v0)
    order = np.argsort(lam)[::-1]
    return lam[order], phi[:, order].T


def buckling_sensitivity(pb, nel, U, lam, phi, penal=3.0, p=8.0,
                         dx=(1.0, 1.0, 1.0), E0=1.0, nu=0.3, solve_rtol=1e-13):
    """The gradient of Stability::Function (Buckling.cpp:113-272) with the
    filter chain rule (TopOpt::Chain_Filter, Material_Interpolation.cpp:
    150-187, which without a max-length filter is P^T), in numpy over the
    oracle.  pb is set up as for `buckling` (design set, assembled, Ks built
    from U); lam (nev) and phi (nev x 3 nNode, K-normalised) the eigenpairs.

    value = (sum lam^p)^(1/p) (:87-88).  The adjoint right-hand side of pair
    i is sum_e Es_e phi_e^T dKsdu[a] phi_e at the element's dofs a, with
    dKsdu[a] = ks_e of a unit displacement (:134-147, :155-178), zero at
    fixed dofs (:186-190); v_i solves K v_i = rhs_i (:193-225).  Per element
    (:229-263): sum_i lam_i^(p-1) (phi^T dKsdy phi - lam_i phi^T dKdy phi +
    v_i^T dKdy U), dKsdy = -dEsdz ks_e(U) (StressFnc :331-332), dKdy =
    dEdz K0, times value^(1-p) (:265).  dEsdz = p rho^(p-1)
    (Material_Interpolation.cpp:67-70).  Returns (value, dvdx, dvdrho)."""
    nel = tuple(int(v) for v in nel)
    ne = int(np.prod(nel))
    n = 3 * pb.nn
    nodes = np.array([element_nodes(nel, e) for e in range(ne)])
    dofs = (3 * nodes[:, :, None] + np.arange(3)).reshape(ne, 24)
    rho, _, dEdz = pb.material()
    Es = pb.es()
    dEsdz = penal * rho ** (penal - 1)
    K0 = element_stiffness(dx, E0, nu)
    eye = np.eye(24)
    dKsdu = np.array([stress_stiffness_element(eye[d], dx, E0, nu) for d in range(24)])
    lam = np.asarray(lam, np.float64)
    phi = np.asarray(phi, np.float64)
    nev = lam.size
    Ue = U[dofs]
    Pe = phi[:, dofs]
    t = np.einsum("kei,aij,kej->kea", Pe, dKsdu, Pe) * Es[None, :, None]
    rhs = np.zeros((nev, n))
    for k in range(nev):
        np.add.at(rhs[k], dofs.ravel(), t[k].ravel())
    fm, _ = pb.get_bc()
    fixed = ((fm[:, None] >> np.arange(3)) & 1).astype(bool).ravel()
    rhs[:, fixed] = 0.0
    o = default_opts(rtol=solve_rtol, maxit=5000)
    V = np.zeros_like(rhs)
    for k in range(nev):
        V[k], st, _, _ = pb.solve(b=np.ascontiguousarray(rhs[k]), opts=o)
        if st != 0:
            raise RuntimeError(f"oracle adjoint solve failed (status {st})")
    Ve = V[:, dofs]
    ks = np.einsum("ed,dij->eij", Ue, dKsdu)      # ks_e(U), linear in U
    pdKsp = -dEsdz[None] * np.einsum("kei,eij,kej->ke", Pe, ks, Pe)
    pdKp = dEdz[None] * np.einsum("kei,ij,kej->ke", Pe, K0, Pe)
    vKu = dEdz[None] * np.einsum("kei,ij,ej->ke", Ve, K0, Ue)
    value = float(np.sum(lam ** p) ** (1.0 / p))
    g = np.sum(lam[:, None] ** (p - 1) * (pdKsp - lam[:, None] * pdKp + vKu), axis=0)
    g *= value ** (1.0 - p)
    return value, pb.filter(g, transpose=True), g


def buckling_dense(pb, nev):
    """The nev largest eigenpairs of Ks phi = lambda K phi by a dense
    generalized symmetric eigensolve (small problems only): lambda
    descending, phi as rows, K-normalised."""
    import scipy.linalg as sla
    n = 3 * pb.nn
    A = dense(pb.ks_apply, n)
    B = dense(pb.apply, n)
    w, v = sla.eigh(0.5 * (A + A.T), 0.5 * (B + B.T))
    order = np.argsort(w)[::-1][:nev]
    return w[order], v[:, order].T


def lumped_mass(pb, nel, density, dx=(1.0, 1.0, 1.0), mlump=None):
    """Frequency::DiagMassFnc (Dynamic.cpp:181-235) with the fixed-dof
    zeroing (:42-44): each element adds V_e * elemSize * density / (2^3 * 3)
    to the three dofs of each of its nodes (V = rho,
    Material_Interpolation.cpp:63-64), then the point masses; 1e-8 on fixed
    dofs."""
    nel = tuple(int(v) for v in nel)
    ne = int(np.prod(nel))
    rho, _, _ = pb.material()
    scale = float(np.prod(dx)) * density / 8.0 / 3.0
    m = np.zeros(3 * pb.nn)
    for e in range(ne):
        for nd in element_nodes(nel, e):
            m[3 * nd:3 * nd + 3] += rho[e] * scale
    if mlump is not None:
        m += mlump
    fm, _ = pb.get_bc()
    fixed = ((fm[:, None] >> np.arange(3)) & 1).astype(bool).ravel()
    m[fixed] = 1e-8
    return m, scale


def frequency_dense(pb, nel, nvals, density, p=8.0, dx=(1.0, 1.0, 1.0),
                    E0=1.0, nu=0.3, mlump=None):
    """Frequency::Function (Dynamic.cpp:18-171) by a dense generalized
    eigensolve (small problems only): the largest eigenvalues of
    M phi = lambda K phi, more than nvals of them until the last is
    separated from the one before it by a relative 1e-5 (UNIQUE_LAST_NEV,
    EigenPeetz.cpp:310-312); value = (sum lambda^p)^(1/p) over all of them;
    the gradient sums the first nvals - 1 pairs (:127-160),
    lambda_j^(p-1) phi_j^T (dMdy - lambda_j dKdy) phi_j per element (dMdy =
    dVdrho * the element mass, dKdy = dEdz K0), times value^(1-p), then
    P^T.  Returns (lambda, value, dvdx, dlam) with dlam[j] = d lambda_j /
    d rho (before the filter) for every pair."""
    import scipy.linalg as sla
    nel = tuple(int(v) for v in nel)
    ne = int(np.prod(nel))
    m, scale = lumped_mass(pb, nel, density, dx, mlump)
    K = dense(pb.apply, 3 * pb.nn)
    w, v = sla.eigh(np.diag(m), 0.5 * (K + K.T))
    order = np.argsort(w)[::-1]
    nev = nvals + 1
    while abs(1.0 - w[order[nev - 2]] / w[order[nev - 1]]) <= 1e-5:
        nev += 1
    lam = w[order[:nev]]
    phi = v[:, order[:nev]].T
    nodes = np.array([element_nodes(nel, e) for e in range(ne)])
    dofs = (3 * nodes[:, :, None] + np.arange(3)).reshape(ne, 24)
    _, _, dEdz = pb.material()
    K0 = element_stiffness(dx, E0, nu)
    Pe = phi[:, dofs]
    pmp = scale * np.sum(Pe * Pe, axis=2)
    pkp = dEdz[None] * np.einsum("kei,ij,kej->ke", Pe, K0, Pe)
    dlam = pmp - lam[:, None] * pkp
    value = float(np.sum(lam ** p) ** (1.0 / p))
    nt = max(0, nvals - 1)
    g = np.sum(lam[:nt, None] ** (p - 1) * dlam[:nt], axis=0) * value ** (1.0 - p)
    return lam, value, pb.filter(g, transpose=True), dlam


MMA_DEFAULTS = dict(move=0.5, asyinit=0.5, asyincr=1.2, asydecr=0.7, albefa=0.1,
                    raa0=1e-5, epsimin=1e-7)   # MMA.h:21-23


def mma_update(st, dfdx, g, dgdx, iter_, **opts):
    """MMA::MMAsub (MMA.cpp:185-343) with MMA::DualSolve (:353-595) for
    m = len(g) constraints, in numpy.  st holds x, xold1, xold2, low, upp,
    xmin, xmax (n-vectors) and fresh_start; it is updated in place (and
    newton_steps set to the number of dual Newton steps taken).  The
    constants are Set_m's (:40-52): a0 = b0 = 1, a = 0, c = 1000, d = 1.
    Returns Change."""
    o = dict(MMA_DEFAULTS, **opts)
    x, x1, x2 = st["x"], st["xold1"], st["xold2"]
    xmin, xmax = st["xmin"], st["xmax"]
    dgdx = np.asarray(dgdx, np.float64).reshape(x.size, -1)
    g = np.asarray(g, np.float64).ravel()
    m = g.size
    a0, b0, a, c, d = 1.0, 1.0, np.zeros(m), 1000.0 * np.ones(m), np.ones(m)
    span = xmax - xmin
    if st["fresh_start"] and iter_ < 3:
        low = x - o["asyinit"] * span
        upp = x + o["asyinit"] * span
    else:
        st["fresh_start"] = False
        zzz = (x - x1) * (x1 - x2)
        factor = np.where(zzz > 0, o["asyincr"], np.where(zzz < 0, o["asydecr"], 1.0))
        low = x - factor * (x1 - st["low"])
        upp = x + factor * (st["upp"] - x1)
        low = np.minimum(np.maximum(low, x - 10 * span), x - 0.01 * span)
        upp = np.maximum(np.minimum(upp, x + 10 * span), x + 0.01 * span)
    alfa = np.maximum(np.maximum(low + o["albefa"] * (x - low), x - o["move"] * span), xmin)
    beta = np.minimum(np.minimum(upp - o["albefa"] * (upp - x), x + o["move"] * span), xmax)
    xmami = np.maximum(upp - low, 1e-5)
    ux1, xl1 = upp - x, x - low
    ux2, xl2 = ux1 * ux1, xl1 * xl1
    p0 = np.maximum(dfdx, 0.0)
    q0 = np.maximum(-dfdx, 0.0)
    pq0 = 0.001 * (p0 + q0) + 0.5 * o["raa0"] / xmami
    p0 = (p0 + pq0) * ux2
    q0 = (q0 + pq0) * xl2
    P = np.maximum(dgdx, 0.0) * ux2[:, None]
    Q = np.maximum(-dgdx, 0.0) * xl2[:, None]
    b = np.sum(P / ux1[:, None] + Q / xl1[:, None], axis=0) - g
    st["xold2"] = x1.copy()
    st["xold1"] = x.copy()
    st["low"], st["upp"] = low, upp

    def xyz(lam):
        plam, qlam = p0 + P @ lam, q0 + Q @ lam
        pr, qr = np.sqrt(plam), np.sqrt(qlam)
        xx = np.minimum(np.maximum((pr * low + qr * upp) / (pr + qr), alfa), beta)
        y = np.maximum((lam - c) / d, 0.0)
        z = 10 * max((lam @ a - a0) / b0, 0.0)
        return xx, y, z, plam, qlam

    def grad(xx, y, z):
        return np.sum(P / (upp - xx)[:, None] + Q / (xx - low)[:, None], axis=0) - (b + a * z + y)

    def hess(xx, lam, plam, qlam):
        u1, l1 = upp - xx, xx - low
        dhdx = (P / (u1 * u1)[:, None] - Q / (l1 * l1)[:, None]).T
        inside = ((xx > alfa) & (xx < beta)).astype(np.float64)
        dLdxx = inside / (2 * plam / u1 ** 3 + 2 * qlam / l1 ** 3)
        H = -(dhdx * dLdxx) @ dhdx.T
        H -= np.diag((lam > c).astype(np.float64))
        if lam @ a > 0:
            H -= 10 * np.outer(a, a)
        return H

    epsi = 1.0
    eta = np.ones(m)
    lam = 500 * eta
    xx, y, z, plam, qlam = xyz(lam)
    G = grad(xx, y, z)
    steps = 0
    while epsi > o["epsimin"]:
        epsvec = np.full(m, epsi)
        resmax = np.max(np.abs(np.concatenate([G + eta, eta * lam - epsvec])))
        it = 0
        while resmax > 0.9 * epsi and it < 100:
            it += 1
            steps += 1
            H = hess(xx, lam, plam, qlam)
            A = H - np.diag(eta / lam)
            A += min(1e-4 * np.trace(A) / m, -1e-7) * np.eye(m)
            dl = np.linalg.solve(A, -G - epsvec / lam)
            de = -eta + epsvec / lam - dl * (eta / lam)
            theta = 1.0
            for r in (-0.99 * lam / dl, -0.99 * eta / de):
                for v in r:
                    if v >= 0:
                        theta = min(theta, v)
            lam = lam + theta * dl
            eta = eta + theta * de
            xx, y, z, plam, qlam = xyz(lam)
            G = grad(xx, y, z)
            resmax = np.max(np.abs(np.concatenate([G + eta, eta * lam - epsvec])))
        epsi *= 0.1
    st["x"] = xx
    st["newton_steps"] = steps
    return float(np.max(np.abs((xx - st["xold1"]) / span)))


def oc_update(x, dfdx, g, dgdx, move, xmin=None, xmax=None):
    """MMA::OCsub (MMA.cpp:103-180); returns (x_new, change)."""
    n = x.size
    xx = np.array(x, np.float64)
    xmin = np.zeros(n) if xmin is None else np.asarray(xmin, np.float64)
    xmax = np.ones(n) if xmax is None else np.asarray(xmax, np.float64)
    df = np.array(dfdx, np.float64)
    ch = lib().tor_oc_update(n, xx, xmin, xmax, df, float(g),
                             np.ascontiguousarray(dgdx, np.float64), float(move))
    return xx, ch


def optimize_oc(pb, x0, volfrac, iters, move=0.5, penal=3.0, opts=None):
    """The optimisation loop of Main.cpp:130-170 restated over the oracle:
    Compliance objective (weight 1, range [0, 1]) and one Volume constraint
    V <= volfrac (Functions.cpp:39-62 with Inputs.cpp:554-557 pre-scaling),
    updated by OCsub (MMA.cpp:103-180) for `iters` updates, i.e. iters + 1
    evaluations.  Each FE solve warm-starts from the previous U
    (FEAnalysis.cpp:389).  Returns per-evaluation C, V, Change and PCG
    iterations, and the final design."""
    opts = opts or default_opts()
    x = np.array(x0, np.float64)
    U = None
    Cs, Vs, chs, its_l = [], [], [], []
    change = 1.0

    def evaluate():
        nonlocal U
        pb.set_design(x, penal, 1e-10)
        pb.assemble(opts)
        U, st, its, _ = pb.solve(U0=U, opts=opts)
        if st != 0:
            raise RuntimeError(f"oracle solve did not converge (status {st})")
        C, dCdx, _ = pb.compliance(U)
        V, dVdx = pb.volume()
        Cs.append(C)
        Vs.append(V)
        chs.append(change)
        its_l.append(its)
        return dCdx, V - volfrac, dVdx

    dfdx, g, dgdx = evaluate()
    for _ in range(iters):
        x, change = oc_update(x, dfdx, g, dgdx, move)
        dfdx, g, dgdx = evaluate()
    return dict(C=np.array(Cs), V=np.array(Vs), change=np.array(chs),
                its=np.array(its_l), x=x)
