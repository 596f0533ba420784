"""Python mirror of the darinpeetz/TopOpt3D call surface over the C ABI.

``TopOpt`` keeps the reference member names (TopOpt.h:210-292):
``Set_BC``, ``FEInitialize``, ``MatIntFnc``, ``FEAssemble``, ``FESolve``,
``Chain_Filter``, and the output and restart files ``MeshOut``,
``PrintVals``, ``LoadMesh`` (TopOpt.cpp:97-508, RecMesh.cpp:34-412);
``Compliance``, ``Volume``, ``Stability`` and ``Frequency`` follow
``Function_Base`` (Functions.h:16-91) with ``Compute`` and
``Function_Call``; ``OC`` and ``MMA`` follow ``MMA::Update``
(MMA.cpp:62-595); ``optimize`` is the loop of Main.cpp:120-178 with the
Output.txt log of StepOut and ResultOut (TopOpt.cpp:372-435).  Where the
reference returns a non-zero PetscErrorCode these methods raise
``TopOptError``; solver non-convergence is reported, as KUF_reason is, in
``last_solve`` without raising.

Vectors are numpy arrays (host) or torch CUDA float64 tensors (device);
every call runs on the GPU through libtopopt_b200.so.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


class TopOptError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _buf(a, n=None, writable=False):
    """(pointer, mem flag, keepalive) for a numpy array or torch tensor."""
    if a is None:
        return None, L.MEM_HOST, None
    if _is_torch(a):
        import torch
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError("device buffers must be contiguous float64 tensors")
        if n is not None and a.numel() < n:
            raise ValueError(f"buffer has {a.numel()} values, need {n}")
        mem = L.MEM_DEVICE if a.is_cuda else L.MEM_HOST
        return C.c_void_p(a.data_ptr()), mem, a
    arr = np.ascontiguousarray(a, dtype=np.float64)
    if writable and arr is not a:
        raise TypeError("output numpy arrays must be contiguous float64")
    if n is not None and arr.size < n:
        raise ValueError(f"buffer has {arr.size} values, need {n}")
    return arr.ctypes.data_as(C.c_void_p), L.MEM_HOST, arr


class TopOpt:
    """One structured hex8 TopOpt problem resident on one GPU."""

    SUPPORT = L.BC_SUPPORT
    LOAD = L.BC_LOAD

    def __init__(self, nel, dx=(1.0, 1.0, 1.0), E0=1.0, Nu0=0.3, rmin=1.5,
                 mg_levels=0):
        self._lib = L.load()
        p = L.MeshParams((C.c_int32 * 3)(*[int(t) for t in nel]),
                         (C.c_double * 3)(*[float(t) for t in dx]),
                         float(E0), float(Nu0), float(rmin), int(mg_levels))
        h = C.c_void_p()
        rc = self._lib.tpo_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise TopOptError(rc, "tpo_create failed (invalid mesh or no GPU)")
        self._attach(h)

    def _attach(self, h):
        self._h = h
        ne, nn, nl = C.c_int64(), C.c_int64(), C.c_int32()
        self._lib.tpo_sizes(h, C.byref(ne), C.byref(nn), C.byref(nl))
        self.nel = tuple(int(t) - 1 for t in self.level_dims(0))
        self.nElem, self.nNode, self.mg_levels = ne.value, nn.value, nl.value
        self.penal = 3.0
        self.eps = 1e-10           # Material_Interpolation.cpp:28
        self.opts = L.default_opts()
        self.last_solve = None
        self.function_list = []

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc, what):
        if rc < 0:
            msg = self._lib.tpo_last_error(self._h).decode(errors="replace")
            raise TopOptError(rc, f"{what}: {msg}")
        return rc

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tpo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def level_dims(self, level):
        d = (C.c_int32 * 3)()
        self._check(self._lib.tpo_level_dims(self._h, level, d), "level_dims")
        return tuple(d)

    # -- boundary conditions (Inputs.cpp:105-223) --------------------------
    def Set_BC(self, center, radius, limits, values, TYPE):
        n = C.c_int64()
        arr = lambda v, k: (C.c_double * k)(*[float(t) for t in v])
        self._check(self._lib.tpo_add_bc(self._h, int(TYPE), arr(center, 3),
                                         arr(radius, 3), arr(limits, 6),
                                         arr(values, 3), C.byref(n)), "Set_BC")
        return n.value

    def set_bc_arrays(self, fixmask=None, F=None):
        fm = None if fixmask is None else np.ascontiguousarray(fixmask, np.uint8)
        fp, mem, keep = _buf(F, 3 * self.nNode)
        self._check(self._lib.tpo_set_bc(
            self._h, None if fm is None else fm.ctypes.data_as(C.c_void_p),
            fp, mem if F is not None else L.MEM_HOST), "set_bc")

    def get_bc(self):
        fm = np.zeros(self.nNode, np.uint8)
        F = np.zeros(3 * self.nNode)
        self._check(self._lib.tpo_get_bc(self._h, fm.ctypes.data_as(C.c_void_p),
                                         F.ctypes.data_as(C.c_void_p),
                                         L.MEM_HOST), "get_bc")
        return fm, F

    # -- FE ----------------------------------------------------------------
    def FEInitialize(self):
        self._check(self._lib.tpo_fe_initialize(self._h), "FEInitialize")

    def MatIntFnc(self, design):
        p, mem, keep = _buf(design, self.nElem)
        self._check(self._lib.tpo_mat_int_fnc(self._h, p, self.penal, self.eps,
                                              mem), "MatIntFnc")

    def set_moduli(self, E, dEdz=None):
        p, mem, k1 = _buf(E, self.nElem)
        q, _, k2 = _buf(dEdz, self.nElem)
        self._check(self._lib.tpo_set_moduli(self._h, p, q, mem), "set_moduli")

    def FEAssemble(self, opts=None):
        if opts is not None:
            self.opts = opts
        self._check(self._lib.tpo_fe_assemble(self._h, C.byref(self.opts)),
                    "FEAssemble")

    def FESolve(self, opts=None):
        info = L.SolveInfo()
        o = opts or self.opts
        rc = self._check(self._lib.tpo_fe_solve(self._h, C.byref(o),
                                                C.byref(info)), "FESolve")
        self.KUF_reason = rc
        self.last_solve = info.as_dict()
        return self.last_solve

    def solve(self, b, U, nrhs=1, opts=None):
        """Solve K U = b for nrhs column-major right-hand sides."""
        info = L.SolveInfo()
        bp, mem, k1 = _buf(b, 3 * self.nNode * nrhs)
        up, mem2, k2 = _buf(U, 3 * self.nNode * nrhs, writable=True)
        if mem != mem2:
            raise ValueError("b and U must both be host or both be device")
        self._check(self._lib.tpo_solve(self._h, bp, up, nrhs, mem,
                                        C.byref(opts or self.opts),
                                        C.byref(info)), "solve")
        return info.as_dict()

    def apply(self, u, y, nrhs=1, precision=L.PREC_FP64):
        up, mem, k1 = _buf(u, 3 * self.nNode * nrhs)
        yp, mem2, k2 = _buf(y, 3 * self.nNode * nrhs, writable=True)
        self._check(self._lib.tpo_apply(self._h, up, yp, nrhs, precision, mem),
                    "apply")
        return y

    def apply_level(self, level, u, y, precision=L.PREC_FP64):
        up, mem, k1 = _buf(u)
        yp, _, k2 = _buf(y, writable=True)
        self._check(self._lib.tpo_apply_level_prec(self._h, level, up, yp,
                                                   precision, mem),
                    "apply_level")
        return y

    def set_level1_form(self, form):
        """0: tensor-core level-1 operator where the mesh allows it (the
        default), 1: the stored stencil.  Returns True when the tensor-core
        form is in use."""
        on = C.c_int32()
        self._check(self._lib.tpo_set_level1_form(self._h, form, C.byref(on)),
                    "set_level1_form")
        return bool(on.value)

    def vcycle(self, r, z, precision=L.PREC_FP64):
        rp, mem, k1 = _buf(r, 3 * self.nNode)
        zp, _, k2 = _buf(z, 3 * self.nNode, writable=True)
        self._check(self._lib.tpo_vcycle(self._h, rp, zp, precision, mem),
                    "vcycle")
        return z

    def level_lambda(self, level):
        v = C.c_double()
        self._check(self._lib.tpo_level_lambda(self._h, level, C.byref(v)),
                    "level_lambda")
        return v.value

    def get(self, which, out=None):
        n = 3 * self.nNode if which in ("U", "F") else self.nElem
        out = np.zeros(n) if out is None else out
        p, mem, keep = _buf(out, n, writable=True)
        self._check(self._lib.tpo_get_vector(self._h, which.encode(), p, mem),
                    f"get {which}")
        return out

    def set(self, which, values):
        n = 3 * self.nNode if which in ("U", "F") else self.nElem
        p, mem, keep = _buf(values, n)
        self._check(self._lib.tpo_set_vector(self._h, which.encode(), p, mem),
                    f"set {which}")

    @property
    def U(self):
        return self.get("U")

    @property
    def F(self):
        return self.get("F")

    @property
    def rho(self):
        return self.get("rho")

    @property
    def E(self):
        return self.get("E")

    @property
    def dEdz(self):
        return self.get("dEdz")

    # -- filter chain (Material_Interpolation.cpp:150-187) -----------------
    def filter(self, v, out=None, transpose=False):
        out = np.zeros(self.nElem) if out is None else out
        ip, mem, k1 = _buf(v, self.nElem)
        op, _, k2 = _buf(out, self.nElem, writable=True)
        self._check(self._lib.tpo_filter(self._h, ip, op, int(bool(transpose)),
                                         mem), "filter")
        return out

    def Chain_Filter(self, dfdV=None, dfdE=None):
        """In-place chain rule through the density filter (vdMin <= 0)."""
        for v in (dfdV, dfdE):
            if v is not None:
                tmp = self.filter(v, transpose=True)
                v[...] = tmp
        return dfdV, dfdE

    def compliance(self, gradient=True, want_drho=False, out=None):
        """C = U.F and dC/dx; `out` may be a host or device float64 buffer
        that receives dC/dx."""
        c = C.c_double()
        if out is not None:
            dx = out
        else:
            dx = np.zeros(self.nElem) if gradient else None
        dr = np.zeros(self.nElem) if want_drho else None
        p, mem, keep = _buf(dx, self.nElem, writable=True)
        if dr is not None and mem != L.MEM_HOST:
            raise ValueError("want_drho needs a host output buffer")
        self._check(self._lib.tpo_compliance(
            self._h, C.byref(c), p,
            None if dr is None else dr.ctypes.data_as(C.c_void_p),
            mem), "compliance")
        return c.value, dx, dr

    # -- output and restart files (TopOpt.cpp:97-508, RecMesh.cpp:34-412) ---
    def MeshOut(self, folder=".", rmax=3.0, index_bytes=4):
        """TopOpt::MeshOut (TopOpt.cpp:97-359) into `folder`; rmax is the
        max-length-scale filter radius (3 by default, Main.cpp:41).
        index_bytes is sizeof(PetscInt) of the PETSc build that reads the
        files."""
        self._check(self._lib.tpo_mesh_out(self._h, os.fsencode(folder), float(rmax),
                                           int(index_bytes)), "MeshOut")

    def PrintVals(self, name_suffix, folder=".", phiB=None, phiD=None, index_bytes=4):
        """TopOpt::PrintVals (TopOpt.cpp:445-508): U, x, V, Es, E and the
        buckling (phiB) and dynamic (phiD) mode shapes, 3*nNode x modes."""
        def modes(phi):
            if phi is None:
                return None, 0, None
            a = np.asfortranarray(np.asarray(phi, np.float64).reshape(3 * self.nNode, -1))
            return a.ctypes.data_as(C.POINTER(C.c_double)), a.shape[1], a
        pb, nb, kb = modes(phiB)
        pd, nd, kd = modes(phiD)
        self._check(self._lib.tpo_print_vals(self._h, os.fsencode(folder),
                                             str(name_suffix).encode(), pb, nb, pd, nd,
                                             int(index_bytes)), "PrintVals")

    @classmethod
    def LoadMesh(cls, folder, E0=1.0, Nu0=0.3, rmin=1.5, mg_levels=0, index_bytes=4):
        """TopOpt::LoadMesh (RecMesh.cpp:34-412): a problem from a MeshOut
        folder of a structured hex8 box, with its supports and loads;
        mg_levels 0 takes the levels the folder's interpolations hold."""
        lib = L.load()
        p = L.MeshParams((C.c_int32 * 3)(1, 1, 1), (C.c_double * 3)(1.0, 1.0, 1.0),
                         float(E0), float(Nu0), float(rmin), int(mg_levels))
        h = C.c_void_p()
        rc = lib.tpo_load_mesh(os.fsencode(folder), C.byref(p), int(index_bytes),
                               C.byref(h))
        if rc != 0:
            raise TopOptError(rc, "LoadMesh: " +
                              lib.tpo_last_error(None).decode(errors="replace"))
        self = cls.__new__(cls)
        self._lib = lib
        self._attach(h)
        self.penal = 3.0
        self.eps = 1e-10
        self.opts = L.default_opts()
        self.last_solve = None
        self.function_list = []
        return self

    def load_design(self, folder, penalties, index_bytes=4):
        """The design of a restart (RecMesh.cpp:391-404, Main.cpp:52-56):
        x = 0.5, then x_pen<p>.bin for each penalty in turn until one is
        missing.  Sets self.penal to the penalty reached and returns
        (x, index of the first penalty still to run)."""
        pen = np.ascontiguousarray(penalties, np.float64)
        x = np.zeros(self.nElem)
        pn = C.c_double(self.penal)
        st = C.c_int32()
        self._check(self._lib.tpo_load_design(
            self._h, os.fsencode(folder), pen.ctypes.data_as(C.POINTER(C.c_double)),
            pen.size, x.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pn), C.byref(st),
            int(index_bytes)), "load_design")
        self.penal = pn.value
        return x, st.value

    def load_point_masses(self, folder, index_bytes=4):
        """massNodes.bin / masses.bin (RecMesh.cpp:147-180) as the 3*nNode
        point-mass vector `frequency` takes."""
        m = np.zeros(3 * self.nNode)
        self._check(self._lib.tpo_load_point_masses(
            self._h, os.fsencode(folder), m.ctypes.data_as(C.POINTER(C.c_double)),
            int(index_bytes)), "load_point_masses")
        return m

    def set_stream(self, stream_handle):
        """Issue all work on a caller cudaStream_t (int handle) or None."""
        self._check(self._lib.tpo_set_stream(
            self._h, None if stream_handle is None else C.c_void_p(stream_handle)),
            "set_stream")

    # -- linear buckling (Buckling.cpp:15-414) ------------------------------
    def ks_assemble(self):
        """Stability::StressFnc from the current U and material."""
        self._check(self._lib.tpo_ks_assemble(self._h), "ks_assemble")

    def ks_apply(self, u, y, nrhs=1):
        up, mem, k1 = _buf(u, 3 * self.nNode * nrhs)
        yp, _, k2 = _buf(y, 3 * self.nNode * nrhs, writable=True)
        self._check(self._lib.tpo_ks_apply(self._h, up, yp, nrhs, mem), "ks_apply")
        return y

    def buckling(self, opts=None, want_vectors=False, **kw):
        """The largest eigenvalues of Ks phi = lambda K phi (descending) and,
        if asked, the K-orthonormal eigenvectors as rows; the solver record
        is kept in last_eig."""
        o = opts or L.default_eig_opts(**kw)
        lam = np.zeros(o.nev)
        phi = np.zeros((o.nev, 3 * self.nNode)) if want_vectors else None
        info = L.EigInfo()
        rc = self._check(self._lib.tpo_buckling(
            self._h, C.byref(o), lam.ctypes.data_as(C.POINTER(C.c_double)),
            None if phi is None else phi.ctypes.data_as(C.c_void_p), L.MEM_HOST,
            C.byref(info)), "buckling")
        self.last_eig = info.as_dict()
        self.last_eig["rc"] = rc
        return (lam, phi) if want_vectors else lam

    def buckling_sensitivity(self, lam, phi, p=8.0, opts=None, want_drho=False):
        """The aggregated buckling value (sum lam^p)^(1/p) and its gradient
        with respect to the design (Buckling.cpp:87-88, 113-272 with the
        filter chain rule) from the eigenpairs `buckling(want_vectors=True)`
        returned (phi as rows, K-normalised); with want_drho also the
        gradient with respect to the filtered density.  The adjoint solves
        use opts (default: FP64, rtol 1e-8); their record is kept in
        last_adjoint."""
        lam = np.ascontiguousarray(lam, np.float64)
        nev = lam.size
        ph, mem, keep = _buf(phi, 3 * self.nNode * nev)
        if _is_torch(phi):
            dvdx = phi.new_zeros(self.nElem)
            drho = phi.new_zeros(self.nElem) if want_drho else None
        else:
            dvdx = np.zeros(self.nElem)
            drho = np.zeros(self.nElem) if want_drho else None
        dp_ = lambda a: None if a is None else C.c_void_p(
            a.data_ptr() if _is_torch(a) else a.ctypes.data)
        value = C.c_double(0.0)
        info = L.SolveInfo()
        self._check(self._lib.tpo_buckling_sensitivity(
            self._h, nev, lam.ctypes.data_as(C.POINTER(C.c_double)), ph, float(p),
            None if opts is None else C.byref(opts), C.byref(value), dp_(dvdx),
            dp_(drho), mem, C.byref(info)), "buckling_sensitivity")
        self.last_adjoint = info.as_dict()
        return (value.value, dvdx, drho) if want_drho else (value.value, dvdx)

    def frequency(self, nvals, density, mlump=None, p=8.0, gradient=False, opts=None,
                  **kw):
        """Frequency::Function (Dynamic.cpp:18-171): the largest eigenvalues
        of M phi = lambda K phi with the lumped mass of DiagMassFnc (lambda =
        1/omega^2), more than nvals of them until the last is separated
        (UNIQUE_LAST_NEV); returns (lambda descending, value) or, with
        gradient, (lambda, value, dvalue/dx).  The solver record is kept in
        last_eig."""
        o = opts or L.default_eig_opts(**kw)
        lam = np.zeros(32)
        ncv = C.c_int32(0)
        value = C.c_double(0.0)
        ml, mem, keep = _buf(mlump, 3 * self.nNode)
        if gradient:
            dvdx = (mlump.new_zeros(self.nElem) if _is_torch(mlump) and mem == L.MEM_DEVICE
                    else np.zeros(self.nElem))
            dp_ = C.c_void_p(dvdx.data_ptr() if _is_torch(dvdx) else dvdx.ctypes.data)
        else:
            dvdx, dp_ = None, None
        info = L.EigInfo()
        rc = self._check(self._lib.tpo_frequency(
            self._h, int(nvals), float(density), ml, C.byref(o), float(p),
            lam.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ncv), C.byref(value),
            dp_, mem, C.byref(info)), "frequency")
        self.last_eig = info.as_dict()
        self.last_eig["rc"] = rc
        lam = lam[:ncv.value].copy()
        return (lam, value.value, dvdx) if gradient else (lam, value.value)

    def volume(self, gradient=True):
        v = C.c_double()
        dv = np.zeros(self.nElem) if gradient else None
        self._check(self._lib.tpo_volume(
            self._h, C.byref(v),
            None if dv is None else dv.ctypes.data_as(C.c_void_p), L.MEM_HOST),
            "volume")
        return v.value, dv


# -- functions (Functions.h:16-91, Functions.cpp:39-109) --------------------
class Function_Base:
    def __init__(self, values, min_val, max_val, objective=True,
                 calc_gradient=True):
        self.weights = list(values)
        self.min_val, self.max_val = float(min_val), float(max_val)
        self.objective = bool(objective)
        self.calc_gradient = bool(calc_gradient)
        self.values = [0.0] * len(self.weights)
        self.gradients = None
        self.value, self.gradient = 0.0, None

    def Function(self, topOpt):  # pragma: no cover - abstract
        raise NotImplementedError

    @property
    def name(self):
        """Function_Base::name[func_type] (Functions.cpp:5): the class name
        of Compliance, Volume, Stability, Frequency."""
        return type(self).__name__

    def Compute(self, topOpt):
        """Functions.cpp:39-62: weighted, normalised value and gradient."""
        self.Function(topOpt)
        w = self.weights[0]
        rng = self.max_val - self.min_val
        if self.objective:
            value = w * (self.values[0] - self.min_val)
            grad = None if self.gradients is None else w * self.gradients
        else:
            value = (self.values[0] - self.min_val) - w
            grad = self.gradients
        self.value = value / rng
        self.gradient = None if grad is None else grad / rng

    @staticmethod
    def Function_Call(topOpt):
        """Functions.cpp:77-109 -> (f, dfdx, g, dgdx) over all functions."""
        f, dfdx, g, dgdx = 0.0, np.zeros(topOpt.nElem), [], []
        for fn in topOpt.function_list:
            fn.Compute(topOpt)
            if fn.objective:
                f += fn.value
                dfdx += fn.gradient
            else:
                g.append(fn.value)
                dgdx.append(fn.gradient)
        dg = np.stack(dgdx, axis=1) if dgdx else np.zeros((topOpt.nElem, 0))
        return f, dfdx, np.array(g), dg


class Compliance(Function_Base):
    """Compliance.cpp:15-57"""

    def Function(self, topOpt):
        c, dcdx, _ = topOpt.compliance(gradient=self.calc_gradient)
        self.values[0] = c
        self.gradients = dcdx


class Volume(Function_Base):
    """Volume.cpp:15-41"""

    def __init__(self, values, min_val, max_val, objective=True,
                 calc_gradient=True):
        # constraint values are pre-scaled by the range (Inputs.cpp:554-557)
        if not objective:
            values = [v * (max_val - min_val) for v in values]
        super().__init__(values, min_val, max_val, objective, calc_gradient)

    def Function(self, topOpt):
        v, dv = topOpt.volume(gradient=self.calc_gradient)
        self.values[0] = v
        self.gradients = dv


class Stability(Function_Base):
    """Stability::Function (Buckling.cpp:15-272): the buckling eigenvalues
    of Ks phi = lambda K phi aggregated as (sum lambda^p)^(1/p), p = 8
    (:87-88), and with calc_gradient its design gradient through one
    adjoint solve per eigenpair (:113-272)."""

    def __init__(self, values, min_val, max_val, objective=True,
                 calc_gradient=False, nev=6, block=12):
        super().__init__(values, min_val, max_val, objective, calc_gradient)
        self.nev, self.block = nev, block
        self.lam = None

    def Function(self, topOpt):
        topOpt.ks_assemble()
        p = 8.0
        if self.calc_gradient:
            self.lam, phi = topOpt.buckling(nev=self.nev, block=self.block,
                                            want_vectors=True)
            self.values[0], self.gradients = topOpt.buckling_sensitivity(self.lam, phi, p)
        else:
            self.lam = topOpt.buckling(nev=self.nev, block=self.block)
            self.values[0] = float(np.sum(self.lam ** p) ** (1.0 / p))
            self.gradients = None


class Frequency(Function_Base):
    """Frequency::Function (Dynamic.cpp:18-171): the largest eigenvalues of
    M phi = lambda K phi (the lowest natural frequencies, lambda =
    1/omega^2) with the lumped mass of DiagMassFnc, aggregated as
    (sum lambda^p)^(1/p), p = 8, and with calc_gradient its design gradient
    (no adjoint solve: K and M do not depend on U)."""

    def __init__(self, values, min_val, max_val, objective=True,
                 calc_gradient=True, nvals=4, density=1.0, block=12):
        super().__init__(values, min_val, max_val, objective, calc_gradient)
        self.nvals, self.density, self.block = nvals, density, block
        self.lam = None

    def Function(self, topOpt):
        r = topOpt.frequency(self.nvals, self.density, gradient=self.calc_gradient,
                             block=self.block)
        self.lam, self.values[0] = r[0], r[1]
        self.gradients = r[2] if self.calc_gradient else None


@dataclass
class OC:
    """MMA::Update for m < 2 constraints, i.e. the OC branch (MMA.cpp:87-94,
    103-180), computed on the GPU."""
    n: int
    move: float = 0.5            # MMA default move (MMA.h:21) / Step_Limit
    xmin: np.ndarray = None
    xmax: np.ndarray = None
    miniter: int = 0
    maxiter: int = 50
    minchange: float = 0.0
    iter: int = 0
    Change: float = 1.0
    xval: np.ndarray = field(default=None)

    def __post_init__(self):
        if self.xmin is None:
            self.xmin = np.zeros(self.n)
        if self.xmax is None:
            self.xmax = np.ones(self.n)

    def Update(self, topOpt, dfdx, g, dgdx):
        if g.size != 1:
            raise TopOptError(-4, "the GPU update implements the OC branch (one constraint)")
        x = np.ascontiguousarray(self.xval, np.float64)
        df = np.ascontiguousarray(dfdx, np.float64)
        dg = np.ascontiguousarray(dgdx[:, 0], np.float64)
        ch = C.c_double()
        lib = topOpt._lib
        topOpt._check(lib.tpo_oc_update(
            topOpt._h, x.ctypes.data_as(C.c_void_p),
            self.xmin.ctypes.data_as(C.c_void_p),
            self.xmax.ctypes.data_as(C.c_void_p), df.ctypes.data_as(C.c_void_p),
            float(g[0]), dg.ctypes.data_as(C.c_void_p), float(self.move),
            C.byref(ch), L.MEM_HOST), "OC update")
        self.xval = x
        self.Change = ch.value
        return x

    def Check(self):
        """MMA.h:83-85"""
        if (self.iter > self.miniter) and (self.Change < self.minchange):
            return True
        self.iter += 1
        return self.iter >= self.maxiter


@dataclass
class MMA(OC):
    """MMA::Update (MMA.cpp:62-100): the OC branch for fewer than two
    constraints (as OC), otherwise MMA::MMAsub with MMA::DualSolve
    (:185-595) -- the whole update in one persistent GPU launch.  xold1, xold2, low and upp are the method's state; they start
    from xval as MMA::Set_Values does.  opts: tpo_mma_opts fields (move is
    taken from the dataclass field)."""
    xold1: np.ndarray = None
    xold2: np.ndarray = None
    low: np.ndarray = None
    upp: np.ndarray = None
    fresh_start: bool = True
    mma_opts: dict = field(default_factory=dict)
    newton_steps: int = 0        # dual Newton steps of the last update

    def Update(self, topOpt, dfdx, g, dgdx):
        g = np.atleast_1d(np.asarray(g, np.float64))
        if g.size < 2:
            return super().Update(topOpt, dfdx, g, dgdx)
        n = self.n
        x = np.ascontiguousarray(self.xval, np.float64).copy()
        if self.xold1 is None:
            self.xold1, self.xold2 = x.copy(), x.copy()
            self.low, self.upp = np.zeros(n), np.ones(n)
        st = [np.ascontiguousarray(a, np.float64) for a in
              (self.xold1, self.xold2, self.low, self.upp)]
        df = np.ascontiguousarray(dfdx, np.float64)
        dg = np.asfortranarray(np.asarray(dgdx, np.float64).reshape(n, g.size))
        o = L.default_mma_opts(move=float(self.move), **self.mma_opts)
        fresh = C.c_int32(1 if self.fresh_start else 0)
        ch = C.c_double()
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        topOpt._check(topOpt._lib.tpo_mma_update(
            topOpt._h, C.byref(o), int(self.iter), C.byref(fresh), int(g.size), ptr(x),
            ptr(st[0]), ptr(st[1]), ptr(st[2]), ptr(st[3]), ptr(self.xmin), ptr(self.xmax),
            ptr(df), g.ctypes.data_as(C.POINTER(C.c_double)), ptr(dg), C.byref(ch),
            L.MEM_HOST), "MMA update")
        self.xold1, self.xold2, self.low, self.upp = st
        self.fresh_start = bool(fresh.value)
        steps = C.c_int32()
        topOpt._lib.tpo_mma_last_info(topOpt._h, C.byref(steps))
        self.newton_steps = steps.value
        self.xval = x
        self.Change = ch.value
        return x


_STARS = "*" * 48


def step_out_text(f, cons, it, function_list):
    """The Output.txt entry of TopOpt::StepOut (TopOpt.cpp:386-401)."""
    s = "Iteration number: %d\nObjective: %1.6g\nConstraints:\n" % (it, f)
    s += "".join("\t%1.12g\t" % c for c in cons)
    s += "\nAll function values:\n"
    s += "".join("\t%12s: %1.8g\n" % (fn.name, fn.value) for fn in function_list)
    return s + "\n"


def result_out_text(it, penal, Esum, Vsum):
    """The Output.txt entry of TopOpt::ResultOut (TopOpt.cpp:421-425)."""
    return ("%s\nAfter %4i iterations with a penalty of %1.4g the\n"
            "ratio of stiffness sum to volume sum is %1.4g\n%s\n\n"
            % (_STARS, it, penal, Esum / Vsum, _STARS))


def optimize(topOpt, optmma, penalties=None, opts=None, callback=None, output=None,
             folder=None, print_every=None, index_bytes=4):
    """The optimisation loop of Main.cpp:120-178: per penalty, MatIntFnc ->
    FEAssemble -> FESolve -> Function_Call, then Update + re-evaluate until
    Check() (a do-while, so maxiter updates and maxiter + 1 evaluations).
    FESolve warm-starts from the previous U (FEAnalysis.cpp:389).

    `output` (a path or a text file) receives the Output.txt log: the
    penalty line of Main.cpp:134, StepOut after every evaluation and
    ResultOut after every penalty (TopOpt.cpp:372-435).  With `folder`,
    PrintVals writes the state there every `print_every` iterations
    (_pen<p>_it<i>) and at the end of every penalty (_pen<p>), as StepOut
    and ResultOut do.

    Returns one record per evaluation (the fields StepOut prints plus the
    solver outcome)."""
    hist = []
    penalties = [topOpt.penal] if penalties is None else list(penalties)
    own = isinstance(output, (str, bytes, os.PathLike))
    log = open(output, "w") if own else output
    every = print_every if print_every else 2**31 - 1     # INT_MAX by default
    last_print = 0

    def step_out(f, g, it):
        nonlocal last_print
        last_print += 1
        if every - last_print == 0:
            if folder is not None:
                topOpt.PrintVals("_pen%1.4g_it%i" % (topOpt.penal, it), folder,
                                 index_bytes=index_bytes)
            last_print = 0
        last_print *= it > 0
        if log is not None:
            log.write(step_out_text(f, g, it, topOpt.function_list))

    def result_out(it):
        nonlocal last_print
        if log is not None:
            E = np.zeros(topOpt.nElem)
            V = np.zeros(topOpt.nElem)
            topOpt.get("E", E)
            topOpt.get("rho", V)
            log.write(result_out_text(it, topOpt.penal, E.sum(), V.sum()))
        if folder is not None:
            topOpt.PrintVals("_pen%1.4g" % topOpt.penal, folder, index_bytes=index_bytes)
        last_print = 0

    def evaluate(it):
        topOpt.MatIntFnc(optmma.xval)
        topOpt.FEAssemble(opts)
        info = topOpt.FESolve(opts)
        f, dfdx, g, dgdx = Function_Base.Function_Call(topOpt)
        rec = {"penal": topOpt.penal, "iter": it, "f": f, "g": g.tolist(),
               "values": [fn.values[0] for fn in topOpt.function_list],
               "change": optmma.Change, "solve": info}
        hist.append(rec)
        if callback is not None:
            callback(rec)
        step_out(f, g, it)
        return dfdx, g, dgdx

    try:
        for p in penalties:
            topOpt.penal = float(p)
            if log is not None:
                log.write("\nPenalty increased to %1.3g\n" % topOpt.penal)
            optmma.iter = 0
            dfdx, g, dgdx = evaluate(0)
            while True:
                optmma.Update(topOpt, dfdx, g, dgdx)
                dfdx, g, dgdx = evaluate(optmma.iter + 1)
                if optmma.Check():
                    break
            result_out(optmma.iter)
    finally:
        if own:
            log.close()
    return hist
