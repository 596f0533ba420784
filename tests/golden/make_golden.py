"""Generate the golden fixtures under tests/golden/.

The reference (darinpeetz/TopOpt3D) ships no tests or golden vectors and
cannot be built here (PETSc, SLEPc, ParMETIS, MPI and Eigen are absent), so
the fixtures come from the CPU oracle, cross-checked at generation time by
an independent path: a scipy sparse direct solve of an element-by-element
assembly (numpy K0 from its own Gauss-point loop) with the reference's
Dirichlet treatment.  Generation fails if the two disagree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O          # noqa: E402
from topopt3d_b200 import problems as P  # noqa: E402


def numpy_K0(dx=(1.0, 1.0, 1.0), E0=1.0, nu=0.3):
    """Independent hex8 stiffness: B^T D B at 2x2x2 Gauss points."""
    c = E0 / ((1 + nu) * (1 - 2 * nu))
    D = np.zeros((6, 6))
    D[:3, :3] = nu * c
    np.fill_diagonal(D[:3, :3], (1 - nu) * c)
    D[3, 3] = D[4, 4] = D[5, 5] = E0 / (2 * (1 + nu))
    sg = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    K = np.zeros((24, 24))
    g = 1 / np.sqrt(3)
    h = np.asarray(dx) / 2
    for q in sg * g:
        dN = np.array([[s[0] * (1 + s[1] * q[1]) * (1 + s[2] * q[2]),
                        s[1] * (1 + s[0] * q[0]) * (1 + s[2] * q[2]),
                        s[2] * (1 + s[0] * q[0]) * (1 + s[1] * q[1])]
                       for s in sg]).T / 8 / h[:, None]
        B = np.zeros((6, 24))
        for n in range(8):
            B[0, 3 * n], B[1, 3 * n + 1], B[2, 3 * n + 2] = dN[:, n]
            B[3, 3 * n], B[3, 3 * n + 1] = dN[1, n], dN[0, n]
            B[4, 3 * n + 1], B[4, 3 * n + 2] = dN[2, n], dN[1, n]
            B[5, 3 * n], B[5, 3 * n + 2] = dN[2, n], dN[0, n]
        K += B.T @ D @ B * np.prod(h)
    return K


def direct_solution(nel, E, fixmask, F):
    K0 = numpy_K0()
    ne = int(np.prod(nel))
    Nx, Ny = nel[0] + 1, nel[1] + 1
    rows, cols, vals = [], [], []
    for e in range(ne):
        i, j, k = e % nel[0], (e // nel[0]) % nel[1], e // (nel[0] * nel[1])
        n0 = i + j * Nx + k * Nx * Ny
        nodes = [n0, n0 + 1, n0 + 1 + Nx, n0 + Nx]
        nodes += [v + Nx * Ny for v in nodes]
        dofs = (3 * np.array(nodes)[:, None] + np.arange(3)).ravel()
        rows.append(np.repeat(dofs, 24))
        cols.append(np.tile(dofs, 24))
        vals.append((E[e] * K0).ravel())
    nd = F.size
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                               np.concatenate(cols))), shape=(nd, nd))
    fixed = np.array([3 * n + c for n in range(nd // 3) for c in range(3)
                      if (fixmask[n] >> c) & 1], dtype=np.int64)
    free = np.setdiff1d(np.arange(nd), fixed)
    U = np.zeros(nd)
    U[free] = spl.spsolve(K[free][:, free].tocsc(), F[free])
    return U


def case(name, nel, levels, rmin, x, spec, store_full):
    pb = O.Problem(nel, rmin=rmin, mg_levels=levels)
    P.apply_bcs(pb, spec)
    pb.set_design(x)
    o = O.default_opts(rtol=1e-12, maxit=1000)
    pb.assemble(o)
    U, st, its, rr = pb.solve(opts=o)
    assert st == 0, (name, st)
    C, dCdx, dCdrho = pb.compliance(U)
    V, dVdx = pb.volume()
    rho, E, dEdz = pb.material()
    fm, F = pb.get_bc()
    Ud = direct_solution(nel, E, fm, F)
    err = np.linalg.norm(U - Ud) / np.linalg.norm(Ud)
    assert err < 1e-9, (name, err)
    out = dict(nel=np.array(nel), levels=levels, rmin=rmin, C=C, V=V,
               its=its, fixmask=fm, direct_err=err)
    if store_full:
        out.update(x=x, rho=rho, E=E, dEdz=dEdz, F=F, U=U, dCdx=dCdx,
                   dVdx=dVdx)
    else:
        sel = np.arange(0, pb.ne, 7)
        out.update(sel=sel, dCdx_sel=dCdx[sel], U_norm=np.linalg.norm(U),
                   U_sel=U[::97], dCdx_sum=dCdx.sum(), F_sum=F.sum())
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: C = {C:.15g}, its = {its}, direct rel err = {err:.2e}")


def oc_trajectory(name, cfg, iters, volfrac=0.3, rtol=1e-10):
    """The oracle's optimisation loop on a configuration: per-evaluation
    compliance, volume and change, and a summary of the final design.  The
    solves run to `rtol` (tighter than the 1e-8 default) so that the
    trajectory is pinned well below the solver's own error."""
    c = P.CONFIGS[cfg]
    pb = O.Problem(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(pb, P.bcs(cfg))
    h = O.optimize_oc(pb, P.design(cfg), volfrac, iters,
                      opts=O.default_opts(rtol=rtol, maxit=1000))
    x = h["x"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), cfg=cfg, iters=iters,
                        volfrac=volfrac, rtol=rtol, C=h["C"], V=h["V"], change=h["change"],
                        its=h["its"], x_sum=x.sum(), x_sel=x[::61],
                        x_zero=int((x == 0).sum()))
    print(f"{name}: C[0] = {h['C'][0]:.12g}, C[-1] = {h['C'][-1]:.12g}, "
          f"V[-1] = {h['V'][-1]:.12g}")


def buckling_fixture(name, cfg, nel=None, levels=None, nev=6, dense_check=False):
    """The oracle's buckling eigenvalues (ARPACK over the oracle's Ks and
    PCG + GMG solves) of a configuration's column; small cases are
    cross-checked against a dense generalized eigensolve at generation."""
    import scipy.linalg as sla
    c = P.CONFIGS[cfg]
    nel = nel or c["nel"]
    levels = levels or c["levels"]
    pb = O.Problem(nel, rmin=c["rmin"], mg_levels=levels)
    P.apply_bcs(pb, P.bcs(cfg, nel))
    pb.set_design(P.design(cfg, nel), 3.0, 1e-10)
    o = O.default_opts(rtol=1e-12, maxit=5000)
    pb.assemble(o)
    U, st, its, rr = pb.solve(opts=o)
    assert st == 0, (name, st)
    C, _, _ = pb.compliance(U)
    pb.ks_assemble(U)
    lam, phi = O.buckling(pb, nev=nev)
    out = dict(cfg=cfg, nel=np.array(nel), levels=levels, nev=nev, lam=lam, C=C,
               solve_rtol=1e-12)
    if dense_check:
        n = 3 * pb.nn
        w = sla.eigh(O.dense(pb.ks_apply, n), O.dense(pb.apply, n),
                     eigvals_only=True)[::-1][:nev]
        err = np.max(np.abs(w - lam) / np.abs(w))
        assert err < 1e-10, (name, err)
        out["dense_err"] = err
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: lambda = {np.array2string(lam, precision=12)}")


def main():
    nel = (12, 6, 6)
    x = np.random.default_rng(7).uniform(0.1, 1.0, int(np.prod(nel)))
    case("cantilever_12x6x6", nel, 2, 1.5, x, P.cantilever_bcs(nel), True)
    nel = (9, 5, 4)
    x = np.random.default_rng(8).uniform(0.2, 1.0, int(np.prod(nel)))
    case("column_9x5x4_r2", nel, 2, 2.0, x, P.column_bcs(nel), True)
    nel = P.CONFIGS["cfg0"]["nel"]
    case("cfg0_48x24x24", nel, 3, 1.5, P.design("cfg0"), P.bcs("cfg0"), False)
    oc_trajectory("oc_cfg3_64x32x32", "cfg3", 50)
    buckling_fixture("buckling_column_8x4x8", "cfg4", nel=(8, 4, 8), levels=2,
                     dense_check=True)
    buckling_fixture("buckling_cfg4_96x48x48", "cfg4")


if __name__ == "__main__":
    main()
