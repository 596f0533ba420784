"""CPU tests: the C ABI library loads and exports every declared symbol
(no GPU calls), and the oracle passes its known-answer tests."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "topopt_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"TPO_API[^;(]*?\b(tpo_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes

    from topopt3d_b200 import _lib, build
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 29
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTS)
    # pure-host entry points need no GPU
    L = _lib.load()
    o = _lib.default_opts()
    assert (o.rtol, o.maxit, o.cheb_degree, o.cheb_lo, o.cheb_hi) == (1e-8, 500, 2, 0.1, 1.1)
    assert L.tpo_kernel_launches() >= 0


def test_noalloc_argument_checks_need_no_gpu():
    """The allocation-free sensitivity refuses a null buffer (TPO_E_ARG) and
    a filter radius whose template exceeds its 128 taps (TPO_E_UNSUPPORTED)
    before it touches the GPU, so both answers come back on a CPU host."""
    import ctypes as C

    from topopt3d_b200 import _lib
    L = _lib.load()
    nel = (C.c_int32 * 3)(8, 4, 4)
    dx = (C.c_double * 3)(1.0, 1.0, 1.0)
    msg = C.create_string_buffer(256)
    dummy = C.c_void_p(16)          # never dereferenced: refused first
    rc = L.tpo_sensitivity_noalloc(nel, dx, 1.0, 0.3, 1.5, None, dummy, dummy,
                                   None, msg, 256)
    assert rc == _lib.TPO_E_ARG and b"null buffer" in msg.value
    rc = L.tpo_sensitivity_noalloc(nel, dx, 1.0, 0.3, 6.0, dummy, dummy, dummy,
                                   None, msg, 256)
    assert rc == _lib.TPO_E_UNSUPPORTED and b"128 taps" in msg.value
    for bad in (float("inf"), float("nan"), -1.0):
        rc = L.tpo_sensitivity_noalloc(nel, dx, 1.0, 0.3, bad, dummy, dummy, dummy,
                                       None, msg, 256)
        assert rc in (_lib.TPO_E_ARG, _lib.TPO_E_UNSUPPORTED), bad


def test_level1_form_and_level_apply_refuse_a_null_context():
    """The level-1 form switch and the precision-selectable level apply
    answer TPO_E_ARG for a null context without touching a GPU."""
    import ctypes as C

    from topopt3d_b200 import _lib
    L = _lib.load()
    on = C.c_int32(-1)
    assert L.tpo_set_level1_form(None, 0, C.byref(on)) == _lib.TPO_E_ARG
    assert L.tpo_apply_level_prec(None, 1, None, None, _lib.PREC_MIXED,
                                  _lib.MEM_HOST) == _lib.TPO_E_ARG


def test_k0_anisotropic_elements_decouple(oracle):
    """K0 of box elements with unequal edges and other materials keeps the
    properties the modal apply relies on: symmetric, 6 rigid-body modes,
    the 45-entry Hadamard block pattern, and the patch test."""
    xyz = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    s = 2 * xyz - 1
    H = np.array([[1, a[0], a[1], a[0] * a[1], a[2], a[0] * a[2], a[1] * a[2],
                   a[0] * a[1] * a[2]] for a in s]).T
    Tm = np.kron(H, np.eye(3))
    for dx, E0, nu in (((1.0, 0.5, 2.0), 1.0, 0.3), ((2.0, 1.0, 1.0), 210.0, 0.25),
                       ((1.0, 0.5, 0.75), 3.0, 0.3)):
        K = oracle.element_stiffness(dx, E0, nu)
        sc = np.abs(K).max()
        assert np.abs(K - K.T).max() < 1e-14 * sc
        w = np.linalg.eigvalsh(K)
        assert np.sum(np.abs(w) < 1e-12 * sc) == 6 and w.min() > -1e-12 * sc
        Kh = Tm @ K @ Tm.T / 64
        assert np.sum(np.abs(Kh) > 1e-12 * sc) == 45
        # uniform strain eps_xx = 1 on the physical element: the +x face
        # carries sigma_xx = D[0,0] over its area dy*dz
        D = np.zeros(36)
        oracle.lib().tor_constitutive(E0, nu, D)
        u = np.zeros((8, 3))
        u[:, 0] = xyz[:, 0] * dx[0]
        f = (K @ u.ravel()).reshape(8, 3)
        assert abs(f[xyz[:, 0] == 1, 0].sum() - D[0] * dx[1] * dx[2]) < 1e-12 * sc


# ----------------------------------------------------------------- oracle KATs

def test_k0_known_answers(oracle):
    K = oracle.element_stiffness((1.0, 1.0, 1.0), 1.0, 0.3)
    assert np.abs(K - K.T).max() < 1e-15
    w = np.linalg.eigvalsh(K)
    assert np.sum(np.abs(w) < 1e-12) == 6 and w.min() > -1e-12
    assert np.abs(K.sum(axis=1)[0::3]).max() < 1e-14   # translations
    # rigid rotations are in the null space
    xyz = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    for a, b in ((0, 1), (1, 2), (0, 2)):
        u = np.zeros((8, 3))
        u[:, a], u[:, b] = xyz[:, b], -xyz[:, a]
        assert np.abs(K @ u.ravel()).max() < 1e-14
    # patch test: uniform strain eps_xx = 1 gives the stress sigma = D eps
    D = np.zeros(36)
    oracle.lib().tor_constitutive(1.0, 0.3, D)
    D = D.reshape(6, 6)
    u = np.zeros((8, 3))
    u[:, 0] = xyz[:, 0]
    f = (K @ u.ravel()).reshape(8, 3)
    # nodal forces on the +x face sum to sigma_xx * area
    assert abs(f[xyz[:, 0] == 1, 0].sum() - D[0, 0]) < 1e-13
    # Hadamard-basis sparsity of K0 (45 of 576 couplings)
    H = np.array([[1, s[0], s[1], s[0] * s[1], s[2], s[0] * s[2], s[1] * s[2],
                   s[0] * s[1] * s[2]] for s in 2 * xyz - 1]).T
    Tm = np.kron(H, np.eye(3))
    Kh = Tm @ K @ Tm.T / 64
    assert np.sum(np.abs(Kh) > 1e-12) == 45


def test_element_numbering(oracle):
    nel = (4, 3, 2)
    Nx, Ny = 5, 4
    for e in range(24):
        i, j, k = e % 4, (e // 4) % 3, e // 12
        n0 = i + j * Nx + k * Nx * Ny
        exp = [n0, n0 + 1, n0 + 1 + Nx, n0 + Nx]
        exp += [v + Nx * Ny for v in exp]
        assert list(oracle.element_nodes(nel, e)) == exp


def test_bc_selection(oracle):
    from topopt3d_b200 import problems as P
    nel = (48, 24, 24)
    spec = P.cantilever_bcs(nel)
    sup = oracle.select_nodes(nel, (1, 1, 1), *spec[0][1:4])
    load = oracle.select_nodes(nel, (1, 1, 1), *spec[1][1:4])
    assert sup.size == 25 * 25 and np.all(sup % 49 == 0)
    assert load.size == 25
    assert np.array_equal(load, 48 + 49 * np.arange(25))
    col = P.column_bcs((96, 48, 48))
    top = oracle.select_nodes((96, 48, 48), (1, 1, 1), *col[1][1:4])
    assert top.size == 97 * 49


@pytest.mark.parametrize("R,taps", [(1.5, 19), (2.0, 27)])
def test_filter_template_and_rows(oracle, R, taps):
    nel = (6, 5, 4)
    rp, col, val = oracle.filter_csr(nel, (1, 1, 1), R)
    counts = np.diff(rp)
    assert counts.max() == taps
    sums = np.add.reduceat(val, rp[:-1])
    assert np.abs(sums - 1).max() < 1e-15
    # interior row weights are 1 - d/R normalised
    e = 2 + 2 * 6 + 2 * 30
    raw = val[rp[e]:rp[e + 1]] / val[rp[e]:rp[e + 1]].min()
    assert raw.max() > 1


def test_vecpow_special_cases(oracle):
    assert oracle.vecpow(0.3, 2.0) == 0.3 * 0.3
    assert oracle.vecpow(0.0, 0.0) == 1.0
    assert oracle.vecpow(-1.0, 3.0) == np.inf


def test_prolongation_rows_sum_to_one(oracle):
    from topopt3d_b200 import problems as PR
    P = oracle.Problem((5, 4, 3), mg_levels=2)
    PR.apply_bcs(P, PR.cantilever_bcs((5, 4, 3)))
    P.set_design(np.full(P.ne, 0.5))
    P.assemble(oracle.default_opts())
    n0, d0 = P.level_nodes(0)
    n1, d1 = P.level_nodes(1)
    assert d1 == tuple((d + 1) // 2 for d in d0)
    for f in range(n0):
        s = sum(P.prolong_weight(0, f, c) for c in range(n1))
        assert abs(s - 1) < 1e-15


def test_oracle_solve_against_sparse_direct(oracle):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    from topopt3d_b200 import problems as P
    nel = (10, 5, 5)
    pb = oracle.Problem(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(pb, P.cantilever_bcs(nel))
    x = np.random.default_rng(0).uniform(0.1, 1, pb.ne)
    pb.set_design(x)
    pb.assemble(oracle.default_opts())
    U, st, its, rr = pb.solve()
    assert st == 0 and rr <= 1e-8
    fm, F = pb.get_bc()
    _, E, _ = pb.material()
    K0 = oracle.element_stiffness()
    rows, cols, vals = [], [], []
    for e in range(pb.ne):
        dofs = (3 * oracle.element_nodes(nel, e)[:, None] + np.arange(3)).ravel()
        rows.append(np.repeat(dofs, 24))
        cols.append(np.tile(dofs, 24))
        vals.append((E[e] * K0).ravel())
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))))
    fixed = np.array([3 * n + c for n in range(pb.nn) for c in range(3) if (fm[n] >> c) & 1])
    free = np.setdiff1d(np.arange(3 * pb.nn), fixed)
    Ur = np.zeros(3 * pb.nn)
    Ur[free] = spl.spsolve(K[free][:, free].tocsc(), F[free])
    assert np.linalg.norm(U - Ur) / np.linalg.norm(Ur) < 1e-7
    C, dcdx, dcdr = pb.compliance(U)
    assert abs(C - Ur @ F) / abs(C) < 1e-8


def test_oracle_sensitivity_central_differences(oracle):
    from topopt3d_b200 import problems as P
    nel = (6, 3, 3)
    pb = oracle.Problem(nel, rmin=1.5, mg_levels=1)
    P.apply_bcs(pb, P.cantilever_bcs(nel))
    x0 = np.random.default_rng(1).uniform(0.2, 0.9, pb.ne)
    o = oracle.default_opts(rtol=1e-14, maxit=5)

    def C_of(x):
        pb.set_design(x)
        pb.assemble(o)
        U, st, _, _ = pb.solve(opts=o)
        return pb.compliance(U)

    C0, dc, _ = C_of(x0)
    h = 1e-6
    for e in (0, 7, 20, 41):
        xp, xm = x0.copy(), x0.copy()
        xp[e] += h
        xm[e] -= h
        fd = (C_of(xp)[0] - C_of(xm)[0]) / (2 * h)
        assert abs(fd - dc[e]) < 1e-6 * abs(dc[e]) + 1e-10


def test_oc_update_satisfies_constraint(oracle):
    rng = np.random.default_rng(2)
    n = 500
    x = rng.uniform(0.2, 0.6, n)
    dfdx = -rng.uniform(0, 1, n)
    dgdx = np.full(n, 1.0 / n)
    g = float(x.mean() - 0.3)
    xn, ch = oracle.oc_update(x, dfdx, g, dgdx, 0.2)
    assert np.all(xn >= 0) and np.all(xn <= 1)
    assert np.all(np.abs(xn - x) <= 0.2 + 1e-12)
    assert abs(g + dgdx @ (xn - x)) < 1e-3
    assert abs(ch - np.max(np.abs(xn - x))) < 1e-15
