"""Linear buckling (Stability, Buckling.cpp:15-414): the stress stiffness Ks
and the largest eigenvalues of Ks phi = lambda K phi.

CPU: the oracle's literal element ks (G and sigtos as the reference builds
them) against an independent numpy form (the scalar matrix
H = sum_q grad N^T sigma grad N detJ, ks = H (x) I_3), and the oracle's
eigenvalues against the committed fixtures (tests/golden/make_golden.py:
ARPACK over the oracle, cross-checked by a dense generalized eigensolve on
the small column).

GPU: Ks apply against the oracle's assembled Ks to round-off, and the
LOBPCG eigenvalues against the fixtures to 1e-6 relative (the bar for the
96x48x48 column; in practice they agree far closer), with the eigenpair
residuals checked through the C ABI.
"""
import os

import numpy as np
import pytest

from topopt3d_b200 import problems as P

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def fixture(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def numpy_ks(u, E0=1.0, nu=0.3):
    """Independent element stress stiffness for u in the reference local
    node order: H (x) I_3 with H = sum_q grad N^T sigma grad N detJ."""
    c = E0 / ((1 + nu) * (1 - 2 * nu))
    lam_, mu = nu * c, E0 / (2 * (1 + nu))
    sg = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    g = 1 / np.sqrt(3)
    U = u.reshape(8, 3)
    H = np.zeros((8, 8))
    for q in sg * g:
        dN = np.array([[s[0] * (1 + s[1] * q[1]) * (1 + s[2] * q[2]),
                        s[1] * (1 + s[0] * q[0]) * (1 + s[2] * q[2]),
                        s[2] * (1 + s[0] * q[0]) * (1 + s[1] * q[1])]
                       for s in sg]).T / 8 * 2      # 3 x 8, unit cube
        F = U.T @ dN.T                               # F[c][a] = du_c/dx_a
        eps = 0.5 * (F + F.T)
        sig = lam_ * np.trace(eps) * np.eye(3) + 2 * mu * eps
        H += dN.T @ sig @ dN / 8.0                   # detJ = 1/8
    return np.kron(H, np.eye(3))


def test_oracle_ks_element_matches_numpy(oracle):
    rng = np.random.default_rng(11)
    for _ in range(3):
        u = rng.standard_normal(24)
        ks = oracle.stress_stiffness_element(u)
        ref = numpy_ks(u)
        assert np.abs(ks - ref).max() < 1e-13 * np.abs(ref).max()
    # a rigid translation carries no stress
    assert np.abs(oracle.stress_stiffness_element(np.tile([1.0, -2.0, 0.5], 8))).max() < 1e-14


def test_oracle_buckling_reproduces_fixture(oracle):
    g = fixture("buckling_column_8x4x8")
    nel = tuple(int(v) for v in g["nel"])
    c = P.CONFIGS[str(g["cfg"])]
    pb = oracle.Problem(nel, rmin=c["rmin"], mg_levels=int(g["levels"]))
    P.apply_bcs(pb, P.bcs(str(g["cfg"]), nel))
    pb.set_design(P.design(str(g["cfg"]), nel), 3.0, 1e-10)
    o = oracle.default_opts(rtol=float(g["solve_rtol"]), maxit=5000)
    pb.assemble(o)
    U, st, _, _ = pb.solve(opts=o)
    pb.ks_assemble(U)
    lam, _ = oracle.buckling(pb, nev=int(g["nev"]))
    np.testing.assert_allclose(lam, g["lam"], rtol=1e-9)
    assert float(g["dense_err"]) < 1e-10


def oracle_column(oracle, nel, levels, rtol=1e-14, x=None):
    """The cfg4 column on the oracle: design set, assembled, U solved, Ks
    built.  Returns (problem, U)."""
    c = P.CONFIGS["cfg4"]
    pb = oracle.Problem(nel, rmin=c["rmin"], mg_levels=levels)
    P.apply_bcs(pb, P.bcs("cfg4", nel))
    pb.set_design(P.design("cfg4", nel) if x is None else x, 3.0, 1e-10)
    o = oracle.default_opts(rtol=rtol, maxit=5000)
    pb.assemble(o)
    U, st, _, _ = pb.solve(opts=o)
    assert st == 0
    pb.ks_assemble(U)
    return pb, U


def test_oracle_buckling_sensitivity_matches_finite_differences(oracle):
    """The oracle's restatement of the gradient (Buckling.cpp:113-272 with
    the filter chain rule) against central differences of the aggregated
    value, each evaluation a full design -> U -> Ks -> dense eigensolve."""
    nel, nev, h = (4, 2, 6), 3, 1e-5
    x0 = P.design("cfg4", nel)
    pb, U = oracle_column(oracle, nel, 2, x=x0)
    lam, phi = oracle.buckling_dense(pb, nev)
    assert lam[-1] > 1.05 * oracle.buckling_dense(pb, nev + 1)[0][-1]  # a gap
    value, dvdx, _ = oracle.buckling_sensitivity(pb, nel, U, lam, phi)
    assert abs(value - np.sum(lam ** 8) ** 0.125) <= 1e-14 * value

    def agg(x):
        q, _ = oracle_column(oracle, nel, 2, x=x)
        return np.sum(oracle.buckling_dense(q, nev)[0] ** 8) ** 0.125

    for e in (0, 7, 20, 33, 47):
        xp, xm = x0.copy(), x0.copy()
        xp[e] += h
        xm[e] -= h
        fd = (agg(xp) - agg(xm)) / (2 * h)
        assert abs(dvdx[e] - fd) <= 1e-7 * abs(fd), (e, dvdx[e], fd)


def gpu_problem(T, g, precision_rtol=1e-12):
    nel = tuple(int(v) for v in g["nel"])
    cfg = str(g["cfg"])
    c = P.CONFIGS[cfg]
    t = T.TopOpt(nel, rmin=c["rmin"], mg_levels=int(g["levels"]))
    P.apply_bcs(t, P.bcs(cfg, nel))
    t.FEInitialize()
    t.MatIntFnc(P.design(cfg, nel))
    o = T.default_opts(rtol=precision_rtol, maxit=5000)
    t.FEAssemble(o)
    info = t.FESolve(o)
    assert info["status"] == 0
    t.ks_assemble()
    return t


@pytest.mark.gpu
def test_ks_apply_matches_oracle(T, oracle):
    """Ks from the same U on both sides, applied to 5 random columns."""
    nel = (10, 6, 9)
    spec = P.column_bcs(nel)
    x = np.random.default_rng(21).uniform(0.2, 1.0, int(np.prod(nel)))
    ref = oracle.Problem(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(ref, spec)
    ref.set_design(x, 3.0, 1e-10)
    o = oracle.default_opts(rtol=1e-13, maxit=2000)
    ref.assemble(o)
    U, st, _, _ = ref.solve(opts=o)
    ref.ks_assemble(U)
    t = T.TopOpt(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(t, spec)
    t.FEInitialize()
    t.MatIntFnc(x)
    t.set("U", U)
    t.ks_assemble()
    rng = np.random.default_rng(5)
    u = rng.standard_normal((5, 3 * t.nNode))
    y = np.zeros_like(u)
    t.ks_apply(u, y, nrhs=5)
    for j in range(5):
        yo = ref.ks_apply(u[j])
        assert np.abs(y[j] - yo).max() <= 1e-12 * np.abs(yo).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["fp64", "mixed"])
def test_buckling_small_column(T, precond):
    g = fixture("buckling_column_8x4x8")
    t = gpu_problem(T, g)
    pc = T.PREC_FP64 if precond == "fp64" else T.PREC_MIXED
    lam, phi = t.buckling(want_vectors=True, nev=int(g["nev"]), block=12,
                          tol=1e-8, precond=pc)
    assert t.last_eig["status"] == 0, t.last_eig
    np.testing.assert_allclose(lam, g["lam"], rtol=1e-9)
    # eigenpair residuals and K-orthonormality through the ABI
    n = phi.shape[1]
    A = np.zeros_like(phi)
    B = np.zeros_like(phi)
    t.ks_apply(phi, A, nrhs=phi.shape[0])
    t.apply(phi, B, nrhs=phi.shape[0])
    for j in range(phi.shape[0]):
        r = A[j] - lam[j] * B[j]
        assert np.linalg.norm(r) <= 1e-7 * abs(lam[j]) * np.linalg.norm(B[j])
    G = phi @ B.T
    assert np.abs(G - np.eye(phi.shape[0])).max() < 1e-8
    assert n == 3 * t.nNode


@pytest.mark.gpu
@pytest.mark.parametrize("block", [5, 16, 32])
def test_buckling_block_widths(T, block):
    """The block eigensolver's tall-skinny kernels at other widths (5: a
    partly filled accumulator block, 16, and 32, the largest block the ABI
    takes, with its two-by-two Gram super-tiles): the same eigenvalues as
    the golden fixture."""
    g = fixture("buckling_column_8x4x8")
    t = gpu_problem(T, g)
    nev = min(int(g["nev"]), block)
    lam = t.buckling(nev=nev, block=block, tol=1e-8)
    assert t.last_eig["status"] == 0, t.last_eig
    np.testing.assert_allclose(lam, g["lam"][:nev], rtol=1e-9)


@pytest.mark.gpu
def test_buckling_cfg4(T):
    """The 96x48x48 column (698,691 dof): the 6 largest lambda, block 12,
    against the oracle's ARPACK eigenvalues to 1e-6 relative."""
    g = fixture("buckling_cfg4_96x48x48")
    t = gpu_problem(T, g)
    lam = t.buckling(nev=int(g["nev"]), block=12)
    assert t.last_eig["status"] == 0, t.last_eig
    np.testing.assert_allclose(lam, g["lam"], rtol=1e-6)


@pytest.mark.gpu
def test_stability_function(T):
    g = fixture("buckling_column_8x4x8")
    t = gpu_problem(T, g)
    f = T.Stability([1.0], 0.0, 1.0, objective=True, calc_gradient=False)
    f.Compute(t)
    expect = np.sum(np.asarray(g["lam"]) ** 8) ** (1 / 8)
    assert abs(f.values[0] - expect) <= 1e-8 * expect
    assert f.gradient is None


@pytest.mark.gpu
def test_buckling_sensitivity_matches_oracle(T, oracle):
    """The gradient through the C ABI from the same eigenpairs as the oracle
    (the oracle's dense eigensolve of the 8x4x8 column, passed in as host
    and as device buffers): value to round-off, dvdx and dvdrho to 1e-8."""
    import torch
    g = fixture("buckling_column_8x4x8")
    nel, levels, nev = tuple(int(v) for v in g["nel"]), int(g["levels"]), 4
    pb, U = oracle_column(oracle, nel, levels)
    lam, phi = oracle.buckling_dense(pb, nev)
    val_o, dvdx_o, drho_o = oracle.buckling_sensitivity(pb, nel, U, lam, phi)
    t = gpu_problem(T, g)
    o = T.default_opts(rtol=1e-12, maxit=5000)
    val, dvdx, drho = t.buckling_sensitivity(lam, phi, opts=o, want_drho=True)
    assert abs(val - val_o) <= 1e-14 * val_o
    assert rel(dvdx, dvdx_o) < 1e-8 and rel(drho, drho_o) < 1e-8
    assert t.last_adjoint["status"] == 0
    dev = torch.tensor(phi, device="cuda")
    val_d, dvdx_d = t.buckling_sensitivity(lam, dev, opts=o)
    assert val_d == val and rel(dvdx_d.cpu().numpy(), dvdx) < 1e-12


@pytest.mark.gpu
def test_stability_gradient_finite_differences(T):
    """Stability with calc_gradient on the GPU's own eigenpairs against
    central differences of the whole GPU pipeline (MatIntFnc, FEAssemble,
    FESolve, Ks, LOBPCG) on the 8x4x8 column."""
    g = fixture("buckling_column_8x4x8")
    nel, cfg = tuple(int(v) for v in g["nel"]), str(g["cfg"])
    x0 = P.design(cfg, nel)
    t = gpu_problem(T, g)
    eig = dict(nev=4, block=12, tol=1e-10)
    lam, phi = t.buckling(want_vectors=True, **eig)
    assert t.last_eig["status"] == 0
    value, dvdx = t.buckling_sensitivity(lam, phi, opts=T.default_opts(rtol=1e-12, maxit=5000))
    o = T.default_opts(rtol=1e-12, maxit=5000)

    def agg(x):
        t.MatIntFnc(x)
        t.FEAssemble(o)
        t.set("U", np.zeros(3 * t.nNode))
        assert t.FESolve(o)["status"] == 0
        t.ks_assemble()
        return np.sum(t.buckling(**eig) ** 8) ** 0.125

    h = 1e-5
    for e in (3, 100, 200):
        xp, xm = x0.copy(), x0.copy()
        xp[e] += h
        xm[e] -= h
        fd = (agg(xp) - agg(xm)) / (2 * h)
        assert abs(dvdx[e] - fd) <= 1e-6 * abs(fd), (e, dvdx[e], fd)
    t.MatIntFnc(x0)
    t.FEAssemble(o)
    t.set("U", np.zeros(3 * t.nNode))
    t.FESolve(o)
    f = T.Stability([1.0], 0.0, 1.0, objective=True, calc_gradient=True, nev=4)
    f.Compute(t)
    assert abs(f.values[0] - value) <= 1e-8 * value
    assert rel(f.gradient, dvdx) < 1e-5
