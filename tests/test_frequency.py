"""Natural frequencies (Frequency, Dynamic.cpp:18-235): the lumped mass M
of DiagMassFnc and the largest eigenvalues of M phi = lambda K phi
(lambda = 1/omega^2), aggregated as (sum lambda^p)^(1/p), with the design
gradient the reference forms from the first nvals - 1 eigenpairs.

CPU: the oracle's eigenvalue derivatives phi^T (dM - lambda dK) phi against
central differences of a dense generalized eigensolve.

GPU: tpo_frequency (the block eigensolver with M in place of Ks) against the
oracle's dense eigensolve: eigenvalues to 1e-9, the number of pairs the
UNIQUE_LAST_NEV rule keeps, the value and the gradient.
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def oracle_cantilever(oracle, nel, x, levels=2):
    pb = oracle.Problem(nel, rmin=1.5, mg_levels=levels)
    P.apply_bcs(pb, P.cantilever_bcs(nel))
    pb.set_design(x, 3.0, 1e-10)
    pb.assemble(oracle.default_opts(rtol=1e-14, maxit=5000))
    return pb


def test_oracle_frequency_derivatives_match_finite_differences(oracle):
    nel, nvals, density, h = (6, 2, 3), 3, 2.5, 1e-6
    x0 = np.random.default_rng(7).uniform(0.2, 1.0, int(np.prod(nel)))
    pb = oracle_cantilever(oracle, nel, x0)
    lam, value, dvdx, dlam = oracle.frequency_dense(pb, nel, nvals, density)
    assert lam.size >= nvals + 1
    assert abs(value - np.sum(lam ** 8) ** 0.125) <= 1e-14 * value
    # the reference's gradient: the first nvals - 1 pairs, p-norm chain, P^T
    g = np.sum(lam[:nvals - 1, None] ** 7 * dlam[:nvals - 1], axis=0) * value ** -7
    assert rel(dvdx, pb.filter(g, transpose=True)) < 1e-14
    for e in (0, 17, 30):
        xp, xm = x0.copy(), x0.copy()
        xp[e] += h
        xm[e] -= h
        lp = oracle.frequency_dense(oracle_cantilever(oracle, nel, xp), nel, nvals, density)[0]
        lm = oracle.frequency_dense(oracle_cantilever(oracle, nel, xm), nel, nvals, density)[0]
        for j in range(lam.size):
            fd = (lp[j] - lm[j]) / (2 * h)
            an = pb.filter(dlam[j], transpose=True)[e]
            assert abs(an - fd) <= 1e-6 * abs(fd), (e, j, an, fd)


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["fp64", "mixed"])
def test_frequency_matches_oracle(T, oracle, precond):
    nel, nvals, density = (12, 4, 6), 3, 2.5
    x = np.random.default_rng(21).uniform(0.2, 1.0, int(np.prod(nel)))
    pb = oracle_cantilever(oracle, nel, x)
    lam_o, val_o, dvdx_o, _ = oracle.frequency_dense(pb, nel, nvals, density)
    t = T.TopOpt(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(t, P.cantilever_bcs(nel))
    t.FEInitialize()
    t.MatIntFnc(x)
    t.FEAssemble(T.default_opts(rtol=1e-12, maxit=5000))
    pc = T.PREC_FP64 if precond == "fp64" else T.PREC_MIXED
    lam, val, dvdx = t.frequency(nvals, density, gradient=True, tol=1e-10, precond=pc)
    assert t.last_eig["status"] == 0, t.last_eig
    assert lam.size == lam_o.size
    np.testing.assert_allclose(lam, lam_o, rtol=1e-9)
    assert abs(val - val_o) <= 1e-9 * val_o
    assert rel(dvdx, dvdx_o) < 1e-6
    f = T.Frequency([1.0], 0.0, 1.0, objective=True, calc_gradient=True, nvals=nvals,
                    density=density)
    f.Compute(t)
    assert abs(f.values[0] - val) <= 1e-6 * val
    assert rel(f.gradient, dvdx) < 1e-4


@pytest.mark.gpu
def test_frequency_point_masses(T, oracle):
    """Point masses (the reference's MLump) add to the lumped diagonal on
    both sides; a heavier tip lowers every frequency (raises lambda)."""
    nel, nvals, density = (12, 4, 6), 2, 1.0
    x = np.random.default_rng(22).uniform(0.3, 1.0, int(np.prod(nel)))
    pb = oracle_cantilever(oracle, nel, x)
    nn = pb.nn
    ml = np.zeros(3 * nn)
    tip = [n for n in range(nn) if n % (nel[0] + 1) == nel[0]]
    for n in tip:
        ml[3 * n:3 * n + 3] = 0.05
    lam_o, val_o, _, _ = oracle.frequency_dense(pb, nel, nvals, density, mlump=ml)
    lam_free = oracle.frequency_dense(pb, nel, nvals, density)[0]
    assert lam_o[0] > lam_free[0]
    t = T.TopOpt(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(t, P.cantilever_bcs(nel))
    t.FEInitialize()
    t.MatIntFnc(x)
    t.FEAssemble(T.default_opts(rtol=1e-12, maxit=5000))
    lam, val = t.frequency(nvals, density, mlump=ml, tol=1e-10)
    np.testing.assert_allclose(lam, lam_o, rtol=1e-9)
    assert abs(val - val_o) <= 1e-9 * val_o
