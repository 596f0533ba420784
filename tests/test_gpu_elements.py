"""Element shapes and materials other than the unit cube with E0 = 1,
nu = 0.3, against the oracle.

The reference builds D from E0 and nu (RecMesh.cpp:443-463) and K0 from the
element edges Dimensions/NEL (Inputs.cpp:284,364; FEAnalysis.cpp:869-1050);
the filter template takes the same edges (Filter.cpp:28-52).  Each case
runs the whole path on a small cantilever whose coordinates are physical:

  apply (FP64 1e-13, FP32 2e-5), filter and SIMP (1e-14), Galerkin levels
  (1e-12), V-cycle (1e-10), FP64 solve U / C / dC (1e-8), mixed solve
  (U, dC 1e-6; C 1e-8), stress stiffness apply (1e-12).
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P

pytestmark = pytest.mark.gpu

CASES = [
    # nel, dx, E0, nu, rmin (physical)
    ((16, 12, 6), (1.0, 0.5, 2.0), 1.0, 0.3, 1.5),
    ((12, 12, 12), (2.0, 1.0, 1.0), 210.0, 0.25, 2.5),
    ((16, 10, 8), (1.0, 0.5, 0.75), 3.0, 0.3, 1.2),
]
IDS = ["dx1-0.5-2", "dx2-1-1_E210_nu0.25", "dx1-0.5-0.75_E3"]


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def nrel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def make_pair(T, O, nel, dx, E0, nu, rmin, levels=2, seed=5):
    x = np.random.default_rng(seed).uniform(0.05, 1.0, int(np.prod(nel)))
    spec = P.cantilever_bcs(nel, dx)
    ref = O.Problem(nel, dx=dx, E0=E0, nu=nu, rmin=rmin, mg_levels=levels)
    P.apply_bcs(ref, spec)
    ref.set_design(x, 3.0, 1e-10)
    ref.assemble(O.default_opts())
    t = T.TopOpt(nel, dx=dx, E0=E0, Nu0=nu, rmin=rmin, mg_levels=levels)
    P.apply_bcs(t, spec)
    t.FEInitialize()
    t.MatIntFnc(x)
    t.FEAssemble()
    return t, ref


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_operators_match_oracle(T, oracle, case):
    nel, dx, E0, nu, rmin = case
    t, ref = make_pair(T, oracle, nel, dx, E0, nu, rmin)
    fm_t, F_t = t.get_bc()
    fm_o, F_o = ref.get_bc()
    assert np.array_equal(fm_t, fm_o) and np.array_equal(F_t, F_o)
    assert fm_t.any() and np.count_nonzero(F_t) == nel[1] + 1
    rng = np.random.default_rng(1)
    v = rng.standard_normal(t.nElem)
    assert rel(t.filter(v), ref.filter(v)) < 1e-14
    assert rel(t.filter(v, transpose=True), ref.filter(v, transpose=True)) < 1e-14
    rho_o, E_o, dE_o = ref.material()
    assert rel(t.rho, rho_o) < 1e-14 and rel(t.E, E_o) < 1e-14
    u = rng.standard_normal(3 * t.nNode)
    y_ref = ref.apply(u)
    assert rel(t.apply(u, np.zeros_like(u)), y_ref) < 1e-13
    assert rel(t.apply(u, np.zeros_like(u), precision=T.PREC_MIXED), y_ref) < 2e-5
    n1 = ref.level_nodes(1)[0]
    u1 = rng.standard_normal(3 * n1)
    assert rel(t.apply_level(1, u1, np.zeros_like(u1)), ref.apply_level(1, u1)) < 1e-12
    r = rng.standard_normal(3 * t.nNode)
    assert rel(t.vcycle(r, np.zeros_like(r)), ref.vcycle(r)) < 1e-10


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_solve_and_sensitivity_match_oracle(T, oracle, case):
    nel, dx, E0, nu, rmin = case
    t, ref = make_pair(T, oracle, nel, dx, E0, nu, rmin)
    Uo, st, its_o, _ = ref.solve()
    assert st == 0
    Co, dco, _ = ref.compliance(Uo)
    for prec, tol in ((T.PREC_FP64, 1e-8), (T.PREC_MIXED, 1e-6)):
        t.set("U", np.zeros(3 * t.nNode))
        info = t.FESolve(T.default_opts(precision=prec))
        assert info["status"] == 0 and info["relres"] <= 1e-8
        C, dc, _ = t.compliance()
        assert abs(C - Co) / abs(Co) < 1e-8
        assert nrel(t.U, Uo) < tol
        assert nrel(dc, dco) < tol
        if prec == T.PREC_FP64:
            assert abs(info["iterations"] - its_o) <= 2
    # stress stiffness from the FP64 solution
    t.set("U", Uo)
    t.ks_assemble()
    ref.ks_assemble(Uo)
    w = np.random.default_rng(3).standard_normal(3 * t.nNode)
    assert rel(t.ks_apply(w, np.zeros_like(w)), ref.ks_apply(w)) < 1e-12
