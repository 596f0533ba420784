"""The FP32 level-1 operator on the tensor cores (kernels_l1tc.cu): the
matrix-free form sum_E sum_i E_i G_i u_E plus the correction rows of the
nodes next to fixed dofs, against the oracle's assembled Galerkin level 1
(FEAnalysis.cpp:410-416) and against the stored FP32 stencil it replaces.

The mesh is 128 x 64 x 64 (level 1: 65 x 33 x 33 nodes, above the
persistent coarse levels, so the tensor-core form is the one the V-cycle
uses).  Tolerances: FP32 operator 1e-5 relative to max |y| (as the FP32
fine apply); the two FP32 forms agree to 2e-6; mixed solves with either
form match the oracle to 1e-6 (U) and 1e-8 (C) and take the same CG
iteration count to within one.
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P

pytestmark = pytest.mark.gpu

NEL = (128, 64, 64)
LEVELS = 4


def mixed_spec(nel):
    """A clamped patch in the middle of the x = 0 face, a y-roller on the
    y = 0 face and the cantilever edge load: fixed dofs of one and of all
    three components inside tiles and across tile edges."""
    nx, ny, nz = nel
    return [
        ("support", (0.0, ny / 2, nz / 2), (P.TINY, ny / 4, nz / 4), P.OPEN,
         (1.0, 1.0, 1.0)),
        ("support", (0.0, 0.0, 0.0), (P.BIG, P.TINY, P.BIG), P.OPEN,
         (0.0, 1.0, 0.0)),
        ("load", (float(nx), 0.0, 0.0), (P.TINY, P.BIG, P.TINY), P.OPEN,
         (0.0, 0.0, -1.0 / (ny + 1))),
    ]


SPECS = {
    "cantilever": P.cantilever_bcs,
    "column": P.column_bcs,
    "mixed": mixed_spec,
}


def make(T, O, spec, seed, lo=0.05):
    ne = int(np.prod(NEL))
    x = np.random.default_rng(seed).uniform(lo, 1.0, ne)
    ref = O.Problem(NEL, rmin=1.5, mg_levels=LEVELS)
    P.apply_bcs(ref, spec)
    ref.set_design(x, 3.0, 1e-10)
    ref.assemble(O.default_opts())
    t = T.TopOpt(NEL, rmin=1.5, mg_levels=LEVELS)
    P.apply_bcs(t, spec)
    t.FEInitialize()
    t.MatIntFnc(x)
    t.FEAssemble()
    return t, ref


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("bc", sorted(SPECS))
def test_level1_tensor_form_matches_oracle_and_stencil(T, oracle, bc):
    t, ref = make(T, oracle, SPECS[bc](NEL), seed=11)
    n1 = ref.level_nodes(1)[0]
    u = np.random.default_rng(5).standard_normal(3 * n1)
    y_ref = ref.apply_level(1, u)
    assert t.set_level1_form(0) is True
    y_tc = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    assert t.set_level1_form(1) is False
    y_st = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    t.set_level1_form(0)
    assert rel(y_tc, y_ref) < 1e-5
    assert rel(y_st, y_ref) < 1e-5
    assert rel(y_tc, y_st) < 2e-6
    assert rel(t.apply_level(1, u, np.zeros_like(u)), y_ref) < 1e-12   # FP64 unchanged


def test_level1_tensor_form_is_deterministic(T, oracle):
    t, ref = make(T, oracle, mixed_spec(NEL), seed=12)
    n1 = ref.level_nodes(1)[0]
    u = np.random.default_rng(6).standard_normal(3 * n1)
    a = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    b = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("bc", ["cantilever", "mixed"])
def test_mixed_solve_with_tensor_level1(T, oracle, bc):
    # densities in [0.2, 1]: with [0.05, 1] the oracle's own PCG breaks down
    # here (its 15-step power estimate of lambda_max is too low for that
    # contrast and the Chebyshev smoother stops being positive definite)
    t, ref = make(T, oracle, SPECS[bc](NEL), seed=13, lo=0.2)
    Uo, st, its_o, _ = ref.solve()
    assert st == 0
    out = {}
    for form in (0, 1):
        t.set_level1_form(form)
        t.FEAssemble(T.default_opts(precision=T.PREC_MIXED))
        t.set("U", np.zeros(3 * t.nNode))
        info = t.FESolve(T.default_opts(precision=T.PREC_MIXED))
        assert info["status"] == 0
        out[form] = (t.U.copy(), info["iterations"], t.compliance(gradient=False)[0])
    t.set_level1_form(0)
    Co = ref.compliance(Uo)[0]
    for form in (0, 1):
        U, its, C = out[form]
        assert rel(U, Uo) < 1e-6
        assert abs(C - Co) <= 1e-8 * abs(Co)
    assert abs(out[0][1] - out[1][1]) <= 1


def test_level1_tensor_form_anisotropic_elements_and_material(T, oracle):
    """Element edges (1, 0.5, 2), E0 = 210, nu = 0.25: the 8 blocks G_i come
    from that K0, so the tensor-core operator must still match the oracle's
    Galerkin level 1 and the stored FP32 stencil."""
    dx, E0, nu = (1.0, 0.5, 2.0), 210.0, 0.25
    spec = P.cantilever_bcs(NEL, dx)
    ne = int(np.prod(NEL))
    x = np.random.default_rng(14).uniform(0.05, 1.0, ne)
    ref = oracle.Problem(NEL, dx=dx, E0=E0, nu=nu, rmin=1.5, mg_levels=LEVELS)
    P.apply_bcs(ref, spec)
    ref.set_design(x, 3.0, 1e-10)
    ref.assemble(oracle.default_opts())
    t = T.TopOpt(NEL, dx=dx, E0=E0, Nu0=nu, rmin=1.5, mg_levels=LEVELS)
    P.apply_bcs(t, spec)
    t.FEInitialize()
    t.MatIntFnc(x)
    t.FEAssemble()
    n1 = ref.level_nodes(1)[0]
    u = np.random.default_rng(7).standard_normal(3 * n1)
    y_ref = ref.apply_level(1, u)
    assert t.set_level1_form(0) is True
    y_tc = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    t.set_level1_form(1)
    y_st = t.apply_level(1, u, np.zeros_like(u), precision=T.PREC_MIXED)
    t.set_level1_form(0)
    assert rel(y_tc, y_ref) < 1e-5
    assert rel(y_tc, y_st) < 2e-6


def test_level1_form_needs_even_counts(T):
    t = T.TopOpt((127, 64, 64), rmin=1.5, mg_levels=LEVELS)
    assert t.set_level1_form(0) is False
    with pytest.raises(T.TopOptError, match="form must be 0"):
        t.set_level1_form(2)
