"""MMA for two or more constraints (MMA::MMAsub with MMA::DualSolve,
MMA.cpp:185-595).

CPU: the oracle's numpy restatement, run as an optimiser on a small convex
problem with two linear constraints, reaches the solution scipy's SLSQP
finds.

GPU: tpo_mma_update against the oracle for consecutive updates on the same
random data (the fresh asymptotes of the first iterations and the adaptive
ones after), with the same number of dual Newton steps, and a compliance
problem with two volume constraints through
`optimize` against the same loop over the oracle.
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P


def new_state(x0, xmin=None, xmax=None):
    n = x0.size
    return {"x": x0.copy(), "xold1": x0.copy(), "xold2": x0.copy(), "low": np.zeros(n),
            "upp": np.ones(n), "xmin": np.zeros(n) if xmin is None else xmin,
            "xmax": np.ones(n) if xmax is None else xmax, "fresh_start": True}


def test_oracle_mma_solves_a_convex_problem(oracle):
    """min sum (x - t)^2 s.t. mean(x) <= 0.4 and mean(x[:n/2]) <= 0.25 over
    [0, 1]^n, by 60 MMA updates, against scipy's SLSQP."""
    from scipy.optimize import minimize
    rng = np.random.default_rng(3)
    n = 40
    t = rng.uniform(0.2, 1.0, n)
    h = n // 2

    def cons(x):
        return np.array([x.mean() - 0.4, x[:h].mean() - 0.25])

    def cons_grad(x):
        g = np.zeros((n, 2))
        g[:, 0] = 1.0 / n
        g[:h, 1] = 1.0 / h
        return g

    st = new_state(np.full(n, 0.3))
    for it in range(60):
        x = st["x"]
        ch = oracle.mma_update(st, 2 * (x - t), cons(x), cons_grad(x), it)
    x = st["x"]
    ref = minimize(lambda v: np.sum((v - t) ** 2), np.full(n, 0.3), jac=lambda v: 2 * (v - t),
                   bounds=[(0, 1)] * n, method="SLSQP",
                   constraints=[{"type": "ineq", "fun": lambda v: -cons(v)}],
                   options={"ftol": 1e-14, "maxiter": 500})
    assert ref.success
    assert np.all(cons(x) <= 1e-6)
    assert np.max(np.abs(x - ref.x)) < 1e-4
    assert ch < 1e-4


def test_oracle_mma_nonlinear_constraints(oracle):
    """min |x|^2 subject to two sphere constraints |x - c_i|^2 <= 9 over
    [0, 5]^3 (the curvature enters both asymptote terms P and Q), by 60
    MMA updates from (4, 3, 2), against scipy's SLSQP."""
    from scipy.optimize import minimize
    c1, c2 = np.array([5.0, 2.0, 1.0]), np.array([3.0, 4.0, 3.0])

    def cons(x):
        return np.array([np.sum((x - c1) ** 2) - 9.0, np.sum((x - c2) ** 2) - 9.0])

    def cons_grad(x):
        return np.stack([2 * (x - c1), 2 * (x - c2)], axis=1)

    x0 = np.array([4.0, 3.0, 2.0])
    st = new_state(x0, np.zeros(3), np.full(3, 5.0))
    for it in range(60):
        x = st["x"]
        oracle.mma_update(st, 2 * x, cons(x), cons_grad(x), it)
    x = st["x"]
    ref = minimize(lambda v: np.sum(v ** 2), x0, jac=lambda v: 2 * v,
                   bounds=[(0, 5)] * 3, method="SLSQP",
                   constraints=[{"type": "ineq", "fun": lambda v: -cons(v),
                                 "jac": lambda v: -cons_grad(v).T}],
                   options={"ftol": 1e-14, "maxiter": 500})
    # SLSQP stops on its line search at this ftol; its point is feasible
    assert np.all(cons(ref.x) <= 1e-9)
    assert np.all(cons(x) <= 1e-6)
    np.testing.assert_allclose(x, ref.x, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("m", [2, 3, 8])
def test_mma_update_matches_oracle(T, oracle, m):
    nel = (12, 6, 6)
    t = T.TopOpt(nel)
    n = t.nElem
    rng = np.random.default_rng(10 + m)
    x0 = rng.uniform(0.2, 0.8, n)
    st_o = new_state(x0)
    mm = T.MMA(n=n)
    mm.xval = x0.copy()
    for it in range(6):
        dfdx = -rng.uniform(0.1, 2.0, n)
        dgdx = rng.uniform(0.0, 1.0, (n, m)) / n
        if m >= 3:
            dgdx[:, 2] -= 0.5 / n          # a constraint with mixed-sign gradient
        g = rng.uniform(-0.05, 0.05, m)
        ch_o = oracle.mma_update(st_o, dfdx, g, dgdx, it)
        prev = mm.xval.copy()
        mm.Update(t, dfdx, g, dgdx)
        mm.iter += 1
        np.testing.assert_allclose(mm.xval, st_o["x"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(mm.low, st_o["low"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(mm.upp, st_o["upp"], rtol=1e-9, atol=1e-12)
        assert np.array_equal(mm.xold1, prev)
        np.testing.assert_allclose(mm.xold1, st_o["xold1"], rtol=0, atol=1e-9)
        assert abs(mm.Change - ch_o) <= 1e-9
        assert mm.fresh_start == st_o["fresh_start"]
        assert mm.newton_steps == st_o["newton_steps"] > 0


@pytest.mark.gpu
def test_mma_compliance_two_volume_constraints(T, oracle):
    """Compliance with V <= 0.3 and V <= 0.35 (m = 2, the MMA branch) on a
    24x12x12 cantilever: 8 updates through `optimize` against the same loop
    over the oracle (solves to 1e-10, warm-started): compliance to 1e-7 at
    every evaluation, and the volume ends at the active limit."""
    nel, iters, limits = (24, 12, 12), 8, (0.3, 0.35)
    x0 = np.full(int(np.prod(nel)), 0.3)
    spec = P.cantilever_bcs(nel)
    t = T.TopOpt(nel, mg_levels=3)
    P.apply_bcs(t, spec)
    t.FEInitialize()
    t.function_list = [T.Compliance([1.0], 0.0, 1.0, True, True)] + \
        [T.Volume([v], 0.0, 1.0, False, True) for v in limits]
    mm = T.MMA(n=t.nElem, maxiter=iters)
    mm.xval = x0.copy()
    hist = T.optimize(t, mm, opts=T.default_opts(rtol=1e-10, maxit=2000))
    C_gpu = np.array([h["values"][0] for h in hist])

    pb = oracle.Problem(nel, mg_levels=3)
    P.apply_bcs(pb, spec)
    o = oracle.default_opts(rtol=1e-10, maxit=2000)
    st = new_state(x0)
    U, C_o = None, []
    for it in range(iters + 1):
        pb.set_design(st["x"], 3.0, 1e-10)
        pb.assemble(o)
        U, s, _, _ = pb.solve(U0=U, opts=o)
        assert s == 0
        C, dC, _ = pb.compliance(U)
        V, dV = pb.volume()
        C_o.append(C)
        if it < iters:
            oracle.mma_update(st, dC, np.array([V - v for v in limits]),
                              np.stack([dV, dV], axis=1), it)
    np.testing.assert_allclose(C_gpu, np.array(C_o), rtol=1e-7)
    assert C_gpu[-1] < C_gpu[0]
    assert abs(hist[-1]["values"][1] - limits[0]) < 5e-3


@pytest.mark.gpu
def test_mma_abi_one_constraint_and_limits(T, oracle):
    """tpo_mma_update is MMAsub for any 1 <= m <= 8 (MMA::Update sends
    m < 2 to OCsub before it, as the MMA classes do): m = 1 against the
    oracle over four updates; m = 0 and m = 9 are refused."""
    import ctypes as C
    from topopt3d_b200 import _lib as L
    t = T.TopOpt((8, 4, 4))
    n = t.nElem
    rng = np.random.default_rng(5)
    x0 = rng.uniform(0.2, 0.8, n)
    st_o = new_state(x0)
    state = [x0.copy(), x0.copy(), x0.copy(), np.zeros(n), np.ones(n)]
    bounds = [np.zeros(n), np.ones(n)]
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    opts = L.default_mma_opts()
    fresh, ch = C.c_int32(1), C.c_double()

    def call(m, dfdx, g, dgdx, it):
        gg = np.ascontiguousarray(g, np.float64)
        return t._lib.tpo_mma_update(t._h, C.byref(opts), it, C.byref(fresh), m,
                                     *[ptr(a) for a in state], *[ptr(a) for a in bounds],
                                     ptr(dfdx), gg.ctypes.data_as(C.POINTER(C.c_double)),
                                     ptr(np.asfortranarray(dgdx)), C.byref(ch), L.MEM_HOST)

    for it in range(4):
        dfdx = -rng.uniform(0.1, 2.0, n)
        dgdx = rng.uniform(0.0, 1.0, (n, 1)) / n
        g = rng.uniform(-0.05, 0.05, 1)
        ch_o = oracle.mma_update(st_o, dfdx, g, dgdx, it)
        assert call(1, dfdx, g, dgdx, it) == 0
        np.testing.assert_allclose(state[0], st_o["x"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(state[3], st_o["low"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(state[4], st_o["upp"], rtol=1e-9, atol=1e-12)
        assert abs(ch.value - ch_o) <= 1e-9
        assert bool(fresh.value) == st_o["fresh_start"]
    dfdx = -np.ones(n)
    for m in (0, 9):
        assert call(m, dfdx, np.zeros(max(m, 1)), np.zeros((n, max(m, 1))), 0) < 0
        assert b"1 <= m <= 8" in t._lib.tpo_last_error(t._h)
