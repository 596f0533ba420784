"""Multi-right-hand-side solves and applies through the C ABI (tpo_solve /
tpo_apply with nrhs > 1): a block of columns shares every operator read,
V-cycle launch and grid barrier, with per-column CG scalars and
convergence.

Parity: each column against the oracle's single solve (1e-8 relative, as
the single-RHS tests), and on the 128x64x64 multi-load workload -- whose
hierarchy runs the half-stored stencil level and the persistent coarse
kernel with every block width -- against block-1 solves of the same
columns and against the FP64 residual of the returned solutions.
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P

from test_gpu_parity import pair, rel

pytestmark = pytest.mark.gpu


def solve_cols(T, t, F, block, precision=None, U0=None, rtol=1e-8):
    nrhs = F.shape[0]
    U = np.zeros_like(F) if U0 is None else U0.copy()
    opts = T.default_opts(rtol=rtol, rhs_block=block)
    if precision is not None:
        opts.precision = precision
    info = t.solve(np.ascontiguousarray(F), U, nrhs=nrhs, opts=opts)
    return U, info


def true_relres(T, t, F, U):
    KU = np.zeros_like(U)
    t.apply(np.ascontiguousarray(U), KU, nrhs=U.shape[0])
    return np.array([np.linalg.norm(F[j] - KU[j]) / np.linalg.norm(F[j])
                     for j in range(F.shape[0])])


@pytest.mark.parametrize("block", [2, 4, 8])
def test_blocks_match_oracle(T, oracle, block):
    nel = (16, 8, 8)
    t, ref = pair(T, oracle, nel, levels=3, spec=P.bcs("cfg2", nel), seed=12)
    F = P.point_loads(nel, 8, seed=2)
    U, info = solve_cols(T, t, F, block)
    assert info["status"] == 0
    for j in range(F.shape[0]):
        Uo, st, _, _ = ref.solve(b=F[j])
        assert st == 0
        assert np.linalg.norm(U[j] - Uo) / np.linalg.norm(Uo) < 1e-8


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cfg2_blocks_agree_with_single(T, prec):
    """8 point loads on the 128x64x64 workload: blocks of 8, 4 (and the
    autotuned choice) give the block-1 solutions, every column reaches the
    FP64 residual target, and the iteration totals agree."""
    c = P.CONFIGS["cfg2"]
    nel = c["nel"]
    t = T.TopOpt(nel, rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(t, P.bcs("cfg2"))
    t.FEInitialize()
    t.MatIntFnc(P.design("cfg2"))
    t.FEAssemble()
    F = P.point_loads(nel, 8, seed=2)
    precision = T.PREC_FP64 if prec == "fp64" else T.PREC_MIXED
    U1, i1 = solve_cols(T, t, F, 1, precision)
    assert i1["status"] == 0
    for block in (8, 4, 0):
        Ub, ib = solve_cols(T, t, F, block, precision)
        assert ib["status"] == 0
        rr = true_relres(T, t, F, Ub)
        assert np.all(rr <= 1e-8), rr
        for j in range(8):
            # both solutions are within 1e-8 (relative residual) of the
            # exact one; their difference is bounded accordingly
            assert np.linalg.norm(Ub[j] - U1[j]) / np.linalg.norm(U1[j]) < 1e-6
        # same arithmetic per column up to reduction order: iteration counts
        # may differ by one per column at most
        assert abs(ib["iterations"] - i1["iterations"]) <= 8


def test_block_columns_converge_independently(T, oracle):
    """A zero right-hand side, a column whose initial guess already solves
    it and ordinary columns share one block: each column is treated as a
    single solve would treat it."""
    nel = (16, 8, 8)
    t, ref = pair(T, oracle, nel, levels=3, spec=P.bcs("cfg2", nel), seed=13)
    F = P.point_loads(nel, 4, seed=5)
    F[1] = 0.0
    Ue, _ = solve_cols(T, t, F[2:3], 1, rtol=1e-12)
    U0 = np.zeros_like(F)
    U0[2] = Ue[0]
    U, info = solve_cols(T, t, F, 4, U0=U0)
    assert info["status"] == 0
    assert np.all(U[1] == 0.0)
    assert np.array_equal(U[2], Ue[0])      # converged on entry: untouched
    for j in (0, 3):
        Uo, st, _, _ = ref.solve(b=F[j])
        assert np.linalg.norm(U[j] - Uo) / np.linalg.norm(Uo) < 1e-8


def test_multi_column_apply(T, oracle):
    nel = (12, 6, 5)
    t, ref = pair(T, oracle, nel, levels=2, seed=3)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((5, 3 * t.nNode))
    y = np.zeros_like(u)
    t.apply(u, y, nrhs=5)
    for j in range(5):
        assert rel(y[j], ref.apply(u[j])) < 1e-12
    y32 = np.zeros_like(u)
    t.apply(u, y32, nrhs=5, precision=T.PREC_MIXED)
    for j in range(5):
        assert rel(y32[j], y[j]) < 1e-5


def test_rhs_block_validation(T, oracle):
    nel = (8, 4, 4)
    t, _ = pair(T, oracle, nel, levels=2, seed=1)
    F = P.point_loads(nel, 3, seed=1)
    with pytest.raises(T.TopOptError):
        solve_cols(T, t, F, 3)
    U, info = solve_cols(T, t, F, 0)       # 3 columns: blocks of 2 + 1
    assert info["status"] == 0
