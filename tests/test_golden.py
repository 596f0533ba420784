"""Golden fixtures (tests/golden/*.npz, made by make_golden.py): the oracle
must reproduce them on the CPU, and the CUDA path must match them."""
import os

import numpy as np
import pytest

from topopt3d_b200 import problems as P

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def spec_for(name, nel):
    return P.column_bcs(nel) if name.startswith("column") else P.cantilever_bcs(nel)


@pytest.mark.parametrize("name", ["cantilever_12x6x6", "column_9x5x4_r2"])
def test_oracle_reproduces_golden(oracle, name):
    g = load(name)
    nel = tuple(int(v) for v in g["nel"])
    pb = oracle.Problem(nel, rmin=float(g["rmin"]), mg_levels=int(g["levels"]))
    P.apply_bcs(pb, spec_for(name, nel))
    fm, F = pb.get_bc()
    assert np.array_equal(fm, g["fixmask"]) and np.array_equal(F, g["F"])
    pb.set_design(g["x"])
    rho, E, dEdz = pb.material()
    assert np.array_equal(rho, g["rho"]) and np.array_equal(E, g["E"])
    o = oracle.default_opts(rtol=1e-12, maxit=1000)
    pb.assemble(o)
    U, st, its, rr = pb.solve(opts=o)
    assert st == 0
    assert np.linalg.norm(U - g["U"]) / np.linalg.norm(g["U"]) < 1e-12
    C, dCdx, _ = pb.compliance(U)
    assert abs(C - g["C"]) < 1e-12 * abs(g["C"])
    assert np.abs(dCdx - g["dCdx"]).max() < 1e-12 * np.abs(g["dCdx"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cantilever_12x6x6", "column_9x5x4_r2"])
def test_gpu_matches_golden(T, name):
    g = load(name)
    nel = tuple(int(v) for v in g["nel"])
    t = T.TopOpt(nel, rmin=float(g["rmin"]), mg_levels=int(g["levels"]))
    P.apply_bcs(t, spec_for(name, nel))
    fm, F = t.get_bc()
    assert np.array_equal(fm, g["fixmask"]) and np.array_equal(F, g["F"])
    t.FEInitialize()
    t.MatIntFnc(g["x"])
    assert np.abs(t.rho - g["rho"]).max() < 1e-15
    o = T.default_opts(rtol=1e-12, maxit=1000)
    t.FEAssemble(o)
    info = t.FESolve(o)
    assert info["status"] == 0
    assert np.linalg.norm(t.U - g["U"]) / np.linalg.norm(g["U"]) < 1e-10
    C, dCdx, _ = t.compliance()
    assert abs(C - g["C"]) < 1e-11 * abs(g["C"])
    assert np.abs(dCdx - g["dCdx"]).max() < 1e-10 * np.abs(g["dCdx"]).max()
    V, dV = t.volume()
    assert abs(V - g["V"]) < 1e-15 and np.abs(dV - g["dVdx"]).max() < 1e-17


@pytest.mark.gpu
def test_gpu_matches_golden_cfg0(T):
    g = load("cfg0_48x24x24")
    nel = tuple(int(v) for v in g["nel"])
    t = T.TopOpt(nel, rmin=1.5, mg_levels=3)
    P.apply_bcs(t, P.bcs("cfg0"))
    t.FEInitialize()
    t.MatIntFnc(P.design("cfg0"))
    for prec, tol in ((T.PREC_FP64, 1e-8), (T.PREC_MIXED, 1e-6)):
        t.FEAssemble()
        t.set("U", np.zeros(3 * t.nNode))
        info = t.FESolve(T.default_opts(precision=prec))
        assert info["status"] == 0 and info["relres"] <= 1e-8
        C, dCdx, _ = t.compliance()
        assert abs(C - g["C"]) / g["C"] < 1e-8
        assert np.abs(dCdx[g["sel"]] - g["dCdx_sel"]).max() < tol * np.abs(g["dCdx_sel"]).max()
        assert abs(np.linalg.norm(t.U) - g["U_norm"]) < tol * g["U_norm"]
