"""The 192x96x96 cantilever (1,769,472 elements, 5,447,811 dof) solved by
the FP64 oracle and by the GPU in both forms, compared on the full vectors.

This is the acceptance check of the benchmark workload: the oracle's
assembled FP64 PCG + 5-level GMG (the reference's KSPSolve with PCMG,
FEAnalysis.cpp:673, and Compliance::Function, Compliance.cpp:15-57) and
the GPU's matrix-free solve, FP64 and mixed FP32/FP64, all from U = 0 to a
relative residual of 1e-8.

Tolerances (relative):
  C                 1e-8 in both forms
  U, dC/dx (FP64)   1e-8 (2-norm)
  U, dC/dx (mixed)  1e-6 (2-norm)
  PCG iterations    the oracle's count +-2
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P

pytestmark = pytest.mark.gpu

CFG = "cfg1"


@pytest.fixture(scope="module")
def oracle_cfg1(oracle):
    c = P.CONFIGS[CFG]
    ref = oracle.Problem(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(ref, P.bcs(CFG))
    ref.set_design(P.design(CFG), 3.0, 1e-10)
    ref.assemble(oracle.default_opts())
    U, st, its, rr = ref.solve(opts=oracle.default_opts())
    assert st == 0 and rr <= 1e-8
    C, dc, _ = ref.compliance(U)
    del ref
    return U, C, dc, its


@pytest.fixture(scope="module")
def gpu_cfg1(T):
    c = P.CONFIGS[CFG]
    t = T.TopOpt(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(t, P.bcs(CFG))
    t.FEInitialize()
    t.MatIntFnc(P.design(CFG))
    t.FEAssemble()
    yield t
    t.close()


def nrel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_cfg1_solution_matches_oracle(T, oracle_cfg1, gpu_cfg1, prec):
    Uo, Co, dco, its_o = oracle_cfg1
    t = gpu_cfg1
    t.set("U", np.zeros(3 * t.nNode))
    p = T.PREC_FP64 if prec == "fp64" else T.PREC_MIXED
    info = t.FESolve(T.default_opts(precision=p))
    assert info["status"] == 0 and info["relres"] <= 1e-8
    C, dc, _ = t.compliance()
    eu, ec, ed = nrel(t.U, Uo), abs(C - Co) / abs(Co), nrel(dc, dco)
    print(f"cfg1 {prec}: U {eu:.3e} C {ec:.3e} dC {ed:.3e} "
          f"its {info['iterations']} (oracle {its_o})")
    tol = 1e-8 if prec == "fp64" else 1e-6
    assert ec < 1e-8
    assert eu < tol
    assert ed < tol
    assert abs(info["iterations"] - its_o) <= 2
