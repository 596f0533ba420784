"""Gradient-check harness of the compliance adjoint on the 64x32x32
cantilever (65,536 elements, 212,355 dof), density filter r_min = 2.0,
seeded uniform [0.1, 0.9] densities (seed 3).

The adjoint dC/dx = P^T(-dE/drho~ .* u_e^T K0 u_e) (Compliance.cpp:37-51,
Chain_Filter in Material_Interpolation.cpp:150-187) comes from the
library's sensitivity kernel through the C ABI.  Here, and only here, it is
wrapped in a torch.autograd.Function:

* forward(x): MatIntFnc, FEAssemble, FP64 PCG+GMG from U = 0 to 1e-12, C;
* backward(gC): gC * dC/dx for the design the forward saw.  The
  displacements U (3 * nNode doubles) are kept from the forward, or, when
  they exceed the harness's memory budget, only x is kept and backward
  solves for U again.

Checks:
* torch.autograd.gradcheck of C restricted to 64 seeded elements (central
  differences, eps = h = 1e-6, FP64) -- each numerical column is one pair
  of full cold FP64 solves;
* the full dC/dx vector against the FP64 oracle's, 1e-8 relative;
* the stored and the recomputed-displacement policies give the same
  gradient (the solve is deterministic, so bit for bit).

The solves start from U = 0 so each PCG iterate is a Galerkin
approximation, whose compliance error is quadratic in the energy-norm
error; with rtol 1e-12 that is far below the rounding of C itself.
"""
import numpy as np
import pytest

from topopt3d_b200 import problems as P

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CFG = "cfg3"
N_CHECK = 64
H = 1e-6


class CompliancePath:
    """The GPU context of one problem and the harness's storage policy."""

    def __init__(self, T, t, u_budget_bytes=None):
        self.T, self.t = T, t
        self.opts = T.default_opts(rtol=1e-12, maxit=2000)
        u_bytes = 3 * t.nNode * 8
        self.recompute = u_budget_bytes is not None and u_bytes > u_budget_bytes
        self.solves = 0
        self.zeros = torch.zeros(3 * t.nNode, dtype=torch.float64, device="cuda")

    def solve(self, x):
        t = self.t
        t.MatIntFnc(x.detach().contiguous())
        t.FEAssemble(self.opts)
        t.set("U", self.zeros)
        info = t.FESolve(self.opts)
        self.solves += 1
        if info["status"] != 0:
            raise RuntimeError(f"solve did not converge: {info}")
        return t.compliance(gradient=False)[0]


class ComplianceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, path):
        C = path.solve(x)
        ctx.path = path
        if path.recompute:
            ctx.save_for_backward(x)
        else:
            U = torch.empty(3 * path.t.nNode, dtype=torch.float64, device="cuda")
            path.t.get("U", out=U)
            ctx.save_for_backward(x, U)
        return x.new_tensor(C)

    @staticmethod
    def backward(ctx, gC):
        path = ctx.path
        t = path.t
        if path.recompute:
            (x,) = ctx.saved_tensors
            path.solve(x)                     # the displacements again
        else:
            x, U = ctx.saved_tensors
            t.MatIntFnc(x.detach().contiguous())
            t.set("U", U)
        dC = torch.empty_like(x)
        t.compliance(out=dC)                  # the adjoint kernel + P^T
        return gC * dC, None


@pytest.fixture(scope="module")
def cfg3(T):
    c = P.CONFIGS[CFG]
    t = T.TopOpt(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(t, P.bcs(CFG))
    t.FEInitialize()
    x0 = torch.tensor(P.design(CFG), device="cuda")
    idx = np.sort(np.random.default_rng(64).choice(t.nElem, N_CHECK, replace=False))
    yield t, x0, torch.tensor(idx, device="cuda")
    t.close()


def subspace(x0, idx, path):
    """C as a function of the 64 seeded elements' densities."""
    def f(s):
        return ComplianceFn.apply(x0.index_add(0, idx, s), path)
    return f


def test_gradcheck_64_elements(T, cfg3):
    t, x0, idx = cfg3
    path = CompliancePath(T, t)
    s = torch.zeros(N_CHECK, dtype=torch.float64, device="cuda", requires_grad=True)
    f = subspace(x0, idx, path)
    C0 = float(f(s).detach())
    # central differences, h = 1e-6; the rounding of C (~1e-15 C) gives
    # ~1e-9 C / h of noise in each difference quotient
    assert torch.autograd.gradcheck(f, (s,), eps=H, atol=2e-9 * C0, rtol=1e-5,
                                    check_undefined_grad=False, nondet_tol=0.0)
    # the same quotients, reported: worst relative error over the 64
    (g,) = torch.autograd.grad(f(s), s)
    g = g.cpu().numpy()
    fd = np.empty(N_CHECK)
    with torch.no_grad():
        for k in range(N_CHECK):
            e = torch.zeros_like(s)
            e[k] = H
            fd[k] = (float(f(s + e)) - float(f(s - e))) / (2 * H)
    err = np.max(np.abs(fd - g) / np.abs(g))
    nerr = np.linalg.norm(fd - g) / np.linalg.norm(g)
    print(f"cfg3 gradcheck: C = {C0:.12g}, over {N_CHECK} elements: max rel error "
          f"{err:.2e}, 2-norm rel error {nerr:.2e}")
    # the same bound as gradcheck's, per element, and a norm-wise one
    assert np.all(np.abs(fd - g) <= 2e-9 * C0 + 1e-5 * np.abs(g))
    assert nerr < 2e-5


def test_full_sensitivity_matches_oracle(T, oracle, cfg3):
    t, x0, _ = cfg3
    c = P.CONFIGS[CFG]
    ref = oracle.Problem(c["nel"], rmin=c["rmin"], mg_levels=c["levels"])
    P.apply_bcs(ref, P.bcs(CFG))
    ref.set_design(P.design(CFG), 3.0, 1e-10)
    o = oracle.default_opts(rtol=1e-12, maxit=2000)
    ref.assemble(o)
    Uo, st, _, _ = ref.solve(opts=o)
    assert st == 0
    Co, dco, _ = ref.compliance(Uo)
    x = x0.clone().requires_grad_(True)
    C = ComplianceFn.apply(x, CompliancePath(T, t))
    C.backward()
    dc = x.grad.cpu().numpy()
    ec = abs(float(C) - Co) / abs(Co)
    ed = np.linalg.norm(dc - dco) / np.linalg.norm(dco)
    print(f"cfg3 vs oracle: C {ec:.2e}, dC/dx {ed:.2e}")
    assert ec < 1e-10 and ed < 1e-8


def test_recompute_policy_gives_the_same_gradient(T, cfg3):
    t, x0, _ = cfg3
    grads = {}
    for name, budget in (("store", None), ("recompute", 1024)):
        path = CompliancePath(T, t, u_budget_bytes=budget)
        assert path.recompute == (name == "recompute")
        x = x0.clone().requires_grad_(True)
        C = ComplianceFn.apply(x, path)
        # a different design in between: backward must restore its own state
        path.solve(x0 * 0.9)
        C.backward()
        grads[name] = (float(C), x.grad.clone(), path.solves)
    assert grads["store"][0] == grads["recompute"][0]
    assert torch.equal(grads["store"][1], grads["recompute"][1])
    # forward + intermediate solve, plus the backward's solve when recomputing
    assert grads["store"][2] == 2 and grads["recompute"][2] == 3
