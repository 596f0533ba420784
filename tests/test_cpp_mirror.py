"""The C++ host mirror (include/topopt_b200.hpp) compiles against the C ABI
and, on a GPU, reproduces the oracle's compliance and volume, and its MMA
object's update (the OCsub branch with one constraint, MMAsub with two)."""
import os
import subprocess

import numpy as np
import pytest

from topopt3d_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp")
LIBDIR = os.path.join(ROOT, "topopt3d_b200")


def build_mirror(tmp_path):
    from topopt3d_b200 import build
    build.build()
    exe = str(tmp_path / "mirror_main")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    SRC, "-o", exe, "-L", LIBDIR, "-ltopopt_b200",
                    "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_cpp_mirror_compiles(tmp_path):
    assert os.path.exists(build_mirror(tmp_path))


def test_cpp_step_out_matches_python_log(tmp_path):
    """tpo::StepOut and the Python optimize log write the same Output.txt
    entry for the same values."""
    from topopt3d_b200 import build
    from topopt3d_b200.topopt import step_out_text
    build.build()
    exe = str(tmp_path / "stepout_main")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "stepout_main.cpp"), "-o", exe, "-L",
                    LIBDIR, "-ltopopt_b200", "-Wl,-rpath," + LIBDIR], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout

    class Fn:
        def __init__(self, name, value):
            self.name, self.value = name, value

    assert out == step_out_text(12.3456789, [-0.00123456789012345, 0.5], 7,
                                [Fn("Compliance", 12.3456789),
                                 Fn("Volume", -0.00123456789012345)])


@pytest.mark.gpu
def test_cpp_mirror_matches_oracle(tmp_path, oracle):
    exe = build_mirror(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    st, its, C, V, sc, sv, ch_oc, s_oc, ch_mma, s_mma = out.split()
    nel = (12, 6, 6)
    ref = oracle.Problem(nel, rmin=1.5, mg_levels=2)
    P.apply_bcs(ref, P.cantilever_bcs(nel))
    e = np.arange(int(np.prod(nel)))
    ref.set_design(0.1 + 0.9 * ((e * 7919) % 101) / 100.0)
    ref.assemble(oracle.default_opts())
    U, _, _, _ = ref.solve()
    Co, dco, _ = ref.compliance(U)
    Vo, dvo = ref.volume()
    assert int(st) == 0
    assert abs(float(C) - Co) < 1e-8 * Co
    assert abs(float(V) - Vo) < 1e-14
    assert abs(float(sc) - dco.sum()) < 1e-7 * abs(dco.sum())
    # constraint gradient = dV/dx / (max - min)
    assert abs(float(sv) - dvo.sum()) < 1e-12
    x = 0.1 + 0.9 * ((e * 7919) % 101) / 100.0
    x_oc, c_oc = oracle.oc_update(x, dco, Vo - 0.3, dvo, 0.5)
    assert abs(float(ch_oc) - c_oc) < 1e-9
    assert abs(float(s_oc) - x_oc.sum()) < 1e-7
    n = x.size
    h = n // 2
    d2 = np.zeros(n)
    d2[:h] = 1.0 / h
    st_o = {"x": x.copy(), "xold1": x.copy(), "xold2": x.copy(), "low": np.zeros(n),
            "upp": np.ones(n), "xmin": np.zeros(n), "xmax": np.ones(n), "fresh_start": True}
    c_mma = oracle.mma_update(st_o, dco, np.array([Vo - 0.3, x[:h].mean() - 0.35]),
                              np.stack([dvo, d2], axis=1), 0)
    assert abs(float(ch_mma) - c_mma) < 1e-9
    assert abs(float(s_mma) - st_o["x"].sum()) < 1e-7
