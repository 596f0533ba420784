"""The reference's output and restart files (TopOpt.cpp:97-508,
RecMesh.cpp:34-412): PETSc binary Vec / AIJ matrices, MeshOut, PrintVals,
LoadMesh and the Output.txt log.

CPU: the library's PETSc-binary writers and readers against the oracle's
independent numpy restatement, both ways, for 4- and 8-byte PetscInt, with
the error cases; the StepOut / ResultOut text against literal strings
written from the reference's printf formats; LoadMesh's refusals of folders
that are not a structured box or hold springs, eigen-only supports or
passive elements.

GPU: MeshOut's files against the oracle's mesh, BC selection, filters and
interpolation weights; PrintVals against the context's vectors; LoadMesh of
a MeshOut folder reproducing the BCs and the solve; the x_pen<p>.bin restart
loop; the Output.txt log and PrintVals schedule of `optimize`.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import petsc_io as PIO
from topopt3d_b200 import _lib as L
from topopt3d_b200 import problems as P

DP = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)


def lib_write_vec(path, v, ib):
    v = np.ascontiguousarray(v, np.float64)
    return L.load().tpo_write_vec_bin(str(path).encode(), v.ctypes.data_as(DP), v.size, ib)


def lib_read_vec(path, ib):
    lib = L.load()
    n = C.c_int64()
    rc = lib.tpo_read_vec_bin(str(path).encode(), None, 0, C.byref(n), ib)
    assert rc == 0, lib.tpo_last_error(None)
    v = np.zeros(n.value)
    assert lib.tpo_read_vec_bin(str(path).encode(), v.ctypes.data_as(DP), v.size,
                                C.byref(n), ib) == 0
    return v


def lib_write_mat(path, rowptr, col, val, shape, ib):
    rp = np.ascontiguousarray(rowptr, np.int64)
    cl = np.ascontiguousarray(col, np.int64)
    vl = np.ascontiguousarray(val, np.float64)
    return L.load().tpo_write_mat_bin(str(path).encode(), shape[0], shape[1],
                                      rp.ctypes.data_as(I64P), cl.ctypes.data_as(I64P),
                                      vl.ctypes.data_as(DP), ib)


def lib_read_mat(path, ib):
    lib = L.load()
    M, N, nnz = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib.tpo_read_mat_bin(str(path).encode(), C.byref(M), C.byref(N), C.byref(nnz),
                              None, None, None, 0, 0, ib)
    assert rc == 0, lib.tpo_last_error(None)
    rp = np.zeros(M.value + 1, np.int64)
    col = np.zeros(nnz.value, np.int64)
    val = np.zeros(nnz.value)
    assert lib.tpo_read_mat_bin(str(path).encode(), C.byref(M), C.byref(N), C.byref(nnz),
                                rp.ctypes.data_as(I64P), col.ctypes.data_as(I64P),
                                val.ctypes.data_as(DP), rp.size, col.size, ib) == 0
    return rp, col, val, (M.value, N.value)


def random_csr(rng, M, N, density=0.3):
    A = (rng.random((M, N)) < density) * rng.standard_normal((M, N))
    A[1] = 0.0                                   # an empty row
    rp = np.concatenate([[0], np.cumsum((A != 0).sum(1))])
    col = np.concatenate([np.nonzero(r)[0] for r in A]).astype(np.int64)
    return rp, col, A[A != 0], A


# ------------------------------------------------------------------- CPU

@pytest.mark.parametrize("ib", [4, 8])
def test_vec_roundtrip_against_oracle(tmp_path, ib):
    rng = np.random.default_rng(ib)
    for n in (0, 1, 1000):
        v = rng.standard_normal(n)
        v[:min(n, 3)] = [np.inf, -0.0, 1e-310][:min(n, 3)]
        assert lib_write_vec(tmp_path / "a.bin", v, ib) == 0
        np.testing.assert_array_equal(PIO.read_vec(tmp_path / "a.bin", ib), v)
        PIO.write_vec(tmp_path / "b.bin", v, ib)
        np.testing.assert_array_equal(lib_read_vec(tmp_path / "b.bin", ib), v)
        assert (tmp_path / "a.bin").read_bytes() == (tmp_path / "b.bin").read_bytes()
        assert os.path.getsize(tmp_path / "a.bin") == 2 * ib + 8 * n


@pytest.mark.parametrize("ib", [4, 8])
def test_mat_roundtrip_against_oracle(tmp_path, ib):
    rng = np.random.default_rng(10 + ib)
    rp, col, val, A = random_csr(rng, 7, 11)
    assert lib_write_mat(tmp_path / "a.bin", rp, col, val, A.shape, ib) == 0
    r2, c2, v2, shape = PIO.read_mat(tmp_path / "a.bin", ib)
    assert shape == A.shape
    np.testing.assert_array_equal(r2, rp)
    np.testing.assert_array_equal(c2, col)
    np.testing.assert_array_equal(v2, val)
    PIO.write_mat(tmp_path / "b.bin", rp, col, val, A.shape, ib)
    r3, c3, v3, shape3 = lib_read_mat(tmp_path / "b.bin", ib)
    assert shape3 == A.shape
    np.testing.assert_array_equal(r3, rp)
    np.testing.assert_array_equal(c3, col)
    np.testing.assert_array_equal(v3, val)
    assert (tmp_path / "a.bin").read_bytes() == (tmp_path / "b.bin").read_bytes()


def test_binary_errors(tmp_path):
    lib = L.load()
    v = np.arange(4.0)
    assert lib_write_vec(tmp_path / "v.bin", v, 4) == 0
    M, N, nnz = C.c_int64(), C.c_int64(), C.c_int64()
    # a Vec is not a matrix
    rc = lib.tpo_read_mat_bin(str(tmp_path / "v.bin").encode(), C.byref(M), C.byref(N),
                              C.byref(nnz), None, None, None, 0, 0, 4)
    assert rc < 0 and b"not a PETSc binary matrix" in lib.tpo_last_error(None)
    # truncated Vec
    b = (tmp_path / "v.bin").read_bytes()
    (tmp_path / "t.bin").write_bytes(b[:-3])
    n = C.c_int64()
    rc = lib.tpo_read_vec_bin(str(tmp_path / "t.bin").encode(), None, 0, C.byref(n), 4)
    assert rc < 0 and b"file size" in lib.tpo_last_error(None)
    # the wrong PetscInt size reads a wrong header
    assert lib.tpo_read_vec_bin(str(tmp_path / "v.bin").encode(), None, 0, C.byref(n), 8) < 0
    # a buffer that is too small
    small = np.zeros(2)
    rc = lib.tpo_read_vec_bin(str(tmp_path / "v.bin").encode(), small.ctypes.data_as(DP), 2,
                              C.byref(n), 4)
    assert rc < 0 and n.value == 4
    # a column index beyond a 4-byte PetscInt, fine with 8 bytes
    big = [0, 1]
    assert lib_write_mat(tmp_path / "m.bin", big, [2**31 + 1], [1.0], (1, 2**31 + 5), 4) < 0
    assert b"4-byte PetscInt" in lib.tpo_last_error(None)
    assert lib_write_mat(tmp_path / "m.bin", big, [2**31 + 1], [1.0], (1, 2**31 + 5), 8) == 0
    rp, col, val, shape = PIO.read_mat(tmp_path / "m.bin", 8)
    assert shape == (1, 2**31 + 5) and col[0] == 2**31 + 1
    # a missing file
    assert lib.tpo_read_vec_bin(str(tmp_path / "none.bin").encode(), None, 0, C.byref(n),
                                4) < 0
    assert b"cannot open" in lib.tpo_last_error(None)


def test_step_and_result_text():
    """StepOut's and ResultOut's entries (TopOpt.cpp:386-401, 421-425),
    spelled out from the reference's formats."""
    from topopt3d_b200.topopt import result_out_text, step_out_text

    class Fn:
        def __init__(self, name, value):
            self.name, self.value = name, value

    s = step_out_text(12.3456789, [-0.00123456789012345, 0.5], 7,
                      [Fn("Compliance", 12.3456789), Fn("Volume", -0.00123456789012345)])
    assert s == ("Iteration number: 7\n"
                 "Objective: 12.3457\n"
                 "Constraints:\n"
                 "\t-0.00123456789012\t\t0.5\t\n"
                 "All function values:\n"
                 "\t  Compliance: 12.345679\n"
                 "\t      Volume: -0.0012345679\n"
                 "\n")
    r = result_out_text(50, 3.0, 10.0, 4.0)
    stars = "*" * 48
    assert r == (stars + "\nAfter   50 iterations with a penalty of 3 the\n"
                 "ratio of stiffness sum to volume sum is 2.5\n" + stars + "\n\n")


# ------------------------------------------------------------------- GPU

NEL = (6, 4, 3)
SPEC = [
    ("support", (0.0, 0.0, 0.0), (1e-10, 1e10, 1e10), P.OPEN, (1.0, 1.0, 1.0)),
    ("support", (6.0, 4.0, 0.0), (1e-10, 1e-10, 1e10), P.OPEN, (0.0, 1.0, 0.0)),
    ("load", (6.0, 0.0, 0.0), (1e-10, 1e10, 1e-10), P.OPEN, (0.0, 0.0, -0.2)),
    ("load", (6.0, 2.0, 0.0), (1e-10, 1e-10, 1e-10), P.OPEN, (0.1, 0.0, 0.0)),
]


def design(nel):
    e = np.arange(int(np.prod(nel)))
    return 0.1 + 0.9 * ((e * 7919) % 101) / 100.0


@pytest.mark.gpu
@pytest.mark.parametrize("ib", [4, 8])
def test_mesh_out_matches_oracle(T, oracle, tmp_path, ib):
    t = T.TopOpt(NEL, rmin=1.5, mg_levels=2)
    P.apply_bcs(t, SPEC)
    t.MeshOut(str(tmp_path), rmax=3.0, index_bytes=ib)
    ne, nn = int(np.prod(NEL)), int(np.prod([n + 1 for n in NEL]))
    f = lambda name: str(tmp_path / name)
    np.testing.assert_array_equal(PIO.read_ints(f("Element_Distribution.bin"), ib), [0, ne])
    np.testing.assert_array_equal(PIO.read_ints(f("Node_Distribution.bin"), ib), [0, nn])
    el = PIO.read_ints(f("elements.bin"), ib).reshape(ne, 8)
    for e in range(ne):
        np.testing.assert_array_equal(el[e], oracle.element_nodes(NEL, e))
    np.testing.assert_array_equal(PIO.read_doubles(f("nodes.bin")).reshape(nn, 3),
                                  oracle.node_coords(NEL, (1.0, 1.0, 1.0)))
    # the Set_BC lists in call order (Inputs.cpp:145-170)
    sn, sv, ln, lv = [], [], [], []
    for kind, center, radius, limits, values in SPEC:
        sel = oracle.select_nodes(NEL, (1.0, 1.0, 1.0), center, radius, limits)
        if kind == "support":
            sn += list(sel)
            sv += [[v != 0 for v in values]] * len(sel)
        else:
            ln += list(sel)
            lv += [list(values)] * len(sel)
    np.testing.assert_array_equal(PIO.read_ints(f("supportNodes.bin"), ib), sn)
    np.testing.assert_array_equal(PIO.read_bools(f("supports.bin")).reshape(-1, 3), sv)
    np.testing.assert_array_equal(PIO.read_ints(f("loadNodes.bin"), ib), ln)
    np.testing.assert_array_equal(PIO.read_doubles(f("loads.bin")).reshape(-1, 3), lv)
    for name in ("eigenSupportNodes", "eigenSupports", "springNodes", "springs",
                 "massNodes", "masses"):
        assert os.path.getsize(f(name + ".bin")) == 0
    assert PIO.read_bools(f("active.bin")).all() and os.path.getsize(f("active.bin")) == ne
    # the density filter, bit for bit
    rp, col, val = oracle.filter_csr(NEL, (1.0, 1.0, 1.0), 1.5)
    r2, c2, v2, shape = PIO.read_mat(f("Filter.bin"), ib)
    assert shape == (ne, ne)
    np.testing.assert_array_equal(r2, rp)
    np.testing.assert_array_equal(c2, col)
    np.testing.assert_array_equal(v2, val)
    # the max-length-scale filter and its edge vector
    rp, col, val, edge = PIO.max_filter(NEL, (1.0, 1.0, 1.0), 3.0)
    r2, c2, v2, _ = PIO.read_mat(f("Max_Filter.bin"), ib)
    np.testing.assert_array_equal(r2, rp)
    np.testing.assert_array_equal(c2, col)
    np.testing.assert_allclose(v2, val, rtol=0, atol=1e-15)
    np.testing.assert_allclose(PIO.read_vec(f("Void_Edge_Volume.bin"), ib), edge,
                               rtol=0, atol=1e-12)
    # the interpolation of level 0 -> 1 and its column split
    pb = oracle.Problem(NEL, rmin=1.5, mg_levels=2)
    P.apply_bcs(pb, SPEC)
    pb.set_design(design(NEL))
    pb.assemble(oracle.default_opts())
    fine, coarse = t.level_dims(0), t.level_dims(1)
    Pd = PIO.prolongation_dense(pb, 0, fine, coarse)
    r2, c2, v2, shape = PIO.read_mat(f("P0.bin"), ib)
    assert shape == Pd.shape
    A = np.zeros(shape)
    for r in range(shape[0]):
        A[r, c2[r2[r]:r2[r + 1]]] = v2[r2[r]:r2[r + 1]]
        assert np.all(np.diff(c2[r2[r]:r2[r + 1]]) > 0)
    np.testing.assert_array_equal(A, Pd)
    np.testing.assert_array_equal(PIO.read_ints(f("P0.bin.split"), ib), [shape[1]])
    assert not os.path.exists(f("P1.bin"))


@pytest.mark.gpu
def test_print_vals_load_mesh_and_restart(T, oracle, tmp_path):
    x = design(NEL)
    t = T.TopOpt(NEL, rmin=1.5, mg_levels=2)
    P.apply_bcs(t, SPEC)
    t.FEInitialize()
    t.MatIntFnc(x)
    o = T.default_opts(rtol=1e-12, maxit=500)
    t.FEAssemble(o)
    t.FESolve(o)
    C0 = t.compliance(gradient=False)[0]
    t.MeshOut(str(tmp_path))
    nd = 3 * t.nNode
    phiB = np.random.default_rng(1).standard_normal((nd, 2))
    t.PrintVals("_pen3", str(tmp_path), phiB=phiB)
    f = lambda name: str(tmp_path / name)
    for name, vec in (("U", "U"), ("x", "x"), ("V", "rho"), ("Es", "Es"), ("E", "E")):
        np.testing.assert_array_equal(PIO.read_vec(f(name + "_pen3.bin")), t.get(vec))
    for i in range(2):
        np.testing.assert_array_equal(PIO.read_vec(f(f"phiB_pen3_mode{i}.bin")), phiB[:, i])
    assert not os.path.exists(f("phiB_pen3_mode2.bin"))
    # restart: the mesh, BCs and levels come back from the folder
    t2 = T.TopOpt.LoadMesh(str(tmp_path), rmin=1.5)
    assert t2.nel == NEL and t2.mg_levels == t.mg_levels
    m1, F1 = t.get_bc()
    m2, F2 = t2.get_bc()
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(F1, F2)
    # MeshOut of the reloaded problem writes the same files, byte for byte
    os.makedirs(tmp_path / "again")
    t2.MeshOut(str(tmp_path / "again"))
    names = sorted(n for n in os.listdir(tmp_path) if n.endswith((".bin", ".split"))
                   and not n.endswith("_pen3.bin") and "_mode" not in n)
    assert len(names) == 20
    for n in names:
        assert (tmp_path / n).read_bytes() == (tmp_path / "again" / n).read_bytes(), n
    xr, start = t2.load_design(str(tmp_path), [3.0, 4.0])
    np.testing.assert_array_equal(xr, x)
    assert t2.penal == 4.0 and start == 1
    # the same state at the same penalty solves to the same compliance
    t2.penal = t.penal
    t2.FEInitialize()
    t2.MatIntFnc(xr)
    t2.FEAssemble(o)
    t2.FESolve(o)
    assert abs(t2.compliance(gradient=False)[0] - C0) <= 1e-12 * C0
    # no file for the first penalty: x = 0.5 and the run starts there
    xr, start = t2.load_design(str(tmp_path), [1.0, 3.0])
    assert np.all(xr == 0.5) and t2.penal == 1.0 and start == 0
    # a filter of another radius is refused
    t3 = T.TopOpt(NEL, rmin=2.5, mg_levels=2)
    P.apply_bcs(t3, SPEC)
    os.makedirs(tmp_path / "r25")
    t3.MeshOut(str(tmp_path / "r25"))
    with pytest.raises(T.TopOptError, match="Filter.bin"):
        T.TopOpt.LoadMesh(str(tmp_path / "r25"), rmin=1.5)
    assert T.TopOpt.LoadMesh(str(tmp_path / "r25"), rmin=2.5).nElem == t.nElem


@pytest.mark.gpu
def test_optimize_output_log_and_print_schedule(T, tmp_path):
    nel = (12, 6, 6)
    t = T.TopOpt(nel, mg_levels=2)
    P.apply_bcs(t, P.cantilever_bcs(nel))
    t.FEInitialize()
    t.function_list = [T.Compliance([1.0], 0.0, 1.0, True, True),
                       T.Volume([0.3], 0.0, 1.0, False, True)]
    oc = T.OC(n=t.nElem, maxiter=4)
    oc.xval = np.full(t.nElem, 0.3)
    out = tmp_path / "Output.txt"
    hist = T.optimize(t, oc, output=str(out), folder=str(tmp_path), print_every=2)
    from topopt3d_b200.topopt import step_out_text
    text = out.read_text()
    assert text.startswith("\nPenalty increased to 3\n")
    body = text[len("\nPenalty increased to 3\n"):]
    # one StepOut entry per evaluation, with the values of that evaluation
    for h in hist:
        class Fn:
            pass
        fns = []
        for name, v in zip(("Compliance", "Volume"), (h["f"], h["g"][0])):
            fn = Fn()
            fn.name, fn.value = name, v
            fns.append(fn)
        entry = step_out_text(h["f"], h["g"], h["iter"], fns)
        assert body.startswith(entry), (body[:200], entry)
        body = body[len(entry):]
    E, V = t.get("E"), t.get("rho")
    assert body == ("*" * 48 + "\nAfter %4i iterations with a penalty of 3 the\n"
                    "ratio of stiffness sum to volume sum is %1.4g\n" % (4, E.sum() / V.sum())
                    + "*" * 48 + "\n\n")
    # PrintVals at iterations 2 and 4 (every 2nd StepOut) and at the end
    for sfx in ("_pen3_it2", "_pen3_it4", "_pen3"):
        assert os.path.exists(tmp_path / f"U{sfx}.bin"), sfx
    assert not os.path.exists(tmp_path / "U_pen3_it1.bin")
    assert not os.path.exists(tmp_path / "U_pen3_it3.bin")
    np.testing.assert_array_equal(PIO.read_vec(str(tmp_path / "x_pen3.bin")), oc.xval)


# ------------------------------------------------ LoadMesh refusals (CPU)

def write_mesh_folder(d, oracle, nel=(3, 2, 2), ib=4):
    """A MeshOut-style folder of a structured box written with numpy from
    the oracle's mesh data (one support node, one load node)."""
    d.mkdir(exist_ok=True)
    idt = "<i4" if ib == 4 else "<i8"
    ne, nn = int(np.prod(nel)), int(np.prod([n + 1 for n in nel]))
    w = lambda name, a, dt: np.asarray(a, dt).tofile(str(d / name))
    w("Element_Distribution.bin", [0, ne], idt)
    w("Node_Distribution.bin", [0, nn], idt)
    w("elements.bin", np.stack([oracle.element_nodes(nel, e) for e in range(ne)]), idt)
    w("nodes.bin", oracle.node_coords(nel, (1.0, 1.0, 1.0)), "<f8")
    w("supportNodes.bin", [0], idt)
    w("supports.bin", [1, 1, 1], np.uint8)
    w("loadNodes.bin", [nn - 1], idt)
    w("loads.bin", [0.0, 0.0, -1.0], "<f8")
    for name in ("eigenSupportNodes", "springNodes", "massNodes"):
        w(name + ".bin", [], idt)
    for name in ("eigenSupports", "springs", "masses"):
        w(name + ".bin", [], np.uint8)
    w("active.bin", np.ones(ne), np.uint8)
    return ne, nn


def load_mesh_error(folder, ib=4):
    lib = L.load()
    p = L.MeshParams((C.c_int32 * 3)(1, 1, 1), (C.c_double * 3)(1.0, 1.0, 1.0),
                     1.0, 0.3, 1.5, 0)
    h = C.c_void_p()
    rc = lib.tpo_load_mesh(str(folder).encode(), C.byref(p), ib, C.byref(h))
    if rc == 0:
        lib.tpo_destroy(h)
    return rc, lib.tpo_last_error(None)


def test_load_mesh_refusals(tmp_path, oracle):
    """The checks of tpo_load_mesh that run before a context exists: a
    folder that is not a structured hex8 box, or that holds data a context
    cannot represent, is refused with a message."""
    ne, nn = write_mesh_folder(tmp_path / "ok", oracle)
    rc, msg = load_mesh_error(tmp_path / "ok")
    # a valid folder passes every check; creating the context then needs a GPU
    assert rc == 0 or b"context creation failed" in msg, msg

    d = tmp_path / "perm"
    write_mesh_folder(d, oracle)
    el = np.fromfile(str(d / "elements.bin"), "<i4").reshape(ne, 8)
    el[1, [1, 3]] = el[1, [3, 1]]
    el.tofile(str(d / "elements.bin"))
    rc, msg = load_mesh_error(d)
    assert rc < 0 and b"structured numbering" in msg
    el[1, [1, 3]] = el[1, [3, 1]]
    el[0, [1, 3]] = el[0, [3, 1]]        # element 0 sets the spacing
    el.tofile(str(d / "elements.bin"))
    rc, msg = load_mesh_error(d)
    assert rc < 0 and b"element size" in msg

    d = tmp_path / "skew"
    write_mesh_folder(d, oracle)
    xyz = np.fromfile(str(d / "nodes.bin"), "<f8").reshape(nn, 3)
    xyz[5, 1] += 0.25
    xyz.tofile(str(d / "nodes.bin"))
    rc, msg = load_mesh_error(d)
    assert rc < 0 and b"regular grid" in msg

    d = tmp_path / "spring"
    write_mesh_folder(d, oracle)
    np.asarray([2], "<i4").tofile(str(d / "springNodes.bin"))
    np.asarray([1.0, 1.0, 1.0], "<f8").tofile(str(d / "springs.bin"))
    rc, msg = load_mesh_error(d)
    assert rc == L.TPO_E_UNSUPPORTED and b"springs" in msg

    d = tmp_path / "eigen"
    write_mesh_folder(d, oracle)
    np.asarray([1], "<i4").tofile(str(d / "eigenSupportNodes.bin"))
    rc, msg = load_mesh_error(d)
    assert rc == L.TPO_E_UNSUPPORTED and b"eigen-analysis supports" in msg

    d = tmp_path / "passive"
    write_mesh_folder(d, oracle)
    act = np.ones(ne, np.uint8)
    act[1] = 0
    act.tofile(str(d / "active.bin"))
    rc, msg = load_mesh_error(d)
    assert rc == L.TPO_E_UNSUPPORTED and b"passive" in msg

    d = tmp_path / "bcsize"
    write_mesh_folder(d, oracle)
    np.asarray([0.0, 1.0], "<f8").tofile(str(d / "loads.bin"))
    rc, msg = load_mesh_error(d)
    assert rc < 0 and b"do not match" in msg

    d = tmp_path / "missing"
    write_mesh_folder(d, oracle)
    os.remove(d / "nodes.bin")
    rc, msg = load_mesh_error(d)
    assert rc < 0 and b"cannot open" in msg and b"nodes.bin" in msg

    # 8-byte PetscInt files read with 8, refused with 4
    write_mesh_folder(tmp_path / "ib8", oracle, ib=8)
    rc, msg = load_mesh_error(tmp_path / "ib8", ib=8)
    assert rc == 0 or b"context creation failed" in msg, msg
    rc, msg = load_mesh_error(tmp_path / "ib8", ib=4)
    assert rc < 0
