"""tpo_sensitivity_noalloc: the filtered compliance sensitivity for callers
that may not allocate device memory (a framework-owned memory pool, code
inside a CUDA graph capture, a fixed up-front memory budget).  It must give
the same dC/dx as the context-based entry point tpo_compliance, on two calls
in a row (the second call reuses the library's fixed scratch array), and
refuse meshes larger than its fixed maximum.

This file is collected last so that a run stopping at its first failure has
already run every other test; it also passes on its own in a fresh process,
where its first call performs the per-device set-up."""
import ctypes as C

import numpy as np
import pytest

from topopt3d_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_noalloc_sensitivity_matches_compliance_entry_point(T):
    torch = pytest.importorskip("torch")
    lib = T.load()
    nel, rmin = (24, 12, 12), 1.5
    t = T.TopOpt(nel, rmin=rmin, mg_levels=2)
    P.apply_bcs(t, P.cantilever_bcs(nel))
    t.FEInitialize()
    t.MatIntFnc(np.random.default_rng(21).uniform(0.05, 1.0, t.nElem))
    t.FEAssemble()
    assert t.FESolve()["status"] == 0
    _, ref, _ = t.compliance()                    # existing entry point
    U = torch.tensor(t.U, device="cuda")
    dEdz = torch.tensor(t.dEdz, device="cuda")
    nel_c = (C.c_int32 * 3)(*nel)
    dx_c = (C.c_double * 3)(1.0, 1.0, 1.0)
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((t.nElem,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.tpo_sensitivity_noalloc(nel_c, dx_c, 1.0, 0.3, rmin,
                                         C.c_void_p(U.data_ptr()),
                                         C.c_void_p(dEdz.data_ptr()),
                                         C.c_void_p(out.data_ptr()),
                                         C.c_void_p(stream.cuda_stream), msg, 256)
        assert rc == 0, msg.value
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)), call


def test_noalloc_anisotropic_element_and_material(T):
    """Element edges (1, 0.5, 0.75), E0 = 3, nu = 0.25, filter radius 1.2:
    the same dC/dx as tpo_compliance on a context made with the same mesh
    parameters, so a swapped or ignored dx, E0 or nu in either the element
    constants or the filter template shows up."""
    torch = pytest.importorskip("torch")
    lib = T.load()
    nel, dx, E0, nu, rmin = (16, 10, 8), (1.0, 0.5, 0.75), 3.0, 0.25, 1.2
    t = T.TopOpt(nel, dx=dx, E0=E0, Nu0=nu, rmin=rmin, mg_levels=2)
    P.apply_bcs(t, P.cantilever_bcs(nel, dx))
    t.FEInitialize()
    t.MatIntFnc(np.random.default_rng(22).uniform(0.05, 1.0, t.nElem))
    t.FEAssemble()
    assert t.FESolve()["status"] == 0
    _, ref, _ = t.compliance()
    U = torch.tensor(t.U, device="cuda")
    dEdz = torch.tensor(t.dEdz, device="cuda")
    msg = C.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((t.nElem,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.tpo_sensitivity_noalloc((C.c_int32 * 3)(*nel), (C.c_double * 3)(*dx),
                                         E0, nu, rmin, C.c_void_p(U.data_ptr()),
                                         C.c_void_p(dEdz.data_ptr()),
                                         C.c_void_p(out.data_ptr()),
                                         C.c_void_p(stream.cuda_stream), msg, 256)
        assert rc == 0, msg.value
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)), call


def test_noalloc_refuses_host_buffers(T):
    """Host memory passed where device buffers belong is refused with
    TPO_E_ARG before anything is launched."""
    lib = T.load()
    nel = (4, 3, 2)
    ne, nn = 24, 5 * 4 * 3
    U = np.zeros(3 * nn)
    dEdz = np.zeros(ne)
    out = np.full(ne, 7.0)
    msg = C.create_string_buffer(256)
    launches = lib.tpo_kernel_launches()
    rc = lib.tpo_sensitivity_noalloc((C.c_int32 * 3)(*nel), (C.c_double * 3)(1, 1, 1),
                                     1.0, 0.3, 1.5, U.ctypes.data_as(C.c_void_p),
                                     dEdz.ctypes.data_as(C.c_void_p),
                                     out.ctypes.data_as(C.c_void_p), None, msg, 256)
    assert rc == T._lib.TPO_E_ARG
    assert b"device memory" in msg.value
    assert lib.tpo_kernel_launches() == launches
    assert np.all(out == 7.0)


def test_noalloc_rejects_meshes_beyond_its_maximum(T):
    lib = T.load()
    big = (128, 128, 65)               # 1,064,960 elements > 2**20
    assert big[0] * big[1] * big[2] > T._lib.NOALLOC_MAX_ELEMS
    msg = C.create_string_buffer(256)
    rc = lib.tpo_sensitivity_noalloc((C.c_int32 * 3)(*big), (C.c_double * 3)(1, 1, 1),
                                     1.0, 0.3, 1.5, None, None, None, None, msg, 256)
    assert rc == T._lib.TPO_E_ARG
    assert b"TPO_NOALLOC_MAX_ELEMS" in msg.value
