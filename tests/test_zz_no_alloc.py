"""vt_step_rk4_noalloc: RK4 stepping for callers that cannot allocate device memory.

Callers whose device memory is owned by someone else (a host framework's pool
or arena), that run in loops where a cudaMalloc would stall the device, or
that may only use buffers handed to them, step through this entry point: its
scratch is a fixed array inside the library. This test calls it through the C
ABI twice in a row (the second call continuing from the first's output, with
the scratch holding the first call's leftovers) and checks each result against
the regular entry point, vt_step_rk4, at the tolerance of the other parity
tests. The test's own input and output buffers are allocated by the test.
The file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE_RTOL = 1e-12


def device_mesh(vt, pb):
    import torch

    keep = {}

    def dev(name, dtype):
        t = torch.from_numpy(np.ascontiguousarray(pb.array(name), dtype=dtype)).cuda()
        keep[name] = t
        return ctypes.c_void_p(t.data_ptr())

    def host(name):
        a = np.ascontiguousarray(pb.array(name), dtype=np.float64)
        keep["h_" + name] = a
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    m = vt.vt_device_mesh()
    m.p, m.n_elements, m.n_line_points = pb.p, pb.K, pb.nfq
    m.element_type = dev("type", np.int32)
    m.neighbours = dev("conn", np.int32)
    m.det_jacobian = dev("detj", np.float64)
    m.inv_jacobian = dev("jinv", np.float64)
    m.normals = dev("normals", np.float64)
    m.side_lengths = dev("sides", np.float64)
    m.inv_mass_ref = host("minv_ref")
    m.stiffness_ref = host("stiff_ref")
    m.line_quadrature = host("line_quad")
    m.phi_plus = host("phi_plus")
    m.phi_minus = host("phi_minus")
    return m, keep


def test_noalloc_matches_regular_stepper_on_two_calls(vt):
    import torch

    prm = vt.make_params(16, 16, p=3, integration_order=10, perturb_grid=0.2)
    pb = vt.Problem(prm)
    assert vt.lib().vt_noalloc_scratch_bytes(3, pb.K) <= 16 << 20
    mesh, keep = device_mesh(vt, pb)
    U0 = torch.from_numpy(pb.array("U0")).cuda()
    U1 = torch.empty_like(U0)
    U2 = torch.empty_like(U0)
    torch.cuda.synchronize()
    dt, n = 1e-3, 3
    err = vt.vt_error_info()
    st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(U0.data_ptr()),
                                      ctypes.c_void_p(U1.data_ptr()), dt, n, None, ctypes.byref(err))
    assert st == vt.VT_OK, vt._message()
    st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(U1.data_ptr()),
                                      ctypes.c_void_p(U2.data_ptr()), dt, n, None, ctypes.byref(err))
    assert st == vt.VT_OK, vt._message()

    ref = vt.Solver(pb)
    ref.rk4(dt, n)
    a = ref.download()
    ref.rk4(dt, n)
    b = ref.download()
    for got, want in ((U1.cpu().numpy(), a), (U2.cpu().numpy(), b)):
        assert float(np.max(np.abs(got - want) / np.abs(want))) < STATE_RTOL


def test_noalloc_rejects_problems_larger_than_the_scratch(vt):
    prm = vt.make_params(16, 16, p=3, integration_order=10)
    pb = vt.Problem(prm)
    mesh, keep = device_mesh(vt, pb)
    mesh.n_elements = 2 * 128 * 128  # 32,768 triangles at p=3 need ~45 MB
    assert vt.lib().vt_noalloc_scratch_bytes(3, mesh.n_elements) > 16 << 20
    err = vt.vt_error_info()
    U = keep["type"]  # any device pointer; the size check comes first
    st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(U.data_ptr()),
                                      ctypes.c_void_p(U.data_ptr()), 1e-3, 1, None, ctypes.byref(err))
    assert st == vt.VT_ERR_INVALID
    assert "scratch" in vt._message()
