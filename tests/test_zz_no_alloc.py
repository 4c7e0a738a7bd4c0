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


def _call(vt, mesh, src, dst, dt, n):
    err = vt.vt_error_info()
    st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(src.data_ptr()),
                                      ctypes.c_void_p(dst.data_ptr()), dt, n, None, ctypes.byref(err))
    return st, err


def test_noalloc_call_takes_no_device_memory(vt):
    """After a first call (which may load the kernels), a call leaves the
    device's free memory exactly as it was: nothing is allocated or freed."""
    import torch

    pb = vt.Problem(vt.make_params(16, 16, p=3, integration_order=10, perturb_grid=0.2))
    mesh, keep = device_mesh(vt, pb)
    U = torch.from_numpy(pb.array("U0")).cuda()
    V = torch.empty_like(U)
    torch.cuda.synchronize()
    assert _call(vt, mesh, U, V, 1e-3, 2)[0] == vt.VT_OK, vt._message()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert _call(vt, mesh, V, U, 1e-3, 2)[0] == vt.VT_OK, vt._message()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_in_place_matches_regular_stepper(vt):
    """dU_in and dU_out may be the same buffer."""
    import torch

    pb = vt.Problem(vt.make_params(16, 16, p=3, integration_order=10, perturb_grid=0.2))
    mesh, keep = device_mesh(vt, pb)
    U = torch.from_numpy(pb.array("U0")).cuda()
    torch.cuda.synchronize()
    st, _ = _call(vt, mesh, U, U, 1e-3, 3)
    assert st == vt.VT_OK, vt._message()
    ref = vt.Solver(pb)
    ref.rk4(1e-3, 3)
    want = ref.download()
    ref.close()
    assert float(np.max(np.abs(U.cpu().numpy() - want) / np.abs(want))) < STATE_RTOL


def test_noalloc_reports_a_nonphysical_state_like_the_regular_stepper(vt):
    """A planted negative density stops the step with the same code and the
    same first failing element, face point, side, step and stage as
    vt_step_rk4 reports through vt_last_error."""
    import torch

    pb = vt.Problem(vt.make_params(16, 16, p=2, integration_order=10))
    mesh, keep = device_mesh(vt, pb)
    U0 = pb.array("U0").copy()
    U0[37, 2, 0] = -0.5
    U = torch.from_numpy(U0).cuda()
    V = torch.empty_like(U)
    torch.cuda.synchronize()
    st, err = _call(vt, mesh, U, V, 1e-3, 2)
    ref = vt.Solver(pb)
    ref.upload(U0)
    with pytest.raises(vt.NonPhysicalState) as exc:
        ref.rk4(1e-3, 2)
    ref.close()
    want = exc.value
    assert st == want.status
    assert (err.code, err.element, err.point, err.side, err.step, err.stage) == \
        (want.code, want.element, want.point, want.side, want.step, want.stage)


def test_noalloc_rejects_a_neighbour_index_out_of_range(vt):
    """A neighbour index outside 0..K-1 in the caller's device arrays is found
    on the device (the packing kernel keeps every access in bounds) and
    reported as VT_ERR_INVALID."""
    import torch

    pb = vt.Problem(vt.make_params(16, 16, p=3, integration_order=10))
    mesh, keep = device_mesh(vt, pb)
    keep["conn"][5, 1] = pb.K + 7
    mesh.neighbours = ctypes.c_void_p(keep["conn"].data_ptr())
    U = torch.from_numpy(pb.array("U0")).cuda()
    V = torch.empty_like(U)
    torch.cuda.synchronize()
    st, _ = _call(vt, mesh, U, V, 1e-3, 1)
    assert st == vt.VT_ERR_INVALID
    assert "neighbour" in vt._message()
