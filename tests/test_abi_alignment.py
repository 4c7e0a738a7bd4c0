"""The device-array entry points reject misaligned arrays before any device work.

Their kernels read states as double2 (16-byte accesses); a view that starts one
double into an array would fault inside a kernel. The checks run on the host
first, so these tests need no GPU: the pointers below are never dereferenced.
"""
import ctypes

import numpy as np


def fake_mesh(vt, pb, base):
    m = vt.vt_device_mesh()
    m.p, m.n_elements, m.n_line_points = pb.p, pb.K, pb.nfq
    for k, name in enumerate(("element_type", "neighbours", "det_jacobian", "inv_jacobian", "normals",
                              "side_lengths")):
        setattr(m, name, ctypes.c_void_p(base + 0x10000 * (k + 1)))
    keep = []
    for name, field in (("minv_ref", "inv_mass_ref"), ("stiff_ref", "stiffness_ref"),
                        ("line_quad", "line_quadrature"), ("phi_plus", "phi_plus"), ("phi_minus", "phi_minus")):
        a = np.ascontiguousarray(pb.array(name), dtype=np.float64)
        keep.append(a)
        setattr(m, field, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return m, keep


def test_noalloc_rejects_misaligned_state_views(vt):
    pb = vt.Problem(vt.make_params(8, 8, p=3, integration_order=10))
    mesh, keep = fake_mesh(vt, pb, 0x7f0000000000)
    err = vt.vt_error_info()
    for src, dst in ((0x7f0000100008, 0x7f0000200000), (0x7f0000100000, 0x7f0000200008)):
        st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(src), ctypes.c_void_p(dst),
                                          1e-3, 1, None, ctypes.byref(err))
        assert st == vt.VT_ERR_INVALID
        assert "16-byte aligned" in vt._message()


def test_noalloc_rejects_misaligned_mesh_arrays(vt):
    pb = vt.Problem(vt.make_params(8, 8, p=3, integration_order=10))
    mesh, keep = fake_mesh(vt, pb, 0x7f0000000000)
    mesh.det_jacobian = ctypes.c_void_p(0x7f0000300004)  # doubles need 8 bytes
    err = vt.vt_error_info()
    st = vt.lib().vt_step_rk4_noalloc(ctypes.byref(mesh), ctypes.c_void_p(0x7f0000100000),
                                      ctypes.c_void_p(0x7f0000200000), 1e-3, 1, None, ctypes.byref(err))
    assert st == vt.VT_ERR_INVALID
    assert "misaligned" in vt._message()
