"""Device-array entry points with a misaligned view, and the bounded waits.

A view starting one double into a device array is rejected with
VT_ERR_INVALID before any kernel runs. The stage kernels' bounded wait on their
bulk copies is made to give up through the test hook vt_test_bulk_wait (no copy
is issued, so none is in flight): the step reports the failure, leaves the
state untouched, and the context steps normally afterwards.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_entry_points_reject_misaligned_views(vt):
    import torch

    pb = vt.Problem(vt.make_params(8, 8, p=3, integration_order=10))
    s = vt.Solver(pb)
    buf = torch.zeros(pb.K * pb.Np * 4 + 2, dtype=torch.float64, device="cuda")
    off = buf.data_ptr() + 8  # one double in: 8-byte, not 16-byte aligned
    lib = vt.lib()
    assert lib.vt_upload_state_device(s._h, ctypes.c_void_p(off)) == vt.VT_ERR_INVALID
    assert lib.vt_download_state_device(s._h, ctypes.c_void_p(off)) == vt.VT_ERR_INVALID
    good = ctypes.c_void_p(buf.data_ptr())
    assert lib.vt_rhs_jvp(s._h, good, ctypes.c_void_p(off), good, 1) == vt.VT_ERR_INVALID
    assert lib.vt_rhs_vjp(s._h, good, good, ctypes.c_void_p(off), 1) == vt.VT_ERR_INVALID
    assert lib.vt_tangent_rk4(s._h, 1e-3, 1, ctypes.c_void_p(off), good, 1) == vt.VT_ERR_INVALID
    # the aligned view still works, and the state was not touched by the rejected calls
    U0 = pb.array("U0")
    assert lib.vt_download_state_device(s._h, good) == vt.VT_OK
    assert np.array_equal(buf[:pb.K * pb.Np * 4].cpu().numpy().reshape(U0.shape), U0)
    s.close()


def test_bounded_bulk_copy_wait_gives_up_and_the_context_recovers(vt):
    pb = vt.Problem(vt.make_params(8, 8, p=3, integration_order=10))
    dt = pb.params.time_step
    s = vt.Solver(pb)
    U0 = s.download()
    lib = vt.lib()
    assert lib.vt_test_bulk_wait(s._h, 16, 1) == vt.VT_OK
    st = lib.vt_step_rk4(s._h, dt, 1)
    assert st == vt.VT_ERR_CUDA
    assert "wait gave up" in vt._message()
    assert np.array_equal(s.download(), U0)  # no stage wrote anything
    assert lib.vt_test_bulk_wait(s._h, 0, 0) == vt.VT_OK
    s.rk4(dt, 2)
    ref = vt.Solver(pb)
    ref.rk4(dt, 2)
    assert np.array_equal(s.download(), ref.download())
    s.close()
    ref.close()
