"""Dump and restart (vt_save_state / vt_load_state): a run split by a dump
continues bit for bit like the unbroken run, time included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_restart_continues_bitwise(vt, tmp_path):
    prm = vt.make_params(24, 16, p=3, integration_order=10, perturb_grid=0.2)
    pb = vt.Problem(prm, vt.vortex(epsilon=0.35, x0=0.5))
    dt = 1e-3
    a = vt.Solver(pb)
    a.rk4(dt, 30)
    path = str(tmp_path / "mid.vts")
    a.save(path)
    t_mid = a.time
    a.rk4(dt, 30)
    b = vt.Solver(pb)
    b.load(path)
    assert b.time == t_mid
    b.rk4(dt, 30)
    np.testing.assert_array_equal(b.download(), a.download())
    assert b.time == a.time
    U, p, t = vt.read_state_file(path)
    assert p == 3 and U.shape == (pb.K, pb.Np, 4)


def test_load_rejects_other_mesh(vt, tmp_path):
    a = vt.Solver(vt.Problem(vt.make_params(8, 8, p=2)))
    path = str(tmp_path / "a.vts")
    a.save(path)
    b = vt.Solver(vt.Problem(vt.make_params(8, 6, p=2)))
    with pytest.raises(vt.VortexError):
        b.load(path)
