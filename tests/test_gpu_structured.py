"""Set-up on the device (vt_create_structured) against the host precompute:
the same mesh, geometry and initial state up to CUDA's sin/cos/pow in the mesh
perturbation and the vortex, and runs that stay within the parity bar. The
reference's perturbation sin(pow(x + 6, y + 6)) evaluates sin at arguments up
to ~1e10, so a last-place difference between CUDA's and glibc's pow or sin is
amplified there; the states still agree to 1e-12 (to 1e-13 in most cases, and
bit for bit without perturbation)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("nx,ny,p,io,pert,init", [(16, 16, 3, 10, 0.2, 0), (24, 10, 2, 6, 0.1, 0),
                                                  (32, 8, 1, 8, 0.0, 1), (9, 7, 3, 19, 0.15, 1)])
def test_device_setup_matches_host(vt, nx, ny, p, io, pert, init):
    prm = vt.make_params(nx, ny, p=p, integration_order=io, perturb_grid=pert, U_initialization_type=init)
    ic = vt.vortex(epsilon=0.33, M_infty=0.48, x0=0.6, y0=-0.9)
    host = vt.Solver(vt.Problem(prm, ic))
    dev = vt.Solver.structured(prm, ic)
    assert rel(dev.download(), host.download()) < 1e-12
    if pert == 0.0 and init == 0:
        np.testing.assert_array_equal(dev.download(), host.download())
    host.rk4(1e-3, 20)
    dev.rk4(1e-3, 20)
    assert rel(dev.download(), host.download()) < 1e-12
    np.testing.assert_allclose(dev.totals(), host.totals(), rtol=1e-13)


def test_device_setup_is_fast_at_scale(vt):
    """768 x 768 cells (1,179,648 triangles): device set-up against host precompute."""
    prm = vt.make_params(768, 768, p=3, integration_order=10, perturb_grid=0.2)
    t0 = time.perf_counter()
    dev = vt.Solver.structured(prm)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    pb = vt.Problem(prm)
    host = vt.Solver(pb)
    t_host = time.perf_counter() - t0
    print(f"set-up at 768x768: device {t_dev:.3f} s, host precompute + upload {t_host:.3f} s")
    assert rel(dev.download(), host.download()) < 1e-13
