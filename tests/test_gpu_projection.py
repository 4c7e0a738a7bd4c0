"""The L2-projection initial condition on the device (vt_project_vortex)
against the host precompute (U_initialization_type=1, bit-exact to the
reference) and the reference's own projected state in the golden fixture.
The device evaluates exp and pow with CUDA's functions, so the states agree to
rounding, not bit for bit."""
import numpy as np
import pytest

from conftest import golden
from test_gpu_parity import problem_for

pytestmark = pytest.mark.gpu


def test_projection_matches_reference_fixture(vt):
    g = golden("p2_io10_8x8_l2proj_rk4")
    pb = problem_for(vt, g)
    s = vt.Solver(pb)
    s.project_vortex(pb)
    np.testing.assert_allclose(s.download(), g["U0"], rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("p,io", [(3, 10), (1, 6), (2, 12)])
def test_projection_matches_host_precompute(vt, p, io):
    ic = vt.vortex(epsilon=0.4, M_infty=0.45, x0=-0.8, y0=1.1)
    prm = vt.make_params(14, 10, p=p, integration_order=io, perturb_grid=0.15, U_initialization_type=1)
    pb = vt.Problem(prm, ic)
    s = vt.Solver(pb)
    s.upload(np.zeros((pb.K, pb.Np, 4)))
    s.project_vortex(pb, ic)
    np.testing.assert_allclose(s.download(), pb.array("U0"), rtol=1e-13, atol=1e-14)
