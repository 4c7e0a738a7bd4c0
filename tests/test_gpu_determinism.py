"""Run-to-run determinism of the stage and reverse-stage kernels: the same
inputs give the same bits. The kernels let the two halves of a block (the
warps of each run) drift apart between barriers; a missing barrier shows up
here as results that change between runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_forward_and_adjoint_repeat_bitwise(vt):
    pb = vt.Problem(vt.make_params(96, 96, p=3, integration_order=10, perturb_grid=0.2, time_step=1e-4))
    U0 = pb.array("U0")
    lam = np.random.default_rng(3).standard_normal(U0.shape)
    runs = []
    for _ in range(3):
        s = vt.Solver(pb)
        s.rk4(1e-4, 40)
        U = s.download().copy()
        s.upload(U0)
        s.adjoint_forward(1e-4, 10, 40)
        g = s.adjoint_backward(lam).copy()
        runs.append((U, g))
        s.close()
    for U, g in runs[1:]:
        np.testing.assert_array_equal(U, runs[0][0])
        np.testing.assert_array_equal(g, runs[0][1])
