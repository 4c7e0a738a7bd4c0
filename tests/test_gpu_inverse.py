"""Batched adjoint and the batched inverse problem (vt_batch_adjoint_*):

* the reverse sweep over a batch group equals, bit for bit, each instance's
  reverse sweep on its own solver (same tiles, same face lists, same kernels),
  with one or several time steps among the instances;
* recovering (eps, M, x0, y0) of several vortices from their final states by
  per-instance L-BFGS on batched gradients converges to the true parameters.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dts", [(3e-4, 3e-4, 3e-4), (3e-4, 2e-4, 2.5e-4)])
def test_batch_adjoint_matches_single_solver(vt, dts):
    """Same and uneven time steps across the instances of one group."""
    prm = vt.make_params(16, 16, p=2, integration_order=10, perturb_grid=0.1)
    pbs = [vt.Problem(prm, vt.vortex(epsilon=e, M_infty=m, x0=x, y0=y))
           for e, m, x, y in [(0.3, 0.5, 0.0, 0.0), (0.2, 0.4, 1.0, -0.5), (0.4, 0.55, -1.2, 0.8)]]
    n = 30
    batch = vt.Batch(pbs)
    batch.set_dt(list(dts))
    assert len(batch.groups) == 1
    batch.adjoint_forward(n, 8)
    rng = np.random.default_rng(2)
    lams = [rng.standard_normal((pb.K, pb.Np, 4)) for pb in pbs]
    got = batch.adjoint_backward(lams)
    assert batch.adjoint_info()["advance_steps"] == batch.adjoint_info()["optimal_advance_steps"]
    import torch
    on_device = batch.adjoint_backward([torch.tensor(x, device="cuda") for x in lams])  # device-pointer path
    for i in range(len(pbs)):
        np.testing.assert_array_equal(on_device[i].cpu().numpy(), got[i])
        U = torch.empty((pbs[i].K, pbs[i].Np, 4), dtype=torch.float64, device="cuda")
        batch.download_device(i, U)
        np.testing.assert_array_equal(U.cpu().numpy(), batch.download(i))
    for i, pb in enumerate(pbs):
        s = vt.Solver(pb)
        s.adjoint_forward(dts[i], n, 8)
        np.testing.assert_array_equal(batch.download(i), s.download())
        np.testing.assert_array_equal(got[i], s.adjoint_backward(lams[i]))


def test_batched_inverse_recovers_parameters(vt):
    from vortex_transport_b200 import inverse
    theta = inverse.true_parameters(6, seed=11)
    guess = inverse.perturbed_guess(theta, seed=12)
    inv = inverse.BatchedInverse(theta, side=16, p=2, steps=60, dt=3e-4, nsnapshots=16)
    f0, _ = inv.loss_and_grad(guess)
    x, f, done = inv.solve(guess, iterations=30)
    err0 = np.abs(guess - theta).max(axis=1)
    err = np.abs(x - theta).max(axis=1)
    assert (err < 1e-4).all(), (err0, err)
    assert (f < 1e-8 * f0).all(), (f0, f)
    inv.close()
