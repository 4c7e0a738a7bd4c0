"""The discrete adjoint on the GPU (vt_adjoint_*, vt_rhs_jvp/vjp, vt_tangent_rk4):

* per stage, <W, R'(U) V> = <R'(U)^T W, V> (adjoint kernels vs the dual-number
  tangent kernel) and R'(U) V against central differences of the stage
  kernel's right-hand side;
* over a run, the tangent-linear model and the checkpointed reverse sweep
  satisfy <lam_T, dU_T> = <lam_0, dU_0> to 1e-10, the reverse sweep is bitwise
  independent of the number of checkpoints (every stage state kept, or step
  starts on the binomial schedule), and its forward sweep is bitwise
  vt_step_rk4; the two-sided face phase (meshes that do not 2-colour) obeys
  the same stage identity as the edge-once one;
* gradients of the mass-weighted loss J = 1/2 ||U(T) - U*(T)||_M agree with
  finite differences of the forward stepper to 1e-6 relative at h = 1e-4,
  1e-5, 1e-6 (fourth-order differences; central ones at 1e-5 and 1e-6, whose
  O(h^2) error at 1e-4 is 1e-6 to 1e-5 here), along state directions and in
  the vortex parameters (eps, M, x0, y0) reached by the chain rule through the
  torch initial condition; the last test does this on the adjoint
  configuration itself (128x128 cells, p=3, 2000 steps, 45 checkpoints).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_RTOL = 1e-6
DOT_RTOL = 1e-10


def problem(vt, nx, ny, p, io=10, pert=0.2, **ic):
    prm = vt.make_params(nx, ny, p=p, integration_order=io, perturb_grid=pert)
    return vt.Problem(prm, vt.vortex(**ic))


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def state_scale(U):
    return np.abs(U).mean(axis=(0, 1))


def smooth_direction(pb, seed):
    """A smooth perturbation field: a few low Fourier modes of the 10x10
    periodic domain at the physical nodes, scaled per component like U. The
    truncation error of central differences (O(h^2)) is about 100 times
    smaller along it than along node-wise random noise of the same size."""
    rng = np.random.default_rng(seed)
    X = pb.array("nodes_phys")
    x, y = 2 * np.pi * X[..., 0] / 10.0, 2 * np.pi * X[..., 1] / 10.0
    U0 = pb.array("U0")
    d = np.zeros_like(U0)
    for c in range(4):
        for _ in range(4):
            kx, ky = rng.integers(0, 3, 2)
            ph = rng.uniform(0, 2 * np.pi)
            d[..., c] += rng.standard_normal() * np.cos(kx * x + ky * y + ph)
    return d * state_scale(U0)


def fd4(f, h):
    """Fourth-order central difference of the scalar function f at 0."""
    return (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)


def mass_loss(pb):
    detj = pb.array("detj")
    M = np.linalg.inv(pb.array("minv_ref"))

    def J(U, T):
        d = U - T
        return 0.5 * np.sum(detj[:, None, None] * d * np.einsum("ij,ejc->eic", M, d))

    def dJ(U, T):
        return detj[:, None, None] * np.einsum("ij,ejc->eic", M, U - T)

    return J, dJ


@pytest.mark.parametrize("nx,ny,p,io", [(16, 16, 3, 10), (12, 10, 2, 6), (10, 14, 1, 4), (8, 8, 0, 2),
                                        (9, 7, 3, 19)])
def test_rhs_vjp_is_transpose_of_jvp(vt, nx, ny, p, io):
    pb = problem(vt, nx, ny, p, io)
    s = vt.Solver(pb)
    rng = np.random.default_rng(p + 10 * io)
    U = pb.array("U0")
    V = rng.standard_normal(U.shape) * state_scale(U)
    W = rng.standard_normal(U.shape)
    JV = s.rhs_jvp(U, V)
    JtW = s.rhs_vjp(U, W)
    assert rel(np.sum(W * JV), np.sum(JtW * V)) < 1e-12


def test_rhs_vjp_two_sided_faces(vt):
    """A mesh that does not 2-colour (one element pair made self-neighbours
    across side 0, which keeps every side paired with itself) takes the
    two-sided face phase; the transpose identity must hold there too."""
    pb = problem(vt, 12, 10, 3, 10)
    conn = pb.array("conn").copy()
    a = 5
    b = conn[a, 2]  # side 0 is the vertical neighbour for both element types
    conn[a, 2], conn[b, 2] = a, b
    desc = vt.mesh_desc_from_arrays(pb.p, pb.array("type"), conn, pb.array("detj"), pb.array("jinv"),
                                    pb.array("normals"), pb.array("sides"), pb.array("minv_ref"),
                                    pb.array("stiff_ref"), pb.array("line_quad"), pb.array("phi_plus"),
                                    pb.array("phi_minus"))
    s = vt.Solver(desc)
    rng = np.random.default_rng(41)
    U = pb.array("U0")
    V = rng.standard_normal(U.shape) * state_scale(U)
    W = rng.standard_normal(U.shape)
    JV = s.rhs_jvp(U, V)
    JtW = s.rhs_vjp(U, W)
    assert rel(np.sum(W * JV), np.sum(JtW * V)) < 1e-12


@pytest.mark.parametrize("nx,ny,p,io", [(16, 16, 3, 10), (12, 10, 2, 6)])
def test_rhs_jvp_matches_central_differences(vt, nx, ny, p, io):
    pb = problem(vt, nx, ny, p, io)
    s = vt.Solver(pb)
    rng = np.random.default_rng(7)
    U = pb.array("U0")
    V = rng.standard_normal(U.shape) * state_scale(U)
    JV = s.rhs_jvp(U, V)
    h = 1e-6
    s.upload(U + h * V)
    Rp = s.rhs()
    s.upload(U - h * V)
    Rm = s.rhs()
    fd = (Rp - Rm) / (2 * h)
    np.testing.assert_allclose(JV, fd, rtol=0, atol=1e-7 * np.abs(fd).max())


@pytest.mark.parametrize("p,io", [(3, 10), (2, 6), (1, 4)])
def test_tangent_adjoint_dot_product_and_checkpoints(vt, p, io):
    pb = problem(vt, 16, 16, p, io)
    dt, n = 1e-3, 24
    U0 = pb.array("U0")
    rng = np.random.default_rng(5)
    d0 = rng.standard_normal(U0.shape) * state_scale(U0)
    lT = rng.standard_normal(U0.shape)
    s = vt.Solver(pb)
    dT = s.tangent_rk4(dt, n, d0)
    UT = s.download()
    ref = vt.Solver(pb)
    ref.rk4(dt, n)
    np.testing.assert_array_equal(UT, ref.download())
    lams = []
    for nsnap in (4 * n, n, 5, 2, 1):
        s.upload(U0)
        s.adjoint_forward(dt, n, nsnap)
        np.testing.assert_array_equal(s.download(), UT)
        info = s.adjoint_info()
        assert info["all_stages"] == (nsnap >= 4 * n)
        assert info["advance_steps"] == info["optimal_advance_steps"]
        assert info["slots_used"] <= nsnap
        lams.append(s.adjoint_backward(lT))
    for lam in lams[1:]:
        np.testing.assert_array_equal(lam, lams[0])
    np.testing.assert_array_equal(s.adjoint_backward(lT), lams[0])  # replays the forward sweep
    np.testing.assert_array_equal(s.download(), UT)  # the reverse sweep leaves U(T)
    assert rel(np.sum(lT * dT), np.sum(lams[0] * d0)) < DOT_RTOL
    s.upload(U0)
    np.testing.assert_array_equal(s.adjoint_rk4(dt, n, 5, lT), lams[0])  # the one-call entry
    np.testing.assert_array_equal(s.download(), UT)


def test_overlapped_recomputation_matches_kept_stage_states(vt):
    """The reverse sweep recomputes step i-1 on a second stream while step i is
    reversed (stage states in two alternating sets). On a mesh of 288 tiles,
    where both kernels are resident at once, the gradient with every step start
    kept and with 3 binomial checkpoints (advances into reused slots) equals,
    bit for bit, the one from the single-stream sweep over kept stage states,
    also when the backward sweep is replayed."""
    pb = problem(vt, 96, 96, 3, 10)
    dt, n = 2e-4, 20
    U0 = pb.array("U0")
    lT = np.random.default_rng(11).standard_normal(U0.shape)
    s = vt.Solver(pb)
    lams = {}
    for nsnap in (4 * n, n, 3):
        s.upload(U0)
        s.adjoint_forward(dt, n, nsnap)
        lams[nsnap] = s.adjoint_backward(lT)
        np.testing.assert_array_equal(s.adjoint_backward(lT), lams[nsnap])  # replayed
    np.testing.assert_array_equal(lams[n], lams[4 * n])
    np.testing.assert_array_equal(lams[3], lams[4 * n])


@pytest.mark.parametrize("p,io", [(3, 10), (2, 6), (1, 4)])
def test_state_gradient_matches_central_differences(vt, p, io):
    pb = problem(vt, 16, 16, p, io)
    target_pb = problem(vt, 16, 16, p, io, epsilon=0.35, x0=0.4, y0=-0.25)
    dt, n = 1e-3, 40
    J, dJ = mass_loss(pb)
    t = vt.Solver(target_pb)
    t.rk4(dt, n)
    T = t.download()
    U0 = pb.array("U0")
    s = vt.Solver(pb)
    s.adjoint_forward(dt, n, 7)
    lam0 = s.adjoint_backward(dJ(s.download(), T))
    d = smooth_direction(pb, 17)
    g = np.sum(lam0 * d)

    def run(U):
        s.upload(U)
        s.rk4(dt, n)
        return J(s.download(), T)

    for h in (1e-4, 1e-5, 1e-6):
        assert rel(fd4(lambda t: run(U0 + t * d), h), g) < FD_RTOL, h
    for h in (1e-5, 1e-6):
        fd = (run(U0 + h * d) - run(U0 - h * d)) / (2 * h)
        assert rel(fd, g) < FD_RTOL, (h, fd, g)


def _parameter_case(vt, nx, p, dt, n, nsnap, pert=0.0):
    import torch
    from vortex_transport_b200 import adjoint as adj
    pb = problem(vt, nx, nx, p, 10, pert)
    s = vt.Solver(pb)
    dev = torch.device("cuda", 0)
    nodes = torch.tensor(pb.array("nodes_phys"), device=dev)
    detj = torch.tensor(pb.array("detj"), device=dev)
    M = torch.tensor(adj.mass_matrix(pb), device=dev)
    with torch.no_grad():
        target = adj.rk4_run(adj.vortex_ic(nodes, 0.35, 0.5, 0.4, -0.25), s, dt, n, nsnap)

    def loss(U0):
        return adj.mass_weighted_loss(adj.rk4_run(U0, s, dt, n, nsnap), target, detj, M)

    def ic(th):
        return adj.vortex_ic(nodes, th[0], th[1], th[2], th[3])

    theta = torch.tensor([0.3, 0.5, 0.0, 0.0], dtype=torch.float64, device=dev, requires_grad=True)
    loss(ic(theta)).backward()
    return s, loss, ic, theta.detach(), theta.grad.cpu().numpy()


def check_parameter_gradients(loss, ic, theta, g, hs=(1e-4, 1e-5, 1e-6)):
    """dJ/dtheta_k (adjoint + torch chain rule) against finite differences:
    (a) fourth-order differences in theta_k, (b) central differences of J(U0)
    along the state direction v_k = dU0/dtheta_k (forward mode through the
    initial condition), which checks the adjoint alone. Central differences in
    theta_k themselves carry an O(h^2) error that is large for M (U0 is
    strongly curved in M: p = 1/(gamma M^2)), so they are not the check."""
    import torch
    for k in range(4):
        e = torch.zeros(4, dtype=torch.float64, device=theta.device)
        e[k] = 1.0
        with torch.no_grad():
            f = lambda h: float(loss(ic(theta + h * e)))  # noqa: E731
            for h in hs:
                fd = fd4(f, h)
                assert rel(fd, g[k]) < FD_RTOL, ("theta", k, h, fd, g[k])
        _, v = torch.autograd.functional.jvp(lambda t: ic(theta + t * e), torch.zeros((), dtype=torch.float64,
                                             device=theta.device), torch.ones((), dtype=torch.float64,
                                                                             device=theta.device))
        U0 = ic(theta).detach()
        with torch.no_grad():
            for h in hs:
                fd = float((loss(U0 + h * v) - loss(U0 - h * v)) / (2 * h))
                assert rel(fd, g[k]) < FD_RTOL, ("state direction", k, h, fd, g[k])


def test_parameter_gradient_through_torch(vt):
    s, loss, ic, theta, g = _parameter_case(vt, 16, 3, 1e-3, 40, 6, pert=0.2)
    check_parameter_gradients(loss, ic, theta, g)


def test_adjoint_configuration_gradient_checks(vt):
    """128x128 cells (32,768 triangles), p=3, 2000 RK4 steps at dt=8.8e-5, 45
    checkpoints: the parameter gradients and a smooth state direction against
    finite differences at h = 1e-4, 1e-5, 1e-6, and the dot-product test."""
    dt, n, nsnap = 8.8e-5, 2000, 45
    s, loss, ic, theta, g = _parameter_case(vt, 128, 3, dt, n, nsnap)
    info = s.adjoint_info()
    assert info["advance_steps"] == info["optimal_advance_steps"] and info["slots_used"] <= nsnap
    check_parameter_gradients(loss, ic, theta, g)
    # dot-product test on the full initial state
    pb = problem(vt, 128, 128, 3, 10, 0.0)
    U0 = pb.array("U0")
    rng = np.random.default_rng(23)
    d0 = rng.standard_normal(U0.shape) * state_scale(U0)
    lT = rng.standard_normal(U0.shape)
    s.upload(U0)
    dT = s.tangent_rk4(dt, n, d0)
    s.upload(U0)
    s.adjoint_forward(dt, n, nsnap)
    lam0 = s.adjoint_backward(lT)
    assert rel(np.sum(lT * dT), np.sum(lam0 * d0)) < DOT_RTOL
    # the state gradient along a smooth direction, by central differences
    Jn, dJn = mass_loss(pb)
    T = s.download() + 1e-3 * smooth_direction(pb, 31)
    s.upload(U0)
    s.adjoint_forward(dt, n, nsnap)
    lam0 = s.adjoint_backward(dJn(s.download(), T))
    ds = smooth_direction(pb, 29)
    gd = np.sum(lam0 * ds)

    def run(U):
        s.upload(U)
        s.rk4(dt, n)
        return Jn(s.download(), T)

    for h in (1e-4, 1e-5, 1e-6):
        assert rel(fd4(lambda t: run(U0 + t * ds), h), gd) < FD_RTOL, h
    for h in (1e-5, 1e-6):
        fd = (run(U0 + h * ds) - run(U0 - h * ds)) / (2 * h)
        assert rel(fd, gd) < FD_RTOL, (h, fd, gd)
