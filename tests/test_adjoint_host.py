"""Host-side pieces of the discrete adjoint, checked without a GPU:

* the binomial checkpoint schedule attains Griewank's bound and reverses the
  steps in order (against an independent dynamic program for small cases);
* the Roe flux in the kernels' algebra matches the oracle's restatement of
  Numericalflux.cpp, its dual-number Jacobian matches central differences of
  the oracle, and the hand-written reverse sweep is its exact transpose, on
  states where the entropy fix is and is not active;
* the torch restatement of the nodal vortex initial condition (used for the
  chain rule to the vortex parameters) equals the host precompute.
"""
from functools import lru_cache

import numpy as np
import pytest

import vt_oracle


@lru_cache(None)
def dp_cost(n, free):
    """Fewest plain steps to reverse n steps from a stored state with `free` more slots."""
    if n == 1:
        return 0
    if free == 0:
        return n * (n - 1) // 2
    return min(m + dp_cost(n - m, free - 1) + dp_cost(m, free) for m in range(1, n))


@pytest.mark.parametrize("n,S", [(1, 1), (2, 1), (7, 1), (10, 2), (33, 3), (60, 4), (100, 6), (57, 57)])
def test_schedule_is_optimal_small(vt, n, S):
    info = vt.checkpoint_plan(n, S)
    assert info["advance_steps"] == dp_cost(n, S - 1) == info["optimal_advance_steps"]
    assert info["stage_steps"] == n and info["adjoint_steps"] == n
    assert info["forward_sweep_steps"] == n - 1
    assert 1 <= info["slots_used"] <= S


@pytest.mark.parametrize("n,S", [(2000, 45), (2000, 2000), (300, 10), (10000, 100)])
def test_schedule_attains_bound(vt, n, S):
    info = vt.checkpoint_plan(n, S)
    assert info["advance_steps"] == info["optimal_advance_steps"]
    assert info["adjoint_steps"] == n
    if S >= n:  # every step start kept: each step advanced once
        assert info["advance_steps"] == n - 1


def test_schedule_rejects_bad_arguments(vt):
    with pytest.raises(vt.VortexError):
        vt.checkpoint_plan(0, 3)
    with pytest.raises(vt.VortexError):
        vt.checkpoint_plan(10, 0)


def random_states(rng, n, fix_l3=False):
    """Pairs of physical states (rho, rho u, rho v, rho E) and unit normals; with
    fix_l3 the velocities are nearly tangential so |u.n| < eps = ci/10 (the
    entropy fix of the middle eigenvalue is active)."""
    out = []
    for _ in range(n):
        th = rng.uniform(0, 2 * np.pi)
        nrm = np.array([np.cos(th), np.sin(th)])
        tang = np.array([-nrm[1], nrm[0]])
        st = []
        for _side in range(2):
            rho = rng.uniform(0.6, 1.4)
            if fix_l3:
                vel = tang * rng.uniform(-0.8, 0.8) + nrm * rng.uniform(-1e-3, 1e-3)
            else:
                vel = rng.uniform(-0.9, 0.9, 2)
            p = rng.uniform(1.5, 3.5)
            E = p / (rho * 0.4) + 0.5 * vel @ vel
            st.append(np.array([rho, rho * vel[0], rho * vel[1], rho * E]))
        out.append((st[0], st[1], nrm))
    return out


@pytest.mark.parametrize("fix_l3", [False, True])
def test_roe_flux_matches_oracle(vt, fix_l3):
    rng = np.random.default_rng(3 + fix_l3)
    for uL, uR, n in random_states(rng, 200, fix_l3):
        f, code = vt.roe_flux(uL, uR, n)
        g, gcode = vt_oracle.numerical_flux(uL, uR, n)
        assert code == gcode == 0
        np.testing.assert_allclose(f, g, rtol=1e-13, atol=1e-13 * np.abs(g).max())


@pytest.mark.parametrize("fix_l3", [False, True])
def test_roe_jvp_matches_central_differences_of_oracle(vt, fix_l3):
    rng = np.random.default_rng(11 + fix_l3)
    h = 1e-6
    for uL, uR, n in random_states(rng, 60, fix_l3):
        dL, dR = rng.standard_normal(4) * uL, rng.standard_normal(4) * uR
        if fix_l3:  # keep the perturbation inside the branch of the entropy fix
            dL[1:3] *= 1e-3
            dR[1:3] *= 1e-3
        jv = vt.roe_flux_jvp(uL, uR, n, dL, dR)
        fp, _ = vt_oracle.numerical_flux(uL + h * dL, uR + h * dR, n)
        fm, _ = vt_oracle.numerical_flux(uL - h * dL, uR - h * dR, n)
        fd = (fp - fm) / (2 * h)
        np.testing.assert_allclose(jv, fd, rtol=1e-6, atol=1e-7 * (np.abs(fd).max() + 1))


@pytest.mark.parametrize("fix_l3", [False, True])
def test_roe_vjp_is_transpose_of_jvp(vt, fix_l3):
    rng = np.random.default_rng(29 + fix_l3)
    for uL, uR, n in random_states(rng, 200, fix_l3):
        dL, dR, bf = rng.standard_normal(4), rng.standard_normal(4), rng.standard_normal(4)
        jv = vt.roe_flux_jvp(uL, uR, n, dL, dR)
        bL, bR = vt.roe_flux_vjp(uL, uR, n, bf)
        lhs, rhs = bf @ jv, bL @ dL + bR @ dR
        assert abs(lhs - rhs) <= 1e-13 * (abs(bf) @ abs(jv) + abs(bL) @ abs(dL) + abs(bR) @ abs(dR))


def test_torch_vortex_ic_equals_host_precompute(vt):
    import torch
    from vortex_transport_b200 import adjoint
    for eps, M, x0, y0 in [(0.3, 0.5, 0.0, 0.0), (0.35, 0.45, 0.4, -0.25), (0.2, 0.62, -1.3, 0.8)]:
        prm = vt.make_params(12, 10, p=3, integration_order=10, perturb_grid=0.15)
        pb = vt.Problem(prm, vt.vortex(epsilon=eps, M_infty=M, x0=x0, y0=y0))
        U = adjoint.vortex_ic(torch.from_numpy(pb.array("nodes_phys")), eps, M, x0, y0).numpy()
        np.testing.assert_allclose(U, pb.array("U0"), rtol=2e-15, atol=1e-14)
