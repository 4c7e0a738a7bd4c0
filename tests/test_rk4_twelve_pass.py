"""The stage kernels' grouping of the RK4 step, restated on the host.

The GPU stepper (vortex-transport_b200/csrc/vt_tile.cuh) forms classical RK4
(Timestepping.cpp:85-306) from its stage states in 12 state-vector passes:

    U1 = U + dt/2 k1,  U2 = U + dt/2 k2,  U3 = U + dt k3   (the reference's stage states)
    X  = (U + U1)/3 + dt/3 k2                                (stage 1)
    U_{n+1} = X + c (k4 + f U3),  c = dt/6, f = 1/(3 c)      (stage 3, U3/3 folded in)

This test applies that grouping with the oracle's right-hand side (the
reference's evolve_elem) and compares it with the oracle's own rk4, which
matches the reference build bit for bit: one step of the shipped vortex at its
time step and at one 100 times smaller (where the folded term f U3 is largest
against k4), and 400 steps of the shipped run. The GPU tests hold the kernels
themselves to the reference at 1e-12 after one step and 1e-9 after 10000.
"""
import numpy as np
import pytest

from conftest import golden


def twelve_pass_step(m, U, dt):
    import vt_oracle

    def k(V):
        out, err = m.rhs(V, vt_oracle.flux_from_state(V))
        assert err.code == 0
        return out

    k1 = k(U)
    U1 = U + (0.5 * dt) * k1
    k2 = k(U1)
    U2 = U + (0.5 * dt) * k2
    X = (U + U1) * (1.0 / 3.0) + (dt / 3.0) * k2
    k3 = k(U2)
    U3 = U + dt * k3
    k4 = k(U3)
    c = dt / 6.0
    f = (1.0 / 3.0) / c
    return X + c * (k4 + f * U3)


def rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.mark.parametrize("scale", [1.0, 0.01])
def test_one_step_matches_reference_rk4(scale):
    import vt_oracle
    g = golden("c1_p3_io10_rk4_10000")
    m = g.oracle_mesh()
    U0 = g["U0"]
    dt = g.meta["dt"] * scale
    ref, _, err = m.step(U0, vt_oracle.flux_from_state(U0), dt, 1, 1)
    assert err.code == 0
    got = twelve_pass_step(m, U0, dt)
    e = rel(got, ref)
    print(f"dt = {dt:.3e}: 12-pass step vs the reference's rk4, max relative difference {e:.2e}")
    assert e < 1e-14


def test_many_steps_match_reference_rk4():
    import vt_oracle
    g = golden("c1_p3_io10_rk4_10000")
    m = g.oracle_mesh()
    U = g["U0"]
    dt = g.meta["dt"]
    n = 400
    ref, _, err = m.step(U, vt_oracle.flux_from_state(U), dt, n, 1)
    assert err.code == 0
    for _ in range(n):
        U = twelve_pass_step(m, U, dt)
    e = rel(U, ref)
    print(f"{n} steps: 12-pass grouping vs the reference's rk4, max relative difference {e:.2e}")
    assert e < 1e-12
