"""Pin the oracle: it must reproduce the reference's own outputs bit for bit.

The fixtures come from the reference compiled from its sources
(tests/golden/make_golden.py). The reference ships no tests, so these are the
known answers; the oracle restates Evolve.cpp / Numericalflux.cpp /
Timestepping.cpp with the same operation order and must match exactly.
"""
import numpy as np
import pytest

from conftest import Golden, golden, golden_paths

SHORT = [p for p in golden_paths() if "10000" not in p]


@pytest.mark.parametrize("path", SHORT, ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_rhs_and_steps_bitwise(path):
    g = Golden(path)
    m = g.oracle_mesh()
    geo = m.geometry()
    for key in ("jac", "jinv", "detj", "detjinv", "normals", "sides"):
        np.testing.assert_array_equal(geo[key], g[key], err_msg=key)
    if "rhs0" in g:
        r, err = m.rhs(g["U0"], g["F0"])
        assert err.code == 0
        np.testing.assert_array_equal(r, g["rhs0"])
    U, F, err = m.step(g["U0"], g["F0"], g.meta["dt"], g.meta["steps"], g.meta["stepping"])
    assert err.code == 0
    np.testing.assert_array_equal(U, g["U_final"])
    np.testing.assert_array_equal(F, g["F_final"])


def test_oracle_flux_refresh_matches_reference():
    """F after a step is the reference's nodal-flux formula of U (Timestepping.cpp:141-158)."""
    import vt_oracle
    g = golden("p3_io10_16x16_pert_rk4")
    np.testing.assert_array_equal(vt_oracle.flux_from_state(g["U_final"]), g["F_final"])


def test_oracle_shipped_10000_steps_bitwise():
    """Config 1 in full (128 triangles, p=3, T=10*sqrt(2), 10000 RK4 steps), every 2500 steps."""
    g = golden("c1_p3_io10_rk4_10000")
    m = g.oracle_mesh()
    U, F = g["U0"], g["F0"]
    for k in range(1, 5):
        U, F, err = m.step(U, F, g.meta["dt"], 2500, 1)
        assert err.code == 0
        np.testing.assert_array_equal(U, g[f"U_step{2500 * k}"])


def test_oracle_numerical_flux_error_codes():
    """The reference's exit conditions (Numericalflux.cpp:42-115) become codes 1/2/3."""
    import vt_oracle
    n = np.array([0.6, 0.8])
    good = np.array([1.0, 0.3, 0.2, 2.5])
    f, code = vt_oracle.numerical_flux(good, good, n)
    assert code == 0
    # consistency: F(u, u, n) is the physical normal flux
    rho, mu, mv, E = good
    u, v = mu / rho, mv / rho
    p = 0.4 * (E - 0.5 * rho * (u * u + v * v))
    un = u * n[0] + v * n[1]
    np.testing.assert_allclose(f, [rho * un, mu * un + p * n[0], mv * un + p * n[1], (E + p) * un],
                               rtol=1e-14, atol=1e-15)
    bad_rho = good.copy(); bad_rho[0] = -1.0
    assert vt_oracle.numerical_flux(bad_rho, good, n)[1] == 1
    assert vt_oracle.numerical_flux(good, bad_rho, n)[1] == 2
    bad_p = good.copy(); bad_p[3] = 0.01  # kinetic energy exceeds total energy
    assert vt_oracle.numerical_flux(bad_p, good, n)[1] == 1
    assert vt_oracle.numerical_flux(good, bad_p, n)[1] == 2


def test_oracle_reports_first_failing_element():
    """A planted negative density is reported at the lowest element index first."""
    g = golden("c1_p3_io10_rk4_1step")
    m = g.oracle_mesh()
    U = g["U0"].copy()
    U[77, :, 0] = -1.0
    U[90, :, 0] = -1.0
    _, err = m.rhs(U, g["F0"])
    # element 77's neighbours see it as the right state first if they come earlier
    assert err.code in (1, 2)
    assert err.element <= 77
    U2, F2, err2 = m.step(g["U0"], g["F0"], g.meta["dt"], 1, 1)
    assert err2.code == 0
