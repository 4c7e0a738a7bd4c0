"""Why the batched inverse problem steps at dt = 3.65e-5 instead of 1.5e-4.

The reference's Roe flux dissipates with the speed ci = c2^2 (Numericalflux.cpp:117),
i.e. c^4 = M^-4 for this vortex: 256 at the lowest Mach number the parameter
search may try (M = 0.25). Run on the CPU oracle (the reference's own algorithm)
for the inverse problem's mesh (64 x 64 cells, p = 2, io = 10): at the configured
dt = 1.5e-4 RK4 reaches a non-physical state within the configured 300 steps;
at the stability rule's dt = 3.65e-5 (workloads.stable_dt at M = 0.25) the same
300 steps stay physical. So the inverse problem keeps the configured horizon
T = 300 x 1.5e-4 = 0.045 and reaches it in 1234 steps of 0.045 / 1234 = 3.647e-5.
"""
import numpy as np

import vt_oracle


def oracle_run(vt, dt, steps, mach=0.25):
    pb = vt.Problem(vt.make_params(64, 64, p=2, integration_order=10, time_step=dt),
                    vt.vortex(epsilon=0.3, M_infty=mach))
    om = vt_oracle.OracleMesh(2, pb.array("vertices"), pb.array("conn"), pb.array("type"),
                              pb.array("minv_ref"), pb.array("stiff_ref"), pb.array("phi_plus"),
                              pb.array("phi_minus"), pb.array("line_quad"))
    return om.step(pb.array("U0"), pb.array("F0"), dt, steps, 1)


def test_configured_time_step_blows_up_at_the_lowest_mach_number(vt):
    U, F, err = oracle_run(vt, 1.5e-4, 300)
    assert err.code in (1, 2, 3)


def test_stability_rule_time_step_stays_physical(vt):
    from vortex_transport_b200 import workloads

    dt = workloads.stable_dt(64, 2, 0.25)
    assert abs(dt - 3.65e-5) < 5e-8
    U, F, err = oracle_run(vt, dt, 300)
    assert err.code == 0
    assert np.all(np.isfinite(U)) and U[:, :, 0].min() > 0
    assert int(np.ceil(300 * 1.5e-4 / dt)) == 1234
