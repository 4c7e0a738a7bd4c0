"""The batched ensemble against the oracle, not only against the standalone
solver: instances of the seeded ensemble (workloads.ensemble_instances, seed 1)
covering p = 1, 2, 3 and the largest mesh side (128), advanced together as one
ragged batch at their own time steps, must each match the oracle's RK4 (the
reference's algorithm restated on the CPU) to 1e-12 relative per node after
every step of a short run (checked after step 1 and step 2)."""
import numpy as np
import pytest

import vt_oracle

pytestmark = pytest.mark.gpu

STATE_RTOL_PER_STEP = 1e-12


def picked_instances():
    from vortex_transport_b200 import workloads

    inst = workloads.ensemble_instances(n=512, seed=1)
    chosen = []
    for p in (1, 2, 3):
        chosen.append(next(i for i in inst if i.p == p and i.side != 128))
    for p in (3, 1):
        chosen.append(next(i for i in inst if i.p == p and i.side == 128))
    return chosen


def test_ensemble_instances_match_the_oracle(vt):
    from vortex_transport_b200 import workloads

    inst = picked_instances()
    assert sorted({i.p for i in inst}) == [1, 2, 3] and max(i.side for i in inst) == 128
    pbs = [workloads.build_problem(i) for i in inst]
    batch = vt.Batch(pbs)
    batch.set_dt([i.dt for i in inst])
    oracles = [vt_oracle.OracleMesh(i.p, pb.array("vertices"), pb.array("conn"), pb.array("type"),
                                    pb.array("minv_ref"), pb.array("stiff_ref"), pb.array("phi_plus"),
                                    pb.array("phi_minus"), pb.array("line_quad")) for i, pb in zip(inst, pbs)]
    want = [(pb.array("U0"), pb.array("F0")) for pb in pbs]
    for step in (1, 2):
        batch.rk4(1)
        for k, (i, pb) in enumerate(zip(inst, pbs)):
            U, F, err = oracles[k].step(want[k][0], want[k][1], i.dt, 1, 1)
            assert err.code == 0
            want[k] = (U, F)
            got = batch.download(k)
            dev = float(np.max(np.abs(got - U) / np.abs(U)))
            assert dev < STATE_RTOL_PER_STEP, (step, k, i.side, i.p, dev)
    batch.close()
