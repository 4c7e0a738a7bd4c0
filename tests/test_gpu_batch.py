"""The batched ensemble (vt_batch_*): each instance of a batch must follow the
same arithmetic as a standalone solver built from the same problem, so the
results are compared bit for bit; errors must name the right instance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_problems(vt):
    specs = [  # (nx, ny, p, perturb, eps, dt): structured and unstructured tilings, all orders
        (16, 16, 3, 0.2, 0.3, 1e-3),
        (32, 32, 2, 0.1, 0.2, 8e-4),
        (10, 14, 1, 0.15, 0.45, 2e-3),
        (16, 8, 3, 0.0, 0.35, 6e-4),
        (48, 48, 1, 0.05, 0.25, 1e-3),
        (9, 7, 2, 0.2, 0.4, 1.5e-3),
    ]
    pbs, dts = [], []
    for nx, ny, p, pert, eps, dt in specs:
        prm = vt.make_params(nx, ny, p=p, integration_order=10, perturb_grid=pert)
        pbs.append(vt.Problem(prm, vt.vortex(epsilon=eps, x0=0.3 * p, y0=-0.2 * p)))
        dts.append(dt)
    return pbs, np.array(dts)


def test_batch_matches_standalone_bitwise(vt):
    pbs, dts = mixed_problems(vt)
    batch = vt.Batch(pbs)
    assert sorted(g[0] for g in batch.groups) == [1, 2, 3]
    batch.set_dt(dts)
    batch.rk4(5)
    for i, pb in enumerate(pbs):
        s = vt.Solver(pb)
        s.rk4(dts[i], 5)
        np.testing.assert_array_equal(batch.download(i), s.download(), err_msg=f"instance {i}")


def test_batch_reports_failing_instance(vt):
    pbs, dts = mixed_problems(vt)
    batch = vt.Batch(pbs)
    batch.set_dt(dts)
    U = pbs[3].array("U0").copy()
    U[17, :, 0] = -1.0
    batch.upload(3, U)
    with pytest.raises(vt.NonPhysicalState) as ei:
        batch.rk4(1)
    s = vt.Solver(pbs[3])
    s.upload(U)
    with pytest.raises(vt.NonPhysicalState) as ej:
        s.rk4(dts[3], 1)
    assert ei.value.instance == 3
    assert (ei.value.code, ei.value.element, ei.value.point, ei.value.side) == \
        (ej.value.code, ej.value.element, ej.value.point, ej.value.side)


def test_batch_autotune_keeps_state_and_caches(vt, tmp_path):
    pbs, dts = mixed_problems(vt)
    batch = vt.Batch(pbs)
    batch.set_dt(dts)
    before = [batch.download(i) for i in range(batch.n)]
    cache = str(tmp_path / "autotune.json")
    best = batch.autotune(trials=2, cache=cache)
    assert len(best) == len(batch.groups)
    assert all(1 <= b <= 32 and m in (0, 1) for b, m in best)
    for i in range(batch.n):
        np.testing.assert_array_equal(batch.download(i), before[i])
    again = vt.Batch(pbs).autotune(trials=2, cache=cache)  # read back from the cache
    assert again == best
    batch.rk4(3)
    mapping_of_p = {g[0]: m for g, (_, m) in zip(batch.groups, best)}
    for i, pb in enumerate(pbs):
        s = vt.Solver(pb)
        s.stage_mapping = mapping_of_p[pb.p]  # the same kernel as the instance's group
        s.rk4(dts[i], 3)
        np.testing.assert_array_equal(batch.download(i), s.download())


def test_ensemble_dt_factor_is_stable(vt):
    """A slice of the seeded ensemble runs its 500 steps at the stable time step."""
    from vortex_transport_b200 import workloads
    inst = workloads.ensemble_instances(n=12, seed=1)
    pbs = workloads.build_problems(inst)
    batch = vt.Batch(pbs)
    batch.set_dt([i.dt for i in inst])
    t0 = [vt.Solver(pb).totals() for pb in pbs[:2]]
    batch.rk4(500)
    for i in range(len(inst)):
        U = batch.download(i)
        assert np.all(np.isfinite(U)) and np.all(U[..., 0] > 0)
