"""The multi-rank path of bench.py on CPU with gloo (world size 2): each rank
advances its own replica, the job time is the maximum over ranks, and the
reference arm runs and prints on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank's replica took a different time; the job is as slow as the slowest
        got = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
        dist.barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.5, 1: 2.5}


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25) == 3.25


def test_reference_arm_prints_on_rank_zero_only():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env.update(RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert ("unavailable" in line) or (line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference")


def _workloads():
    from conftest import load_package
    load_package()
    from vortex_transport_b200 import workloads
    return workloads


def test_partition_covers_and_balances():
    """The ensemble split: every instance on exactly one rank, each rank's
    DOF-stages within one instance of the mean, the same split on every call."""
    wl = _workloads()
    inst = wl.ensemble_instances(n=512, seed=1)
    costs = [wl.instance_cost(i, 500) for i in inst]
    for world in (1, 2, 3, 4, 8):
        parts = wl.partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(inst)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == wl.partition(costs, world)
    assert wl.partition([1.0] * 5, 2) == [[0, 2, 4], [1, 3]]
    assert wl.partition([], 3) == [[], [], []]


def _split_rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = _workloads()
        inst = wl.ensemble_instances(n=64, seed=1)
        mine = wl.partition([wl.instance_cost(i) for i in inst], world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)  # what the inverse problem gathers: one list per rank
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_partition_agrees_across_gloo_ranks():
    """Two ranks compute their shares on their own; together they hold every
    instance once, and both see the same split."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_split_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1]
    assert sorted(res[0][0] + res[0][1]) == list(range(64))
    assert res[0][0] and res[0][1]
