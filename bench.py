"""Benchmark of the fused FP64 RK4 stepper (headline: DOF-stages/s at p=3).

Workload: the isentropic vortex (reference IC) on the 10x10 periodic domain,
768x768 cells = 1,179,648 triangles, p=3 (10 nodes), integration_order=10,
perturb_grid=0.2, RK4 with dt=1.4e-5. A step is one RK4 step over all
elements; one DOF-stage is one element node (4 conserved components) advanced
through one RK stage, so a step is K*Np*4 DOF-stages.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's own CPU code (oracle/_ref, the
reference compiled from its sources with -O2 -fopenmp) with all host threads on
the same 768x768 mesh (W untimed, then K timed RK4 steps). With N>1 (torchrun) every rank
advances its own replica of the headline problem (it needs no collective), the
ensemble and inverse-problem instances are split over the ranks
(workloads.partition, no exchange), and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 768
P, IO, PERTURB, DT = 3, 10, 0.2, 1.4e-5
NP = (P + 1) * (P + 2) // 2
# The roofline's unit of work, algorithmic HBM bytes per DOF-stage of the
# 3-register RK4 scheme: 16 state vectors of 4 doubles over 4 stages (128 B)
# plus per-element geometry and connectivity (124 B per element, i.e. 124/Np
# per node). The stepper itself makes 12 state-vector passes per step (the
# accumulator is written once and read once), i.e. it moves B_MOVED.
B_ALG = 128.0 + 124.0 / NP
B_MOVED = 96.0 + 124.0 / NP
WORKLOAD = (f"isentropic vortex, {NX}x{NY} cells ({2 * NX * NY:,} triangles), p={P}, "
            f"integration_order={IO}, perturb_grid={PERTURB}, RK4 dt={DT}")
METRIC = "FP64 DOF-stages/s p=3"
UNIT = "DOF-stages/s"
HARNESS = os.path.join(ROOT, "oracle", "_ref", "vt_ref_harness")
# single-thread sample: the same per-element work on 256x256 cells (131,072
# triangles, the reference's own OpenMP performance mesh size)
CPU_1T_CELLS = 256


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per stage launch at 768x768 from the committed full-size ncu capture
    (profiles/tile_stage_kernel_p3_768x768_traffic.txt), if present."""
    path = os.path.join(ROOT, "profiles", "tile_stage_kernel_p3_768x768_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.dev), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_harness(cells: int, steps: int, threads: int, warmup: int = 0):
    """The reference's own code (oracle/_ref/vt_ref_harness: its translation
    units and its time loop without the text dumps) on `cells` x `cells`;
    `warmup` untimed steps, then `steps` timed ones."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores",
               OMP_SCHEDULE="static", OMP_DYNAMIC="false")
    out = subprocess.run([HARNESS, "--nx", str(cells), "--ny", str(cells), "--p", str(P), "--io",
                          str(IO), "--perturb", str(PERTURB), "--dt", str(DT), "--steps", str(steps),
                          "--warmup", str(warmup), "--no-ops", "--time"], env=env, capture_output=True,
                         text=True, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_baseline():
    """The reference's own code timed on this host's cores: all threads on the
    headline mesh itself (768x768, 2 timed RK4 steps after 1 untimed, about 20 s
    of CPU work), and one thread on a 256x256 sample of the same per-element
    work (1 RK4 step)."""
    threads = os.cpu_count() or 1
    if os.path.exists(HARNESS):
        r = run_reference_harness(NX, 2, threads, warmup=1)
        r1 = run_reference_harness(CPU_1T_CELLS, 1, 1)
        return {"value": r["dof_stages_per_s"], "unit": UNIT, "cores": r["threads"], "kind": "reference",
                "same_config": True,
                "sample": (f"2 timed RK4 steps (after 1 untimed) of the headline workload itself "
                           f"({NX}x{NY} cells, p={P}, io={IO}, perturb {PERTURB}, dt {DT}); reference "
                           f"-O2 -fopenmp build, {r['threads']} threads"),
                "init_s": r["init_s"],
                "single_thread": {"value": r1["dof_stages_per_s"], "unit": UNIT, "cores": 1,
                                  "sample": (f"1 RK4 step of the same per-element work on {CPU_1T_CELLS}x"
                                             f"{CPU_1T_CELLS} cells ({2 * CPU_1T_CELLS ** 2:,} triangles), "
                                             "OMP_NUM_THREADS=1")}}
    # the C restatement when the reference build is absent
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import vt_oracle
    vt = import_package()
    cells = 64
    pb = vt.Problem(vt.make_params(cells, cells, p=P, integration_order=IO, perturb_grid=PERTURB))
    om = vt_oracle.OracleMesh(P, pb.array("vertices"), pb.array("conn"), pb.array("type"),
                              pb.array("minv_ref"), pb.array("stiff_ref"), pb.array("phi_plus"),
                              pb.array("phi_minus"), pb.array("line_quad"))
    steps = 5
    t0 = time.perf_counter()
    om.step(pb.array("U0"), pb.array("F0"), DT, steps, 1)
    dt = time.perf_counter() - t0
    return {"value": pb.K * NP * 4 * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} RK4 steps on {cells}x{cells} cells with the C restatement"}


def import_package():
    import importlib.util
    name = "vortex_transport_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "vortex-transport_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def ensemble(vt, steps: int, n: int = 512, device: int = 0, rank: int = 0, world: int = 1, pg=None):
    """The batched forward ensemble: n seeded vortex problems of uneven size and
    order (workloads.ensemble_instances, seed 1) advanced `steps` RK4 steps as
    one ragged batch (one persistent launch per stage and order group, the step
    in a CUDA graph, grid autotuned), against the same n problems run one at a
    time through the plain solver. Set-up (host precompute, device upload, graph
    capture, tuning) is outside both timed regions; both are host wall-clock
    around synchronous calls, the device idle at the start of each.

    With several ranks the instances are split by DOF-stages
    (workloads.partition, no exchange between ranks); each rank runs its share
    both ways, and each time is the slowest rank's. Every rank calls this."""
    import torch
    from vortex_transport_b200 import workloads

    inst_all = workloads.ensemble_instances(n=n, seed=1)
    parts = workloads.partition([workloads.instance_cost(i, steps) for i in inst_all], world)
    inst = [inst_all[i] for i in parts[rank]]

    def start():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        return time.perf_counter()

    t0 = time.perf_counter()
    pbs = workloads.build_problems(inst, threads=os.cpu_count() or 1)
    precompute_s = time.perf_counter() - t0
    batch = vt.Batch(pbs, device=device)
    batch.set_dt([i.dt for i in inst])
    tuned = batch.autotune(trials=2)
    batch.rk4(2)
    t0 = start()
    batch.rk4(steps)
    torch.cuda.synchronize()
    batched_s = max_over_ranks(time.perf_counter() - t0, pg)
    groups = batch.groups
    group_ms = batch.time_groups(5)  # each group's step on its own, device time
    batch.close()

    seq_local = 0.0
    for i, pb in enumerate(pbs):
        s = vt.Solver(pb, device=device)
        s.rk4(inst[i].dt, 2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.rk4(inst[i].dt, steps)
        seq_local += time.perf_counter() - t0
        s.close()
    seq_s = max_over_ranks(seq_local, pg)

    dof_stages = sum(workloads.instance_cost(i, steps) for i in inst_all)
    bytes_alg = 4 * steps * sum(2 * i.side * i.side * (128 * (i.p + 1) * (i.p + 2) // 2 + 124) for i in inst_all)
    peak, peak_kind = load_peaks()
    achieved = bytes_alg / batched_s / 1e9 / world
    per_group = []
    for (gp, gn, gk), ms in zip(groups, group_ms):
        gnp = (gp + 1) * (gp + 2) // 2
        rate = gk * gnp * 4 / (ms * 1e-3)
        gbs = gk * 4 * (128 * gnp + 124) / (ms * 1e-3) / 1e9
        per_group.append({"p": gp, "instances": gn, "elements": gk, "ms_per_step": ms,
                          "dof_stages_per_s": rate, "bytes_per_dof_stage": 128 + 124 / gnp,
                          "hbm_gbs": gbs, "frac": gbs / peak})
    return {
        "workload": (f"{n} seeded vortex problems (seed 1): side in {{16..128}}, p in {{1,2,3}}, "
                     f"eps~U[0.1,0.5], M~U[0.3,0.7], centre~U[-2,2]^2, perturb~U[0,0.2], io=10, "
                     f"{steps} RK4 steps each"),
        "dt_rule": f"dt = {workloads.ENSEMBLE_CFL} h / ((2p+1)(1 + M^-4)) (0.1 h/(2p+1) is unstable "
                   "in the reference: its Roe dissipation speed is c^4)",
        "dofs": int(workloads.dof_count(inst_all)),
        "ranks": world,
        "instances_per_rank": [len(q) for q in parts],
        "groups": [list(g) for g in groups],
        "per_group": per_group,
        "tuning": {"per_group": [{"p": g[0], "blocks_per_sm": b, "mapping": "pair" if m == 1 else "component"}
                                 for g, (b, m) in zip(groups, tuned)],
                   "note": "autotuned per group over both warp mappings and 1..3 resident blocks per SM"},
        "batched_solves_per_s": n / batched_s,
        "sequential_solves_per_s": n / seq_s,
        "speedup": seq_s / batched_s,
        "batched_dof_stages_per_s": dof_stages / batched_s,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "note": "per GPU" if world > 1 else "single GPU"},
        "batched_s": batched_s, "sequential_s": seq_s, "precompute_s": precompute_s,
    }


def adjoint(vt, steps: int = 2000, snapshots=None, device: int = 0):
    """Adjoint/forward time ratio on the adjoint configuration: the reference
    vortex on 128x128 cells (32,768 triangles), p=3, io=10, RK4 dt=8.8e-5.
    forward = `steps` plain RK4 steps (vt_step_rk4); adjoint = forward sweep
    with checkpoints + reverse sweep (recomputation included) through
    vt_adjoint_forward/backward, for each checkpoint budget (default: 45
    states on the binomial schedule, every step start, and every step start
    and stage state, 4 x steps states = 84 GB at 2000 steps: nothing
    recomputed). Device time with CUDA events on the solver's stream, after
    one untimed run of each."""
    snapshots = snapshots or (45, steps, 4 * steps)
    import numpy as np
    import torch

    dt = 8.8e-5
    pb = vt.Problem(vt.make_params(128, 128, p=3, integration_order=10, time_step=dt))
    s = vt.Solver(pb, device=device)
    U0 = pb.array("U0")
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", device))
    lamT = torch.tensor(np.random.default_rng(3).standard_normal(U0.shape), device=torch.device("cuda", device))

    def timed(fn):
        fn()  # untimed: graph capture, buffers
        s.upload(U0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def fwd():
        s.upload(U0)
        s.rk4(dt, steps)

    fwd_ms = timed(fwd)
    out = {"workload": f"reference vortex, 128x128 cells (32,768 triangles), p=3, io=10, RK4 dt={dt}, "
                       f"{steps} steps; J gradient w.r.t. U(0) (1.31M values)",
           "forward_ms": fwd_ms, "runs": []}
    for ns in snapshots:
        def adj(ns=ns):
            s.upload(U0)
            s.adjoint_forward(dt, steps, ns)
            s.adjoint_backward(lamT)
        ms = timed(adj)
        info = s.adjoint_info()
        out["runs"].append({"snapshots": ns, "adjoint_ms": ms, "ratio": ms / fwd_ms,
                            "state_mb_per_snapshot": U0.nbytes / 1e6,
                            "advance_steps": info["advance_steps"], "stage_steps": info["stage_steps"],
                            "optimal_advance_steps": info["optimal_advance_steps"],
                            "all_stages": bool(info["all_stages"])})
    s.close()
    return out


def inverse_problem(vt, iterations: int = 50, n: int = 128, device: int = 0, rank: int = 0, world: int = 1,
                    pg=None):
    """The batched adjoint inverse problem: n vortices on 64x64 cells (8,192
    triangles), p=2, observed at the configured horizon T = 300 x 1.5e-4 =
    0.045; seeded true (eps, M, x0, y0) and a perturbed guess; per-instance
    L-BFGS on the host with every loss evaluation one batched forward + reverse
    sweep (400 step starts kept on the binomial schedule, the rest recomputed).
    The configured dt = 1.5e-4 blows up at the
    lowest Mach number the search may try (0.25), as it does in the reference
    (its Roe dissipation speed is c^4 = M^-4 = 256; tests/test_inverse_time_step.py
    shows it on the oracle), so T is reached in 1234 steps of 0.045 / 1234 =
    3.647e-5, below the ensemble's stability rule at M = 0.25.

    With several ranks each solves its share of the vortices (the problems
    are independent); the solve time is the slowest rank's and the per-vortex
    results are gathered. Every rank calls this."""
    import numpy as np
    import torch
    from vortex_transport_b200 import inverse, workloads

    theta_all = inverse.true_parameters(n, seed=5)
    guess_all = inverse.perturbed_guess(theta_all, seed=6)
    mine = workloads.partition([1.0] * n, world)[rank]
    theta, guess = theta_all[mine], guess_all[mine]
    horizon = 300 * 1.5e-4
    steps = int(math.ceil(horizon / workloads.stable_dt(64, 2, float(inverse.LOWER[1]))))
    dt = horizon / steps
    t0 = time.perf_counter()
    # 400 stored step starts (80 GB for the 128 instances) on the binomial
    # schedule: every step start (1234, 248 GB) would not fit in HBM
    inv = inverse.BatchedInverse(theta, side=64, p=2, steps=steps, dt=dt, nsnapshots=min(steps, 400),
                                 device=device)
    setup_s = max_over_ranks(time.perf_counter() - t0, pg)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    x, f, done = inv.solve(guess, iterations=iterations)
    solve_s = max_over_ranks(time.perf_counter() - t0, pg)
    evaluations = int(max_over_ranks(float(inv.evaluations), pg))
    local = {"err0": np.abs(guess - theta).max(axis=1), "err": np.abs(x - theta).max(axis=1), "done": done,
             "ratio": f / np.maximum(inv.loss_and_grad(guess)[0], 1e-300)}
    if pg:
        got = [None] * world
        pg.all_gather_object(got, local)
    else:
        got = [local]
    err0, err, done_all, ratio = (np.concatenate([g[k] for g in got]) for k in ("err0", "err", "done", "ratio"))
    out = {"workload": f"{n} vortices, 64x64 cells (8,192 triangles) each, p=2, io=10, observed at T={horizon:g} "
                       f"(300 x 1.5e-4) reached in {steps} RK4 steps of dt={dt:.4g}; true eps~U[0.15,0.45], "
                       "M~U[0.3,0.6], centre~U[-1.5,1.5]^2 (seed 5); guess eps/M +-0.05, centre +-0.3 (seed 6)",
           "horizon": horizon, "steps": steps, "dt": dt,
           "dt_rule": "1.5e-4 blows up at M=0.25 in the reference's scheme (c^4 dissipation speed); "
                      "dt = T / ceil(T / stable_dt(64, 2, 0.25))",
           "ranks": world, "iterations_max": iterations, "accepted_steps_median": float(np.median(done_all)),
           "evaluations": evaluations, "solve_s": solve_s, "s_per_evaluation": solve_s / evaluations,
           "iterations_per_s": float(np.median(done_all)) / solve_s,
           "instance_iterations_per_s": float(np.sum(done_all)) / solve_s,
           "setup_s": setup_s, "max_param_error_initial": float(err0.max()),
           "max_param_error_final": float(err.max()),
           "median_param_error_final": float(np.median(err)),
           "loss_reduction_worst": float(ratio.max()),
           "checkpoints": inv.batch.adjoint_info()}
    inv.close()
    return out


def max_over_ranks(x: float, pg=None, device: str = "cuda") -> float:
    """The slowest rank's time: every rank's replica must be done, so the job
    time is the maximum (all ranks call this, in the same order)."""
    if not pg:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    if not os.path.exists(HARNESS):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/vt_ref_harness was not built "
                          "(needs the reference sources at build time)"}))
        return 0
    r = run_reference_harness(NX, args.steps, threads, warmup=args.warmup)
    value = r["dof_stages_per_s"]
    sample = (f"each step: one RK4 step of the headline workload itself ({NX}x{NY} cells, p={P}, io={IO}, "
              f"perturb {PERTURB}, dt {DT}), {args.warmup} untimed then {args.steps} timed; reference "
              f"compiled -O2 -fopenmp, {r['threads']} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * r["stepping_s"] / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the reference's isentropic-vortex IC on its generated mesh",
            "config": {"workload": WORKLOAD, "elements": 2 * NX * NY, "nodes_per_element": NP,
                       "sample": sample, "same_config": True, "init_s": r["init_s"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def b200_arm(args):
    import numpy as np
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    vt = import_package()

    cells = args.cells
    workload = WORKLOAD if cells == NX else WORKLOAD.replace(f"{NX}x{NY} cells ({2 * NX * NY:,}",
                                                             f"{cells}x{cells} cells ({2 * cells * cells:,}")
    prm = vt.make_params(cells, cells, p=P, integration_order=IO, perturb_grid=PERTURB, time_step=DT)
    pb = vt.Problem(prm)
    solver = vt.Solver(pb, device=local)
    K_el = pb.K
    dof_stages_per_step = K_el * NP * 4
    stream = torch.cuda.ExternalStream(solver.stream, device=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    # warm-up (also captures the step graph)
    solver.rk4(DT, max(args.warmup, 1))

    # ---- timed region: K steps, state resident in HBM -----------------------
    barrier()
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        solver.rk4_async(DT, args.steps)
        ev1.record(stream)
        solver.synchronize()
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg)
    barrier()
    value = world * dof_stages_per_step * args.steps / (ms * 1e-3)

    # ---- per-stage kernel times (individual launches, events) ---------------
    stage_ms = solver.profile_stages(DT, 5)

    # ---- end to end through the public API with host buffers -----------------
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 10))
    host_U = torch.empty((K_el, NP, 4), dtype=torch.float64, pin_memory=True).numpy()
    host_U[...] = solver.download()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        solver.upload(host_U)  # pinned host -> device
        vt.rk4(solver, DT, 1)
        solver.download(out=host_U)  # device -> pinned host
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), pg)
    e2e_value = world * dof_stages_per_step * e2e_steps / (e2e_ms * 1e-3) if e2e_steps else None
    state_bytes = K_el * NP * 4 * 8

    # independent instances split over the ranks (all ranks take part)
    ens = (ensemble(vt, args.ensemble_steps, device=local, rank=rank, world=world, pg=pg)
           if args.ensemble_steps > 0 else None)
    inv = (inverse_problem(vt, args.inverse_iters, device=local, rank=rank, world=world, pg=pg)
           if args.inverse_iters > 0 else None)
    if pg:
        pg.barrier()
    if rank == 0:
        peak, peak_kind = load_peaks()
        avg_launch_s = ms * 1e-3 / (4 * args.steps)
        bytes_per_launch = K_el * NP * B_ALG
        achieved = bytes_per_launch / avg_launch_s / 1e9
        traffic = profile_traffic()
        cpu = cpu_baseline() if world == 1 and not args.no_cpu_baseline else None
        adj = adjoint(vt, args.adjoint_steps, device=local) if world == 1 and args.adjoint_steps > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the reference's isentropic-vortex IC on its generated mesh",
            "config": {"workload": workload, "elements": K_el, "nodes_per_element": NP,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (4 resident state vectors of "
                             f"{state_bytes / 1e6:.0f} MB)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_dof_stage": B_ALG,
                         "bytes_per_dof_stage_moved": B_MOVED,
                         "frac_of_bytes_moved": achieved * (B_MOVED / B_ALG) / peak,
                         "note": "achieved = K*Np*B_alg per stage launch / mean launch time in "
                                 "the timed region (4 launches per step); B_alg is the 3-register RK4 "
                                 "scheme's 16 state-vector passes per step, the stepper makes 12 "
                                 "(bytes_per_dof_stage_moved), which traffic measures"},
            "stage_ms": [float(x) for x in stage_ms],
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": e2e_steps,
                    "note": "per step: pinned host U -> device, one RK4 step, device -> host U"},
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
            "ensemble": ens,
            "adjoint": adj,
            "inverse": inv,
        }
        print(json.dumps(line))
    solver.close()
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cells", type=int, default=NX, help="cells per side (profiling runs use fewer)")
    ap.add_argument("--ensemble-steps", type=int, default=500,
                    help="RK4 steps of the 512-problem ensemble comparison at N=1 (0 skips it)")
    ap.add_argument("--adjoint-steps", type=int, default=2000,
                    help="RK4 steps of the adjoint/forward time ratio at N=1 (0 skips it)")
    ap.add_argument("--inverse-iters", type=int, default=50,
                    help="L-BFGS iterations of the 128-vortex batched inverse problem (0 skips it)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
