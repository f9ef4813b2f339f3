#!/usr/bin/env python
"""Throughput of the multi-layer XPBD step on B200 (one JSON line on rank 0).

Default workload (the metric's configuration, config 5): the learned warm
start's Neo-Hookean block -- 64x32x32 cubes of 0.1 m, 6 tets per cube (70,785
vertices, 393,216 tets), per-tet E log-uniform in [1e4, 1e7] Pa, nu uniform in
[0.25, 0.45] (seeded), three layers (8^3-cube clusters, 4^3-cube clusters,
fine), dt = 1/60 s, base pinned, seeded surface impulse at t = 0.  Synthetic
data.  A step is one xpbdLayer3D.integrate step solved to residual 1e-4
(runUntilResSmallerThan = 1e-4, the stop rules of simpleMonitorError on the
device).

`value` is steps/s of the learned warm-start solve to residual 1e-4 on the
device-resident stepper (state in HBM, one CUDA graph per step with the
monitor as conditional nodes, L2 flushed between timed steps); the plain solve
of the same steps, both iteration counts and the FP32-vs-FP64 position error
are in `to_residual`.  `e2e` is steps/s of the plain solve to residual 1e-4
through the public host API (XpbdLayer3D.integrate -> mlx_layer_solve, host
buffers in and out every step).  `fixed_iterations` times the same scene at
the configuration's fixed iteration counts (the colour-sweep roofline).
Multi-GPU runs are independent replicas (weak scaling).

Other workloads (`--config`): 1 = `--replicas` copies of the 8x2x2
single-layer cantilever merged into one mesh, 2 = the plain multi-layer block
64x16x16, 3 = the 256-scene batch, 4 = the contact-heavy drop (2 and 4 also
run the learned leg, with a network trained in the run).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config C]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sim steps/sec & iters to residual 1e-4: learned warm-start vs plain, 1 B200"
WORKLOADS = {
    2: ("config2: plain multi-layer Neo-Hookean block 64x16x16 cubes (18785 vertices, 98304 tets), "
        "coarse 8^3-cube rigid clusters (5 it) + fine layer (10 it), dt=1/60, base pinned, "
        "seeded surface impulse at t=0"),
    3: ("config3: 256 independent Neo-Hookean blocks of 2k-40k tets (log-uniform, seeded; 696279 vertices, "
        "3352014 tets) merged into one mesh (colours overlaid as Mesh3D.mergeMesh), E log-uniform [1e4,1e6], "
        "nu=0.35, coarse 4^3-cube rigid clusters (5 it) + fine layer (10 it), dt=1/60, bases pinned, "
        "seeded surface impulses, per-colour tiles autotuned"),
    5: ("config5: learned warm-start workload, Neo-Hookean block 64x32x32 cubes (70785 vertices, 393216 tets), "
        "E log-uniform [1e4,1e7], nu [0.25,0.45], 3 layers (8^3-cube clusters 5 it, 4^3-cube clusters 5 it, fine 10 it), "
        "dt=1/60, base pinned, seeded surface impulse at t=0"),
    4: ("config4: contact-heavy drop, 32 StVK boxes of 12^3 cubes (70304 vertices, 331776 tets), E=5e5, nu=0.3, "
        "seeded rotations and heights 0.5-3 m over a ground plane + 4 analytic spheres (r 0.3-0.6 m), contacts "
        "detected on the device every step and coloured together with the elastic constraints, 3 layers "
        "(4^3-cube clusters 1 it, 2^3-cube clusters 4 it, fine 10 it), "
        "contact resistance 0.9, dt=1/120; timed after the boxes have landed"),
}
WORKLOAD = WORKLOADS[5]
REPLICAS = 4096


def config1_workload(copies):
    nv, nt = 81 * copies, 192 * copies
    return (f"config1: {copies} independent copies of the 8x2x2 StVK cantilever (81 vertices, 192 tets each; "
            f"{nv} vertices, {nt} tets) merged into one mesh (colours overlaid as Mesh3D.mergeMesh), E=1e5, nu=0.3, "
            "one layer [0] (20 it), dt=0.01, x=0 faces pinned, undamped")


def max_over_ranks(x, dist, device="cuda"):
    """The max of a per-rank float over the process group (the job's time is
    its slowest rank's); `x` itself without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", rank))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def profiled_dram_bytes_per_tet(kernel="k_project_color"):
    """DRAM bytes per projected tet of `kernel` from the committed ncu summary
    of this workload (profiles/<kernel>_config<N>.json), or None."""
    f = ROOT / "profiles" / f"{kernel}_config{CONFIG}.json"
    if f.exists():
        return float(json.loads(f.read_text())["dram_bytes_per_tet"])
    return None


def measured_peak_hbm():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        if d.get("hbm_gbs"):
            return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


CONFIG = 5
# configurations whose line is the metric: the learned warm start vs the
# plain solve, both to residual 1e-4
RESIDUAL_CONFIGS = (2, 4, 5)
RUN_UNTIL = 1e-4


def make_scene():
    from multilayersolver2024_b200 import scenes
    if CONFIG == 1:
        return scenes.config1_replicated(REPLICAS)
    return {2: scenes.config2, 3: scenes.config3, 4: scenes.config4, 5: scenes.config5}[CONFIG]()


def make_training_scene():
    """Another seed of the workload's scene class (other materials, impulse
    or drop): the warm start's network is trained on its solver records when
    no trained network is shipped for the workload."""
    from multilayersolver2024_b200 import scenes
    return {2: lambda: scenes.config2(seed=3), 4: lambda: scenes.config4(seed=14),
            5: lambda: scenes.config5(seed=6)}[CONFIG]()


def start_velocity(scene, m):
    """Velocity at t = 0: the scene's seeded impulse, if it has one."""
    if scene.impulse is not None:
        m.v[scene.impulse[0] - 1] += scene.impulse[1]


def make_integrator(scene, precision, residual=False, cap=15000, host_contacts=False):
    """The scene's integrator settings.  `host_contacts`: the step takes a
    host contact list (mlx_layer_solve), which keeps the reference's contact
    order (contacts coloured with the elastic constraints need the contacts
    detected on the device)."""
    from multilayersolver2024_b200 import XpbdLayer3D
    integ = XpbdLayer3D()
    integ.Gravity = scene.gravity
    integ.setLayers(scene.layers)
    integ.iterations = list(scene.iterations)
    integ.customRigidSets = scene.custom_sets
    integ.precision = precision
    integ.contactResistance = scene.settings.get("contactResistance", integ.contactResistance)
    integ.contactColoring = bool(scene.settings.get("contactColoring", False)) and not host_contacts
    if residual:
        integ.computeResiduals = True
        integ.runUntilResSmallerThan = RUN_UNTIL
        integ.hangingStop = cap
    return integ


def cpu_port(nsteps, threads, state=None, residual=False, cap=15000, budget_s=None):
    """The oracle (FP64 C++ restatement of the reference path, all given host
    threads) on the same workload from the scene's t = 0 state or from
    `state` = (positions, velocities): (steps, seconds, projectGS iterations
    per step).  With `residual` every step runs to residual 1e-4 (at most
    `cap` iterations); with `budget_s` steps stop once that much time has
    passed (at least one step)."""
    from oracle import oracle as O
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet, StepCache
    O.load().orc_set_threads(threads)
    sc = make_scene()
    integ = make_integrator(sc, 1, residual, cap)
    m = sc.mesh
    start_velocity(sc, m)
    if state is not None:
        m.p, m.v = (a.copy() for a in state)
    cache = StepCache()

    def contacts():
        # simulate3D's loop: the finders on the step-start positions
        return O.find_contacts(sc.contact_finders, m.p) if sc.contact_finders else ContactSet()

    t0 = time.perf_counter()
    iters = []
    for frame in range(1, nsteps + 1):
        if residual:
            integ.runUntilResSmallerThan = RUN_UNTIL
        iters.append(int(O.integrate(integ, m, sc.h, contacts(), cache, frame)[1]))
        if budget_s is not None and time.perf_counter() - t0 >= budget_s:
            break
    return len(iters), time.perf_counter() - t0, iters


# untimed steps of the device stepper that bring a scene into its timed phase
# (config 4: the boxes have landed on the obstacles after 150 steps, 1.25 s)
ADVANCE = {4: 150}
_PHASE = {}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    # the reference arm runs the oracle alone: its scenes are coloured by the
    # oracle's own first-fit colouring, so the product library is never loaded
    from oracle import oracle as O
    from multilayersolver2024_b200 import mesh3d
    mesh3d.use_coloring(O.greedy_coloring)
    threads = os.cpu_count() or 1
    if CONFIG in RESIDUAL_CONFIGS:
        # full steps to residual 1e-4 (the metric's solve), as many as fit a
        # bounded time; every step is a whole step, none is extrapolated
        n, dt, iters = cpu_port(max(args.warmup, 0) + args.steps, threads, residual=True, budget_s=args.ref_budget)
        sample = (f"{n} consecutive steps of the full workload from t = 0, each solved to residual 1e-4 "
                  f"(projectGS iterations {iters}; oracle restatement, OpenMP over the tets of a colour; stops "
                  f"once {args.ref_budget:.0f} s have passed; MATLAB, the reference's runtime, is not installed)")
        solver = "plain multi-layer to residual 1e-4, CPU port"
    else:
        n, dt, _ = cpu_port(max(args.warmup, 0) + args.steps, threads)
        sample = (f"{n} consecutive steps of the full workload (oracle restatement; MATLAB, the reference's "
                  "runtime, is not installed)")
        solver = "plain multi-layer, CPU port"
    value = n / dt
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "solver": solver},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local):
    import torch
    from multilayersolver2024_b200 import MLX_ENERGY_NEOHOOKEAN, MLX_FP32, MLX_FP64, StepCache, load
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet, ResidentSim, Solver, find_boundary_vertices

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    lib = load()
    assert lib.mlx_device_count() > 0, "no sm_100 device visible"

    def barrier():
        if dist:
            dist.barrier()

    sc = make_scene()
    m = sc.mesh
    diag = m.bbox_diagonal()
    sets = sc.custom_sets
    ls = find_boundary_vertices(m, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    advance = ADVANCE.get(CONFIG, 0) if args.advance is None else args.advance

    def stepper(precision, residual, state=None):
        integ = make_integrator(sc, precision, residual, args.residual_cap)
        solver = Solver(m, precision=precision, device=local, material="lame")
        if state is None:
            sim = ResidentSim(solver, integ, ls, sc.h, p0=m.p, v0=np.zeros_like(m.p))
            if sc.impulse is not None:
                sim.add_velocity(sc.impulse[0], sc.impulse[1])
        else:
            sim = ResidentSim(solver, integ, ls, sc.h, p0=state[0], v0=state[1])
        if sc.contact_finders:
            sim.set_obstacles(sc.contact_finders, restitution=1e-2)
        return solver, sim

    # ---- fixed iteration counts (the configuration's own): colour-sweep
    # roofline and steps/s ----
    solver, sim = stepper(MLX_FP32, False)
    if advance:
        sim.step(advance, graph=True)
        torch.cuda.synchronize()
        _PHASE["state"] = tuple(a.copy() for a in sim.state()[:2])
    tuned = None
    if args.autotune:
        before, after = sim.autotune(reps=5)
        tuned = {"step_ms_default_tiles": before, "step_ms_tuned_tiles": after}
    sim.sweep_timing(True)
    for _ in range(args.warmup):
        sim.step(1, graph=True)
    torch.cuda.synchronize()
    sim.sweep_stats(reset=True)
    contacts_at_start = sim.contact_count() if sc.contact_finders else None
    residual_metric = CONFIG in RESIDUAL_CONFIGS and not args.no_residual_leg
    clocks = ClockSampler(local)
    if not residual_metric:
        clocks.start()
    barrier()
    torch.cuda.synchronize()
    fixed_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        fixed_ms += sim.step(1, graph=True, timed=True)
    torch.cuda.synchronize()
    barrier()
    if not residual_metric:
        clocks.stop()
    sweep_ms, sweep_bytes, sweep_launches = sim.sweep_stats(reset=True)
    contacts_at_end = sim.contact_count() if sc.contact_finders else None
    fixed_max_ms = max_over_ranks(fixed_ms, dist)
    fixed_value = args.steps * world / (fixed_max_ms / 1000.0)
    fixed_launches = sim.launches_per_step
    finite = bool(np.all(np.isfinite(sim.state()[0])))
    solver_launch_path = solver.launch_path
    solver.close()
    state0 = _PHASE.get("state")
    reference_order = None
    if sc.settings.get("contactColoring"):
        # the same steps with the reference's contact order (contacts after
        # the colours, Jacobi), for the cost of colouring the contacts
        sc.settings["contactColoring"] = False
        solver_r, sim_r = stepper(MLX_FP32, False, state0)
        for _ in range(args.warmup):
            sim_r.step(1, graph=True)
        ref_ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ref_ms += sim_r.step(1, graph=True, timed=True)
        solver_r.close()
        sc.settings["contactColoring"] = True
        reference_order = {"steps_per_s": args.steps / (ref_ms / 1000.0),
                           "note": "fixed iterations, contacts after the colours (xpbdLayer3D.m:330, 422-485)"}

    # ---- to residual 1e-4: the plain solve, the learned warm start and the
    # FP64 plain solve of the same steps ----
    to_res = None
    if residual_metric:
        from multilayersolver2024_b200.learned import collect_warm_start_data, fit_warm_start
        from multilayersolver2024_b200.warm_start_training import DEFAULT_NET, load_warm_start

        def run_leg(sim3, n, timed, record_clocks=False):
            iters, ms_steps, finals, fallbacks = [], [], [], []
            if record_clocks:
                clocks.start()
            barrier()
            for _ in range(n):
                if timed:
                    flush.zero_()
                    torch.cuda.synchronize()
                ms_steps.append(sim3.step(1, graph=not args.host_monitor, timed=True))
                ra, it_total, _, status = sim3.monitor()
                iters.append(int(it_total))
                finals.append(float(ra[-1]))
                if getattr(sim3, "_ws_nb", 0):
                    fallbacks.append(sim3.warm_start_fallbacks())
            barrier()
            if record_clocks:
                clocks.stop()
            return {"iterations_per_step": iters, "ms_per_step": ms_steps,
                    "steps_per_s": len(ms_steps) / (max_over_ranks(sum(ms_steps), dist) / 1000.0),
                    "final_residual": finals, "reached": [bool(abs(r) <= RUN_UNTIL) for r in finals],
                    "clusters_fallen_back_per_step": fallbacks or None}

        # the network: shipped (trained on 20k block-steps by
        # warm_start_training) for config 5, else trained here on recorded
        # steps of another seed of the scene class
        t0 = time.perf_counter()
        if CONFIG == 5 and DEFAULT_NET.exists() and not args.train_in_bench:
            net, fn, on, meta = load_warm_start(DEFAULT_NET)
            training = {"source": f"shipped network {DEFAULT_NET.name} (warm_start_training)", **meta}
        else:
            tsc = make_training_scene()
            integ_t = make_integrator(tsc, MLX_FP32, True, args.residual_cap)
            ls_t = find_boundary_vertices(tsc.mesh, tsc.custom_sets,
                                          [int(tsc.custom_sets[:, c].max(initial=0))
                                           for c in range(tsc.custom_sets.shape[1])])
            solver_t = Solver(tsc.mesh, precision=MLX_FP32, device=local, material="lame")
            if advance:
                solver_a = Solver(tsc.mesh, precision=MLX_FP32, device=local, material="lame")
                sim_a = ResidentSim(solver_a, make_integrator(tsc, MLX_FP32), ls_t, tsc.h, p0=tsc.mesh.p,
                                    v0=np.zeros_like(tsc.mesh.p))
                sim_a.set_obstacles(tsc.contact_finders, restitution=1e-2)
                sim_a.step(advance, graph=True)
                pa, va = sim_a.state()
                solver_a.close()
                sim_t = ResidentSim(solver_t, integ_t, ls_t, tsc.h, p0=pa, v0=va)
            else:
                sim_t = ResidentSim(solver_t, integ_t, ls_t, tsc.h, p0=tsc.mesh.p, v0=np.zeros_like(tsc.mesh.p))
                if tsc.impulse is not None:
                    sim_t.add_velocity(tsc.impulse[0], tsc.impulse[1])
            if tsc.contact_finders:
                sim_t.set_obstacles(tsc.contact_finders, restitution=1e-2)
            ftr, ttr, _ = collect_warm_start_data(sim_t, args.learned_train_steps)
            solver_t.close()
            net, fn, on, losses = fit_warm_start(ftr, ttr, epochs=300, lr=2e-3, batch=128)
            training = {"source": f"trained in this run on {args.learned_train_steps} recorded steps of "
                                  f"{tsc.name}", "rows": int(ftr.shape[0]), "epochs": 300,
                        "loss_first_last": [float(losses[0]), float(losses[-1])]}
        training["seconds_in_bench"] = time.perf_counter() - t0

        # the PCG in the layer solve (Newton-PCG corrections of the last
        # layer) covers the Neo-Hookean pair
        use_pcg = m.energy_type == MLX_ENERGY_NEOHOOKEAN and args.layer_pcg > 0
        full = "learned_pcg" if use_pcg else "learned"
        plan = [("plain", MLX_FP32, False, False), ("learned", MLX_FP32, True, False)]
        if use_pcg:
            plan += [("layer_pcg", MLX_FP32, False, True), ("learned_pcg", MLX_FP32, True, True)]
        plan.append(("plain_fp64", MLX_FP64, False, False))
        if args.legs:
            # profiling runs: only the named legs (each leg's work is unchanged)
            plan = [x for x in plan if x[0] in args.legs.split(",") or x[0] == full]
        legs, states = {}, {}
        for name, precision, warm, pcg in plan:
            solver3, sim3 = stepper(precision, True, state0)
            if warm:
                sim3.warm_start(record=False, mode=1, net=net, feature_norm=fn, output_norm=on,
                                fallback_residual=args.fallback_residual)
            if pcg:
                solver3.layer_pcg(args.layer_pcg, args.layer_pcg_every)
            run_leg(sim3, args.warmup, timed=False)
            legs[name] = run_leg(sim3, args.steps, timed=True, record_clocks=(name == full))
            states[name] = sim3.state()[0]
            if name == "plain":
                states["plain_state"] = sim3.state()[:2]
            solver3.close()
        net.close()
        # one step from the same state (the plain FP32 leg's last): the
        # kernels' own error, apart from any divergence of the trajectories
        one = {}
        if "plain_state" in states and "plain_fp64" in legs:
            for name, precision in (("plain", MLX_FP32), ("plain_fp64", MLX_FP64)):
                solver3, sim3 = stepper(precision, True, states["plain_state"])
                sim3.step(1, graph=True)
                one[name] = sim3.state()[0]
                solver3.close()
        fu = legs[full]
        pl = legs.get("plain")
        to_res = {"run_until": RUN_UNTIL, "hanging_stop": args.residual_cap, "untimed_steps_before": args.warmup,
                  "steps": args.steps, "value_leg": full, "plain": pl,
                  "learned_warm_start": ({**legs["learned"], "training": training,
                                          "fallback_residual_m": args.fallback_residual} if "learned" in legs
                                         else {"training": training}),
                  "plain_fp64": ({k: legs["plain_fp64"][k] for k in ("iterations_per_step", "steps_per_s",
                                                                       "final_residual")}
                                 if "plain_fp64" in legs else None),
                  "value_over_plain_steps_per_s": fu["steps_per_s"] / pl["steps_per_s"] if pl else None,
                  "plain_over_value_iterations": (sum(pl["iterations_per_step"]) /
                                                  max(sum(fu["iterations_per_step"]), 1)) if pl else None,
                  "ablation_steps_per_s": {k: legs[k]["steps_per_s"] for k in legs},
                  "monitor": "device (layers as conditional IF nodes, projectGS as conditional WHILE nodes)"}
        for name in ("layer_pcg", "learned_pcg"):
            if name in legs:
                to_res[name] = {**legs[name], "pcg_iterations": args.layer_pcg,
                                "gs_iterations_between": args.layer_pcg_every}

        def err(a, b):
            return float(np.abs(states[a] - states[b]).max() / diag) if a in states and b in states else None

        parity = {"reference": "FP64 plain solve of the same steps on the GPU (the FP64 path matches the CPU "
                               "oracle to 1e-9)",
                  "max_rel_pos_err": err(full, "plain_fp64"), "max_rel_pos_err_of": full,
                  "max_rel_pos_err_learned": err("learned", "plain_fp64"),
                  "max_rel_pos_err_layer_pcg": err("layer_pcg", "plain_fp64"),
                  "max_rel_pos_err_plain_fp32": err("plain", "plain_fp64"),
                  "learned_vs_plain_fp32": err("learned", "plain"),
                  "after_steps": args.warmup + args.steps,
                  "one_step_plain_fp32": (float(np.abs(one["plain"] - one["plain_fp64"]).max() / diag)
                                          if one else None),
                  "one_step_note": "FP32 and FP64 plain solves to residual 1e-4, one step from the same state",
                  "unit": "max |x - x_ref| / bounding-box diagonal"}

    # ---- e2e: public host API, host buffers, every step copies in and out ----
    sc2 = make_scene()
    m2 = sc2.mesh
    integ2 = make_integrator(sc2, MLX_FP32, residual_metric, args.residual_cap, host_contacts=True)
    cache = StepCache()
    start_velocity(sc2, m2)
    if advance:
        m2.p, m2.v = (a.copy() for a in state0)
    from multilayersolver2024_b200.contacts import find_contacts
    contact_bytes, e2e_iters = [], []

    def e2e_step(frame):
        # simulate3D's step: the finders on the step-start positions (on the
        # device, mlx_find_contacts), then integrate (mlx_layer_solve)
        cs = find_contacts(integ2.solver(m2), sc2.contact_finders, m2.p) if sc2.contact_finders else ContactSet()
        contact_bytes.append(cs.vertex_ids.size)
        if residual_metric:
            integ2.runUntilResSmallerThan = RUN_UNTIL
        integ2.integrate(m2, sc2.h, cs, cache, frame)

    e2e_pcg = residual_metric and m2.energy_type == MLX_ENERGY_NEOHOOKEAN and args.layer_pcg > 0
    if e2e_pcg:
        integ2.solver(m2).layer_pcg(args.layer_pcg, args.layer_pcg_every)
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, {2: 20, 3: 3, 5: 5}.get(CONFIG, 10)))
    for frame in range(1, 3 if e2e_steps else 1):  # warm-up: solver creation and layer caches
        e2e_step(frame)
    barrier()
    contact_bytes.clear()
    e2e_s = 1e-30
    for frame in range(3, 3 + e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step(frame)
        e2e_s += time.perf_counter() - t0
    barrier()
    e2e_s = max_over_ranks(e2e_s, dist)
    N, T = m2.N, m2.T
    K = float(np.mean(contact_bytes)) if contact_bytes else 0.0
    # layer solve: xi and v in (2 x 3N; oldp too when the material is
    # damped; lambdai is passed as zeros, NULL), pinned x, contacts (normal,
    # point, compliance, id: 7 x 8 + 4 bytes each); detection: positions in
    # (3N), contact lists back; the residual array back when monitored
    damped = m2.energy_type != MLX_ENERGY_NEOHOOKEAN and bool(np.any(np.asarray(m2.alpha1) != 0))
    h2d = (8 * ((3 if damped else 2) * 3 * N + m2.pinnedDOFs.size) + 60 * K
           + (8 * 3 * N if sc2.contact_finders else 0))
    d2h = 8 * 3 * N + (60 * K if sc2.contact_finders else 0)

    # ---- buildLayers for strain-rate layers (the reference's default
    # ordering): on the device against the native host helpers ----
    layer_builder = None
    if not args.no_e2e and CONFIG not in (3,):
        from multilayersolver2024_b200.xpbd_layer3d import (build_layers_device, find_boundary_vertices as fbv,
                                                            strain_rate_norms, union_find_layers)
        solver_b = Solver(m, precision=MLX_FP32, device=local, material="lame")
        rng = np.random.default_rng(0)
        oldp5 = m.p + rng.normal(0, 1e-3, m.p.size)
        p5 = oldp5 + rng.normal(0, 1e-3, m.p.size)
        forced5 = np.zeros(m.T, np.uint8)
        forced5[m.pinnedTets - 1] = 1
        pct = [0.0, 25.0, 50.0]
        reps = 5 if m.T < 1_000_000 else 2
        build_layers_device(solver_b, m, p5, oldp5, sc.h, pct, forced5)  # warm-up (DmInv copy)
        t0 = time.perf_counter()
        for _ in range(reps):
            dev = build_layers_device(solver_b, m, p5, oldp5, sc.h, pct, forced5)
        dev_ms = (time.perf_counter() - t0) * 1000.0 / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            order5 = np.argsort(strain_rate_norms(m, p5, oldp5, sc.h), kind="stable").astype(np.int32) + 1
            sets5, nr5 = union_find_layers(m, order5, pct, forced5)
            host = fbv(m, sets5, nr5)
        host_ms = (time.perf_counter() - t0) * 1000.0 / reps
        solver_b.close()
        layer_builder = {"layers_pct": pct, "device_ms": dev_ms, "host_ms": host_ms,
                         "identical": bool(np.array_equal(dev.rigidBodySetsPerLayer, host.rigidBodySetsPerLayer)
                                           and np.array_equal(dev.vertexRigidBody, host.vertexRigidBody)),
                         "api": "mlx_build_layers (host buffers in and out) vs mlx_strain_rate_norms + stable "
                                "argsort + mlx_union_find_layers + mlx_find_boundary_vertices"}

    line = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        if solver_launch_path.startswith("cluster"):
            sweep_kernel = "k_layer_cluster (whole projectGS loop of a layer)"
        elif "CTAs each owning whole components" in solver_launch_path:
            sweep_kernel = ("k_layer_groups (whole projectGS loop of each body-free layer; algorithmic bytes without "
                            "vertex records, which stay in shared memory) + k_project_color (layers with bodies)")
        else:
            sweep_kernel = "k_project_color (all colours of a sweep)"
        achieved = (sweep_bytes / (sweep_ms / 1000.0)) / 1e9 if sweep_ms > 0 else None
        groups_only = sweep_kernel.startswith("k_layer_groups") and all(n == 0 for n in sc.layers)
        if groups_only and profiled_dram_bytes_per_tet("k_layer_groups") is not None:
            # one launch = the whole projectGS loop of the layer: T x iterations projections
            traffic = profiled_dram_bytes_per_tet("k_layer_groups") * m.T * sum(sc.iterations)
        elif profiled_dram_bytes_per_tet() is not None:
            traffic = (profiled_dram_bytes_per_tet() * sweep_bytes / solver_bytes_per_tet(m, MLX_FP32)
                       / max(sweep_launches, 1))
        else:
            traffic = None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            if residual_metric:
                # a bounded sample: the first step with the monitor on, capped
                # at cpu_iters iterations, scaled to the plain GPU solve's
                # iterations per step (same algorithm, same residual rule)
                n, dt, it = cpu_port(1, threads, state0, residual=True, cap=args.cpu_iters)
                per_it = dt / max(it[0], 1)
                gpu_it = float(np.mean((to_res["plain"] or fleg_of(to_res))["iterations_per_step"]))
                cpu = {"value": 1.0 / (per_it * gpu_it), "unit": "steps/s", "cores": threads, "kind": "port",
                       "sample": f"{it[0]} projectGS iterations of one step with the residual monitor on ({dt:.1f} s, "
                                 f"FP64 oracle restatement, OpenMP over the tets of a colour), scaled to "
                                 f"{gpu_it:.0f} iterations per step (the plain GPU solve's mean to residual 1e-4)"}
            else:
                n, dt, _ = cpu_port(args.cpu_steps + 1, threads, state0)
                cpu = {"value": n / dt, "unit": "steps/s", "cores": threads, "kind": "port",
                       "sample": f"{n} steps of the full workload ({dt:.1f} s, FP64 oracle restatement, OpenMP "
                                 "over the tets of a colour" + (", from the same landed state, oracle contact "
                                                                 "finders every step)" if advance else ")")}
        if residual_metric:
            fleg = fleg_of(to_res)
            value = fleg["steps_per_s"] * world
            ms_per_step = 1000.0 * world / value
            solver_desc = ("learned warm start (coarse-cluster corrections, BF16 perceptron on tcgen05)"
                           + (f" with the PCG in the layer solve (Newton-PCG corrections of the fine layer, "
                              f"{args.layer_pcg} PCG iterations after every {args.layer_pcg_every} Gauss-Seidel "
                              f"iterations)" if to_res["value_leg"] == "learned_pcg" else "")
                           + " to residual 1e-4")
            iters_le = fleg["iterations_per_step"]
            per_iter = fixed_launches / max(sum(sc.iterations), 1)
            launches = int(sum(it * (per_iter + 2) for it in iters_le))
            launch_note = ("estimate: iterations of the timed steps x (launches per fixed-count iteration + the "
                           "monitor's 2)")
            if to_res["value_leg"] == "learned_pcg":
                # each Newton-PCG correction: 7 launches + 2 per PCG iteration, one before the fine layer
                # and one after every `every` of its iterations (the fine layer holds most iterations)
                per_corr = 7 + 2 * args.layer_pcg
                launches += int(sum((1 + max(it - 1, 0) // max(args.layer_pcg_every, 1)) * per_corr
                                    for it in iters_le))
                launch_note += " + Newton-PCG corrections x (7 + 2 x PCG iterations)"
        else:
            value, ms_per_step = fixed_value, fixed_max_ms / args.steps
            solver_desc = "plain multi-layer (no warm-start), fixed iteration counts"
            launches = int(fixed_launches * args.steps)
            launch_note = "launches of the captured step graph x timed steps"
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": solver_desc,
                       "fixed_iterations_per_step": int(sum(sc.iterations)),
                       "precision": "FP32 bulk projection; FP64 rigid bodies, polar decomposition and residual norm; "
                                    "BF16 perceptron with FP32 accumulation",
                       "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{world}",
                       "graph": "one CUDA graph per step", "autotune": tuned,
                       "untimed_advance_steps": advance,
                       "contacts_first_last_timed_step": [contacts_at_start, contacts_at_end]},
            "to_residual": to_res,
            "parity": parity if residual_metric else None,
            "fixed_iterations": {"steps_per_s": fixed_value, "ms_per_step": fixed_max_ms / args.steps,
                                 "iterations_per_step": int(sum(sc.iterations)),
                                 "contacts": ("coloured with the elastic constraints" if sc.settings.get("contactColoring")
                                              else ("after the colours (reference order)" if sc.contact_finders
                                                    else None)),
                                 "reference_contact_order": reference_order},
            "roofline": {"bound": "hbm", "kernel": sweep_kernel, "measured_on": "fixed_iterations leg",
                         "launch_path": solver_launch_path,
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic,
                         "traffic_note": "DRAM bytes per launch from one ncu capture (cold cache) scaled by the "
                                         "tets per launch; achieved uses algorithmic bytes",
                         "peak_kind": peak_kind, "bytes_per_tet": solver_bytes_per_tet(m, MLX_FP32),
                         "sweep_ms_per_step": sweep_ms / args.steps,
                         "colour_launches_per_step": sweep_launches / args.steps,
                         "avg_launch_us": 1000.0 * sweep_ms / max(sweep_launches, 1)},
            "cpu_baseline": cpu,
            "e2e": None if not e2e_steps else {"value": e2e_steps * world / e2e_s, "unit": "steps/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "XpbdLayer3D.integrate -> mlx_layer_solve"
                    + (" (+ mlx_find_contacts on the step-start positions)" if sc.contact_finders else "")
                    + ((", to residual 1e-4 with the PCG in the layer solve (mlx_layer_pcg; the learned warm "
                        "start is an option of the device-resident stepper only)")
                       if e2e_pcg else (", plain solve to residual 1e-4" if residual_metric else ""))
                    + ("; from the second step on each call replays the recorded loop with the stop rules on "
                       "the device" if residual_metric and not sc.contact_finders else
                       ("; stop rules on the host (host contact list)" if residual_metric else ""))},
            "layer_builder": layer_builder,
            "gpu_launches": launches, "gpu_launches_note": launch_note,
            "clocks": clocks.summary(),
            "state_finite": finite,
        }
        if CONFIG in (1, 3):
            # independent scenes in the merged mesh
            line["scene_steps_per_s"] = value * (REPLICAS if CONFIG == 1 else 256)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def fleg_of(to_res):
    """The value leg's record of a to_residual block."""
    return to_res[to_res["value_leg"]] if to_res["value_leg"] != "learned" else to_res["learned_warm_start"]


def solver_bytes_per_tet(mesh, precision):
    """Algorithmic bytes of one tet projection in the device layout: vertex
    ids (16), DmInv (9 r), volume (r, StVK only), material (2 r for the
    Neo-Hookean compliances, which include the volume, 3 r for StVK from Lame
    parameters), lambda read + write (2 x 2 r or 2 x 6 r), four vertex records
    read and written (8 x 4 r); r = 4 (FP32) or 8 (FP64)."""
    from multilayersolver2024_b200 import MLX_ENERGY_NEOHOOKEAN
    r = 4 if precision == 0 else 8
    nh = mesh.energy_type == MLX_ENERGY_NEOHOOKEAN
    return 16 + 9 * r + (0 if nh else r) + (2 if nh else 3) * r + 2 * (2 if nh else 6) * r + 8 * 4 * r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-API leg (profiling runs)")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4, 5], default=5,
                    help="1: copies of the single-layer cantilever (--replicas); 2: the plain multi-layer block; "
                    "3: the 256-scene batch; 4: the contact-heavy drop; 5: the learned warm-start workload "
                    "(64x32x32, 3 layers; default)")
    ap.add_argument("--replicas", type=int, default=4096, help="config 1: copies of the cantilever in the mesh")
    ap.add_argument("--autotune", action="store_true", help="run the per-colour tile autotuner before timing "
                    "(on by default for config 3)")
    ap.add_argument("--no-autotune", action="store_true", help="never run the autotuner (profiling runs)")
    ap.add_argument("--no-residual-leg", action="store_true", help="skip the iterations-to-residual-1e-4 leg")
    ap.add_argument("--cpu-iters", type=int, default=150,
                    help="projectGS iterations of the CPU-baseline sample on the residual workloads")
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="--impl reference on the residual workloads: whole steps to residual until this many "
                    "seconds have passed (at least one)")
    ap.add_argument("--fallback-residual", type=float, default=1e-3,
                    help="learned warm start: clusters with a predicted rigid-fit residual above this (m) keep the "
                    "plain start")
    ap.add_argument("--layer-pcg", type=int, default=50,
                    help="PCG iterations of each Newton-PCG correction of the fine layer (Neo-Hookean residual "
                    "workloads; 0: none)")
    ap.add_argument("--layer-pcg-every", type=int, default=35,
                    help="Gauss-Seidel iterations between the Newton-PCG corrections")
    ap.add_argument("--host-monitor", action="store_true",
                    help="residual legs without the step graph: the same kernels with the stop rules on the host "
                    "(ncu cannot profile kernels of graphs with conditional nodes)")
    ap.add_argument("--legs", default="",
                    help="comma-separated residual legs to run (profiling; the value leg always runs)")
    ap.add_argument("--train-in-bench", action="store_true",
                    help="config 5: train the network on recorded steps here instead of loading the shipped one")
    ap.add_argument("--advance", type=int, default=None,
                    help="untimed steps before the warm-up (default: 150 for config 4, which lands the boxes; "
                    "0 for the others)")
    ap.add_argument("--learned-train-steps", type=int, default=24,
                    help="recorded steps (another seed) the warm-start network is trained on when it is trained "
                    "in the bench")
    ap.add_argument("--residual-cap", type=int, default=15000,
                    help="hangingStop of the residual leg (bounds the iterations of a step)")
    args = ap.parse_args()
    global CONFIG, WORKLOAD, REPLICAS
    CONFIG = args.config
    REPLICAS = max(1, args.replicas)
    WORKLOAD = config1_workload(REPLICAS) if CONFIG == 1 else WORKLOADS[CONFIG]
    if CONFIG == 3:
        args.autotune = True
        args.cpu_steps = min(args.cpu_steps, 1)
    if args.no_autotune:
        args.autotune = False
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
