#!/usr/bin/env python
"""Throughput of the multi-layer XPBD step on B200 (one JSON line on rank 0).

Workload: the plain multi-layer Neo-Hookean block -- 64x16x16 cubes of 0.1 m,
6 tets per cube (18,785 vertices, 98,304 tets), per-tet E log-uniform in
[1e4, 1e7] Pa, nu uniform in [0.25, 0.45] (seeded), a coarse layer of fixed
8^3-cube rigid clusters (5 iterations) then the fine layer (10 iterations),
dt = 1/60 s, base pinned, seeded surface impulse at t = 0.  Synthetic data.

A step is one xpbdLayer3D.integrate step.  `value` is steps/s of the
device-resident stepper (state in HBM, one CUDA graph per step) with L2
flushed between timed steps; `e2e` is steps/s through the public host API
(XpbdLayer3D.integrate -> mlx_layer_solve with host buffers, every step copies
its inputs host->device and its positions back).  Multi-GPU runs are
independent replicas (weak scaling): the step does not shard.

Other workloads (`--config`): 1 = `--replicas` copies of the 8x2x2
single-layer cantilever merged into one mesh, 3 = the 256-scene batch, 4 = the
contact-heavy drop, 5 = the learned warm start's block.

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
        "detected on the device every step, 3 layers (4^3-cube clusters 1 it, 2^3-cube clusters 4 it, fine 10 it), "
        "contact resistance 0.9, dt=1/120; timed after the boxes have landed"),
}
WORKLOAD = WORKLOADS[2]
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


CONFIG = 2


def make_scene():
    from multilayersolver2024_b200 import scenes
    if CONFIG == 1:
        return scenes.config1_replicated(REPLICAS)
    return {2: scenes.config2, 3: scenes.config3, 4: scenes.config4, 5: scenes.config5}[CONFIG]()


def make_training_scene():
    """Another seed of the workload's scene class (other materials and
    impulse): the warm start's network is trained on its solver records."""
    from multilayersolver2024_b200 import scenes
    return {2: lambda: scenes.config2(seed=3), 5: lambda: scenes.config5(seed=6)}[CONFIG]()


def start_velocity(scene, m):
    """Velocity at t = 0: the scene's seeded impulse, if it has one."""
    if scene.impulse is not None:
        m.v[scene.impulse[0] - 1] += scene.impulse[1]


def make_integrator(scene, precision):
    from multilayersolver2024_b200 import XpbdLayer3D
    integ = XpbdLayer3D()
    integ.Gravity = scene.gravity
    integ.setLayers(scene.layers)
    integ.iterations = list(scene.iterations)
    integ.customRigidSets = scene.custom_sets
    integ.precision = precision
    integ.contactResistance = scene.settings.get("contactResistance", integ.contactResistance)
    return integ


def cpu_port_steps_per_s(nsteps, threads, state=None):
    """The oracle (FP64 C++ restatement of the reference path, all given host
    threads) on the same workload: steps/s over `nsteps` steps, from the
    scene's t = 0 state or from `state` = (positions, velocities)."""
    from oracle import oracle as O
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet, StepCache
    O.load().orc_set_threads(threads)
    sc = make_scene()
    integ = make_integrator(sc, 1)
    m = sc.mesh
    start_velocity(sc, m)
    if state is not None:
        m.p, m.v = (a.copy() for a in state)
    cache = StepCache()

    def contacts():
        # simulate3D's loop: the finders on the step-start positions
        return O.find_contacts(sc.contact_finders, m.p) if sc.contact_finders else ContactSet()

    O.integrate(integ, m, sc.h, contacts(), cache, 1)  # warm-up (frame 1)
    t0 = time.perf_counter()
    for frame in range(2, nsteps + 2):
        O.integrate(integ, m, sc.h, contacts(), cache, frame)
    dt = time.perf_counter() - t0
    return nsteps / dt, dt


# untimed steps of the device stepper that bring a scene into its timed phase
# (config 4: the boxes have landed on the obstacles after 150 steps, 1.25 s)
ADVANCE = {4: 150}
_PHASE = {}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    warm = max(args.warmup, 0)
    # warm-up steps are part of the same run of the port
    total = warm + args.steps
    sps, dt = cpu_port_steps_per_s(total, threads)
    value = sps
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "solver": "plain multi-layer, CPU port"},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": f"{total} consecutive steps of the full workload (oracle restatement; "
                                       "MATLAB, the reference's runtime, is not installed)"
                                       + (", from t = 0 with the oracle contact finders every step" if CONFIG == 4
                                          else "")},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local):
    import torch
    from multilayersolver2024_b200 import MLX_ENERGY_NEOHOOKEAN, MLX_FP32, StepCache, XpbdLayer3D, load
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
    integ = make_integrator(sc, MLX_FP32)
    sets = sc.custom_sets
    ls = find_boundary_vertices(m, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    solver = Solver(m, precision=MLX_FP32, device=local, material="lame")
    sim = ResidentSim(solver, integ, ls, sc.h, p0=m.p, v0=np.zeros_like(m.p))
    if sc.impulse is not None:
        sim.add_velocity(sc.impulse[0], sc.impulse[1])
    if sc.contact_finders:
        sim.set_obstacles(sc.contact_finders, restitution=1e-2)
    advance = ADVANCE.get(CONFIG, 0) if args.advance is None else args.advance
    if advance:
        sim.step(advance, graph=True)
        torch.cuda.synchronize()
        _PHASE["state"] = tuple(a.copy() for a in sim.state()[:2])
    tuned = None
    if args.autotune:
        before, after = sim.autotune(reps=5)
        tuned = {"step_ms_default_tiles": before, "step_ms_tuned_tiles": after}
    sim.sweep_timing(True)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    for _ in range(args.warmup):
        sim.step(1, graph=True)
    torch.cuda.synchronize()
    sim.sweep_stats(reset=True)
    contacts_at_start = sim.contact_count() if sc.contact_finders else None

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        total_ms += sim.step(1, graph=True, timed=True)
    torch.cuda.synchronize()
    barrier()
    clocks.stop()
    sweep_ms, sweep_bytes, sweep_launches = sim.sweep_stats(reset=True)
    contacts_at_end = sim.contact_count() if sc.contact_finders else None
    max_ms = max_over_ranks(total_ms, dist)
    value = args.steps * world / (max_ms / 1000.0)
    launches_per_step = sim.launches_per_step
    p_gpu, _ = sim.state()
    finite = bool(np.all(np.isfinite(p_gpu)))

    # ---- e2e: public host API, host buffers, every step copies in and out ----
    sc2 = make_scene()
    m2 = sc2.mesh
    integ2 = make_integrator(sc2, MLX_FP32)
    cache = StepCache()
    start_velocity(sc2, m2)
    if advance:
        m2.p, m2.v = (a.copy() for a in _PHASE["state"])
    from multilayersolver2024_b200.contacts import find_contacts
    contact_bytes = []

    def e2e_step(frame):
        # simulate3D's step: the finders on the step-start positions (on the
        # device, mlx_find_contacts), then integrate (mlx_layer_solve)
        cs = find_contacts(integ2.solver(m2), sc2.contact_finders, m2.p) if sc2.contact_finders else ContactSet()
        contact_bytes.append(cs.vertex_ids.size)
        integ2.integrate(m2, sc2.h, cs, cache, frame)

    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, {2: 20, 3: 3}.get(CONFIG, 10)))
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
    # (3N), contact lists back
    damped = m2.energy_type != MLX_ENERGY_NEOHOOKEAN and bool(np.any(np.asarray(m2.alpha1) != 0))
    h2d = (8 * ((3 if damped else 2) * 3 * N + m2.pinnedDOFs.size) + 60 * K
           + (8 * 3 * N if sc2.contact_finders else 0))
    d2h = 8 * 3 * N + (60 * K if sc2.contact_finders else 0)

    # ---- iterations to residual 1e-4: the same workload with the residual
    # monitor and stop rules on the device (conditional graph nodes) ----
    to_res = None
    if not args.no_residual_leg:
        from multilayersolver2024_b200.learned import collect_warm_start_data, fit_warm_start

        def residual_sim(scene):
            integ3 = make_integrator(scene, MLX_FP32)
            integ3.computeResiduals = True
            integ3.runUntilResSmallerThan = 1e-4
            integ3.hangingStop = args.residual_cap
            sets3 = scene.custom_sets
            ls3 = find_boundary_vertices(scene.mesh, sets3,
                                         [int(sets3[:, c].max(initial=0)) for c in range(sets3.shape[1])])
            solver3 = Solver(scene.mesh, precision=MLX_FP32, device=local, material="lame")
            if advance:
                p0, v0 = _PHASE["state"]
            else:
                p0, v0 = scene.mesh.p, np.zeros_like(scene.mesh.p)
            sim3 = ResidentSim(solver3, integ3, ls3, scene.h, p0=p0, v0=v0)
            if scene.impulse is not None and not advance:
                sim3.add_velocity(scene.impulse[0], scene.impulse[1])
            if scene.contact_finders:
                sim3.set_obstacles(scene.contact_finders, restitution=1e-2)
            return solver3, sim3

        def run_leg(sim3, n):
            iters, ms_steps, finals = [], [], []
            for _ in range(n):
                ms_steps.append(sim3.step(1, graph=True, timed=True))
                ra, it_total, _, status = sim3.monitor()
                iters.append(int(it_total))
                finals.append(float(ra[-1]))
            return {"iterations_per_step": iters, "ms_per_step": ms_steps,
                    "steps_per_s": len(ms_steps) / (sum(ms_steps) / 1000.0), "final_residual": finals,
                    "reached": [bool(abs(r) <= 1e-4) for r in finals]}

        solver_p, sim_p = residual_sim(make_scene())
        plain_leg = run_leg(sim_p, args.residual_steps)
        p_plain = sim_p.state()[0]
        solver_p.close()
        learned_leg = None
        if CONFIG in (2, 5) and args.learned_train_steps > 0:
            # the warm start's network is trained on another seed of the same
            # scene class, then steps the benchmark scene
            solver_t, sim_t = residual_sim(make_training_scene())
            ftr, ttr, _ = collect_warm_start_data(sim_t, args.learned_train_steps)
            solver_t.close()
            t0 = time.perf_counter()
            net, fn, on, losses = fit_warm_start(ftr, ttr, epochs=300, lr=2e-3, batch=128)
            train_s = time.perf_counter() - t0
            solver_w, sim_w = residual_sim(make_scene())
            sim_w.warm_start(record=False, mode=1, net=net, feature_norm=fn, output_norm=on)
            learned_leg = run_leg(sim_w, args.residual_steps)
            learned_leg.update({
                "training": {"samples": int(ftr.shape[0]), "steps_recorded": args.learned_train_steps,
                             "scene": f"config{CONFIG} seed {3 if CONFIG == 2 else 6}", "epochs": 300,
                             "seconds": train_s,
                             "loss_first_last": [float(losses[0]), float(losses[-1])]},
                "max_position_deviation_from_plain": float(np.abs(sim_w.state()[0] - p_plain).max()
                                                           / make_scene().mesh.bbox_diagonal())})
            solver_w.close()
            net.close()
        to_res = {"run_until": 1e-4, "hanging_stop": args.residual_cap, "steps": args.residual_steps,
                  **plain_leg, "learned_warm_start": learned_leg,
                  "monitor": "device (layers as conditional IF nodes, projectGS as conditional WHILE nodes)"}

    # ---- buildLayers for strain-rate layers (the reference's default
    # ordering): on the device against the native host helpers ----
    layer_builder = None
    if not args.no_e2e:
        from multilayersolver2024_b200.xpbd_layer3d import (build_layers_device, find_boundary_vertices as fbv,
                                                            strain_rate_norms, union_find_layers)
        sc5 = make_scene()
        m5 = sc5.mesh
        rng = np.random.default_rng(0)
        oldp5 = m5.p + rng.normal(0, 1e-3, m5.p.size)
        p5 = oldp5 + rng.normal(0, 1e-3, m5.p.size)
        forced5 = np.zeros(m5.T, np.uint8)
        forced5[m5.pinnedTets - 1] = 1
        pct = [0.0, 25.0, 50.0]
        reps = 5 if m5.T < 1_000_000 else 2
        build_layers_device(solver, m5, p5, oldp5, sc5.h, pct, forced5)  # warm-up (DmInv copy)
        t0 = time.perf_counter()
        for _ in range(reps):
            dev = build_layers_device(solver, m5, p5, oldp5, sc5.h, pct, forced5)
        dev_ms = (time.perf_counter() - t0) * 1000.0 / reps
        t0 = time.perf_counter()
        for _ in range(reps):
            order5 = np.argsort(strain_rate_norms(m5, p5, oldp5, sc5.h), kind="stable").astype(np.int32) + 1
            sets5, nr5 = union_find_layers(m5, order5, pct, forced5)
            host = fbv(m5, sets5, nr5)
        host_ms = (time.perf_counter() - t0) * 1000.0 / reps
        layer_builder = {"layers_pct": pct, "device_ms": dev_ms, "host_ms": host_ms,
                         "identical": bool(np.array_equal(dev.rigidBodySetsPerLayer, host.rigidBodySetsPerLayer)
                                           and np.array_equal(dev.vertexRigidBody, host.vertexRigidBody)),
                         "api": "mlx_build_layers (host buffers in and out) vs mlx_strain_rate_norms + stable "
                                "argsort + mlx_union_find_layers + mlx_find_boundary_vertices"}

    line = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        if solver.launch_path.startswith("cluster"):
            sweep_kernel = "k_layer_cluster (whole projectGS loop of a layer)"
        elif "CTAs each owning whole components" in solver.launch_path:
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
            sps, dt = cpu_port_steps_per_s(args.cpu_steps, threads, _PHASE.get("state"))
            cpu = {"value": sps, "unit": "steps/s", "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_steps} steps of the full workload after 1 warm-up step "
                             f"({dt:.1f} s, FP64 oracle restatement, OpenMP over the tets of a colour"
                             + (", from the same landed state, oracle contact finders every step)" if advance
                                else ")")}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "plain multi-layer (no warm-start)",
                       "iterations_per_step": int(sum(sc.iterations)), "precision": "FP32 bulk, FP64 rigid bodies",
                       "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{world}",
                       "graph": "one CUDA graph per step", "autotune": tuned,
                       "untimed_advance_steps": advance,
                       "contacts_first_last_timed_step": [contacts_at_start, contacts_at_end]},
            "roofline": {"bound": "hbm", "kernel": sweep_kernel,
                         "launch_path": solver.launch_path,
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
            "e2e": None if not e2e_steps else {"value": e2e_steps * world / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "api": "XpbdLayer3D.integrate -> mlx_layer_solve"
                    + (" (+ mlx_find_contacts on the step-start positions)" if sc.contact_finders else "")},
            "to_residual": to_res,
            "layer_builder": layer_builder,
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks.summary(),
            "state_finite": finite,
        }
        if CONFIG in (1, 3):
            # independent scenes in the merged mesh
            line["scene_steps_per_s"] = value * (REPLICAS if CONFIG == 1 else 256)
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.destroy_process_group()
    return 0


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
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-API leg (profiling runs)")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4, 5], default=2,
                    help="1: copies of the single-layer cantilever (--replicas); 2: the plain multi-layer block "
                    "(default); 3: the 256-scene batch; 4: the contact-heavy drop; 5: the learned warm-start "
                    "workload (64x32x32, 3 layers)")
    ap.add_argument("--replicas", type=int, default=4096, help="config 1: copies of the cantilever in the mesh")
    ap.add_argument("--autotune", action="store_true", help="run the per-colour tile autotuner before timing "
                    "(on by default for config 3)")
    ap.add_argument("--no-autotune", action="store_true", help="never run the autotuner (profiling runs)")
    ap.add_argument("--no-residual-leg", action="store_true", help="skip the iterations-to-residual-1e-4 leg")
    ap.add_argument("--residual-steps", type=int, default=4)
    ap.add_argument("--advance", type=int, default=None,
                    help="untimed steps before the warm-up (default: 150 for config 4, which lands the boxes; "
                    "0 for the others)")
    ap.add_argument("--learned-train-steps", type=int, default=16,
                    help="recorded steps (another seed) the warm-start network is trained on; 0 skips that leg")
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
