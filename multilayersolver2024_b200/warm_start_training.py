"""Training set and training of the learned warm start (config-5 scene class).

The warm start's perceptron is trained on solver steps the library itself
generates: batches of config-5-class Neo-Hookean blocks, each with its own
seed (materials and surface impulse; scenes.config5_batch), merged side by
side into one mesh and stepped together by the resident stepper with the
residual monitor on the device (runUntilResSmallerThan = 1e-4 over the merged
mesh, so every block ends below 1e-4).  Every step records, for each rigid
cluster of the first layer, its 44 features and 8 targets (the corrections
that put it on the best-fit rigid motion of the converged step, its mean
boundary multiplier, the log10 RMS residual of that fit).  The default set is
20,000 block-steps.  Training uses the library's tensor-core forward and
backward kernels and Adam (mlx_mlp_train); the result is saved as an .npz
(parameters, normalisations, provenance) that `load_warm_start` reads.

    python -m multilayersolver2024_b200.warm_start_training --out net.npz
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import _lib, scenes
from .learned import Mlp, fit_warm_start
from .xpbd_layer3d import ResidentSim, Solver, XpbdLayer3D, find_boundary_vertices

DEFAULT_NET = Path(__file__).resolve().parent / "data" / "warm_start_config5.npz"


def residual_stepper(scene, precision=_lib.MLX_FP32, run_until=1e-4, hanging_stop=15000, device=0,
                     p0=None, v0=None):
    """The resident stepper of `scene` with the residual monitor on (stop at
    `run_until`, at most `hanging_stop` iterations per step), starting from
    the scene's t = 0 state with its impulse, or from (p0, v0)."""
    integ = XpbdLayer3D()
    integ.Gravity = scene.gravity
    integ.setLayers(scene.layers)
    integ.iterations = list(scene.iterations)
    integ.customRigidSets = scene.custom_sets
    integ.precision = precision
    integ.contactResistance = scene.settings.get("contactResistance", integ.contactResistance)
    integ.computeResiduals = True
    integ.runUntilResSmallerThan = run_until
    integ.hangingStop = hanging_stop
    sets = scene.custom_sets
    ls = find_boundary_vertices(scene.mesh, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    solver = Solver(scene.mesh, precision=precision, device=device, material="lame")
    if p0 is None:
        sim = ResidentSim(solver, integ, ls, scene.h, p0=scene.mesh.p, v0=np.zeros_like(scene.mesh.p))
        if scene.impulse is not None:
            sim.add_velocity(scene.impulse[0], scene.impulse[1])
    else:
        sim = ResidentSim(solver, integ, ls, scene.h, p0=p0, v0=v0)
    if scene.contact_finders:
        sim.set_obstacles(scene.contact_finders, restitution=1e-2)
    return solver, sim


def generate(total_steps=20000, scenes_per_batch=16, steps_per_scene=250, dims=(32, 16, 16), seed=100,
             device=0, log=print):
    """Features (rows x 44), targets (rows x 8) and the projectGS iterations
    of every merged step, from total_steps block-steps."""
    feats, tgts, iters = [], [], []
    batches = -(-total_steps // (scenes_per_batch * steps_per_scene))
    for b in range(batches):
        sc = scenes.config5_batch(seed=seed + b, n_scenes=scenes_per_batch, nx=dims[0], ny=dims[1], nz=dims[2])
        solver, sim = residual_stepper(sc, device=device)
        sim.warm_start(record=True, mode=0)
        t0 = time.perf_counter()
        for _ in range(steps_per_scene):
            sim.step(1, graph=True)
            f, t = sim.warm_start_records()
            feats.append(f)
            tgts.append(t)
            iters.append(int(sim.monitor()[1]))
        solver.close()
        log(f"batch {b + 1}/{batches}: {scenes_per_batch} blocks x {steps_per_scene} steps, "
            f"{time.perf_counter() - t0:.1f} s, iterations {iters[-steps_per_scene]}..{iters[-1]}")
    return np.concatenate(feats), np.concatenate(tgts), np.asarray(iters)


def save_warm_start(path, net, fn, on, meta):
    np.savez_compressed(path, params=net.get_params(), feature_mean=fn[0], feature_std=fn[1], output_mean=on[0],
                        output_std=on[1], hidden=net.n_hidden, hidden_layers=net.n_hidden_layers,
                        meta=json.dumps(meta))


def load_warm_start(path=DEFAULT_NET, max_batch=4096):
    """(network, feature normalisation, output normalisation, provenance) of
    a saved warm start."""
    d = np.load(path)
    net = Mlp(44, 8, n_hidden=int(d["hidden"]), n_hidden_layers=int(d["hidden_layers"]), max_batch=max_batch)
    net.set_params(d["params"])
    return (net, (d["feature_mean"], d["feature_std"]), (d["output_mean"], d["output_std"]),
            json.loads(str(d["meta"])))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(DEFAULT_NET))
    ap.add_argument("--steps", type=int, default=20000, help="block-steps of the training set")
    ap.add_argument("--scenes-per-batch", type=int, default=16)
    ap.add_argument("--steps-per-scene", type=int, default=250)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--seed", type=int, default=100)
    a = ap.parse_args()
    t0 = time.perf_counter()
    f, t, iters = generate(a.steps, a.scenes_per_batch, a.steps_per_scene, seed=a.seed)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    net, fn, on, losses = fit_warm_start(f, t, epochs=a.epochs, lr=1e-3, batch=1024, seed=a.seed)
    train_s = time.perf_counter() - t0
    meta = {"block_steps": a.steps, "rows": int(f.shape[0]), "scenes_per_batch": a.scenes_per_batch,
            "steps_per_scene": a.steps_per_scene, "block_dims": [32, 16, 16], "seed": a.seed,
            "epochs": a.epochs, "loss_first_last": [float(losses[0]), float(losses[-1])],
            "generate_s": gen_s, "train_s": train_s, "mean_iterations": float(iters.mean())}
    Path(a.out).parent.mkdir(parents=True, exist_ok=True)
    save_warm_start(a.out, net, fn, on, meta)
    print(json.dumps(meta))
    net.close()


if __name__ == "__main__":
    main()
