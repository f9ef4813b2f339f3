"""Whole-step parity: the device-resident stepper (integrate on the GPU) and
the host-driven integrate mirror against the oracle's integrate restatement.

Tolerances (max position difference / bounding-box diagonal):
  FP64 GPU vs FP64 oracle, 20 steps of config 1:           <= 1e-9
  FP32 GPU vs FP64 oracle, 200 steps of config 1 (full run): <= 1e-3
    (an undamped oscillating cantilever: FP32 rounding shifts its phase)
  FP32 GPU vs FP64 oracle, 3 steps of config 2 (NH, 2 layers, clusters): <= 1e-4
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, ResidentSim, Solver, StepCache, XpbdLayer3D,
                                                    find_boundary_vertices)

pytestmark = pytest.mark.gpu


def _integ(scene, precision):
    integ = XpbdLayer3D()
    integ.Gravity = scene.gravity
    integ.setLayers(scene.layers)
    integ.iterations = list(scene.iterations)
    integ.customRigidSets = scene.custom_sets
    integ.precision = precision
    return integ


def _oracle_run(scene, steps, oracle, threads=8):
    oracle.load().orc_set_threads(threads)
    m = scene.mesh
    m.p = m.p.copy()
    m.v = np.zeros_like(m.p)
    integ = _integ(scene, _lib.MLX_FP64)
    cache = StepCache()
    traj = []
    for frame in range(1, steps + 1):
        if frame == 1 and scene.impulse is not None:
            m.v[scene.impulse[0] - 1] += scene.impulse[1]
        oracle.integrate(integ, m, scene.h, ContactSet(), cache, frame)
        traj.append(m.p.copy())
    return traj


def _resident_run(scene, steps, precision, graph=True):
    m = scene.mesh
    integ = _integ(scene, precision)
    if scene.custom_sets is not None:
        sets = scene.custom_sets
        nr = [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])]
    else:
        sets = np.zeros((m.T, 1), np.int32, order="F")
        nr = [0]
    ls = find_boundary_vertices(m, sets, nr)
    s = Solver(m, precision=precision, material="blocks" if precision == _lib.MLX_FP64 else "lame")
    sim = ResidentSim(s, integ, ls, scene.h, p0=m.p, v0=np.zeros_like(m.p))
    if scene.impulse is not None:
        sim.add_velocity(scene.impulse[0], scene.impulse[1])
    traj = []
    for _ in range(steps):
        sim.step(1, graph=graph)
        traj.append(sim.state()[0])
    return traj, sim


@pytest.mark.parametrize("graph", [True, False])
def test_config1_fp64_resident_matches_oracle(gpu, oracle, graph):
    sc = scenes.config1()
    ref = _oracle_run(scenes.config1(), 20, oracle)
    got, sim = _resident_run(sc, 20, _lib.MLX_FP64, graph)
    d = sc.mesh.bbox_diagonal()
    errs = [np.abs(a - b).max() / d for a, b in zip(got, ref)]
    assert max(errs) <= 1e-9, max(errs)
    assert sim.launches_per_step > 0


def test_config1_fp32_full_run_error(gpu, oracle):
    """The config-1 parity statement: 200 steps, FP32 bulk vs the FP64 oracle."""
    sc = scenes.config1()
    ref = _oracle_run(scenes.config1(), 200, oracle)
    got, _ = _resident_run(sc, 200, _lib.MLX_FP32)
    d = sc.mesh.bbox_diagonal()
    err = max(np.abs(a - b).max() / d for a, b in zip(got, ref))
    print(f"config1 FP32 max position error / bbox diagonal over 200 steps: {err:.3e}")
    assert err <= 1e-3


def test_host_integrate_mirror_matches_oracle(gpu, oracle):
    """The drop-in path: Python integrate mirror -> mlx_layer_solve (host buffers)."""
    sc = scenes.config1()
    ref = _oracle_run(scenes.config1(), 10, oracle)
    m = sc.mesh
    integ = _integ(sc, _lib.MLX_FP64)
    cache = StepCache()
    for frame in range(1, 11):
        integ.integrate(m, sc.h, ContactSet(), cache, frame)
        assert np.abs(m.p - ref[frame - 1]).max() / m.bbox_diagonal() <= 1e-9


_CONFIG2_REF = {}


@pytest.mark.parametrize("cluster", ["1", "0"])
def test_config2_fp32_resident_matches_oracle(gpu, oracle, monkeypatch, cluster):
    """Config 2 (98,304 Neo-Hookean tets, rigid clusters) through the cluster
    kernel (16 CTAs, vertex records and multipliers in distributed shared
    memory) and through per-colour launches (the default)."""
    monkeypatch.setenv("MLXPBD_CLUSTER", cluster)
    monkeypatch.delenv("MLXPBD_CLUSTER_SIZE", raising=False)
    monkeypatch.delenv("MLXPBD_PERSISTENT", raising=False)
    if "ref" not in _CONFIG2_REF:
        _CONFIG2_REF["ref"] = _oracle_run(scenes.config2(), 3, oracle, threads=16)
    ref = _CONFIG2_REF["ref"]
    sc = scenes.config2()
    got, sim = _resident_run(sc, 3, _lib.MLX_FP32)
    path = sim.solver.launch_path
    print(path)
    assert path.startswith("cluster") == (cluster == "1")
    d = sc.mesh.bbox_diagonal()
    err = max(np.abs(a - b).max() / d for a, b in zip(got, ref))
    print(f"config2 FP32 max position error / bbox diagonal over 3 steps: {err:.3e}")
    assert err <= 1e-4
