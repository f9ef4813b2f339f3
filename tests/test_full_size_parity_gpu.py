"""FP32 bulk projection on the GPU against the FP64 oracle, per configuration
at full size (max position difference / bounding-box diagonal, worst step):

  config 2 (98,304 NH tets, 2 layers), 3 steps from t = 0:        <= 1e-4
  config 2 to residual 1e-4 (device stop rules vs the oracle's
    host stop rules), 1 step from t = 0:                           <= 1e-4
    (and projectGS iterations within 10 % of the oracle's)
  config 3 (all 256 scenes, 3.35 M tets, 2 layers), 2 steps:      <= 1e-4
  config 4 (32 StVK boxes, 331,776 tets, 3 layers, plane + 4
    spheres, contacts detected every step and coloured with the
    elastic constraints; the oracle in the same order), 3 steps
    from the landed state after 150 steps:                        <= 1e-4
  config 4 in the reference's contact order, the same steps:      <= 1e-4
  config 5 (393,216 NH tets, 3 layers), 3 steps from t = 0:        <= 1e-4

The oracle runs with every host thread; each case starts both sides from the
same state.  Printed errors are the figures quoted in the design notes.
"""
import os

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, ResidentSim, Solver, StepCache, XpbdLayer3D,
                                                    find_boundary_vertices)

pytestmark = pytest.mark.gpu


def _integ(scene, precision, residual=False):
    integ = XpbdLayer3D()
    integ.Gravity = scene.gravity
    integ.setLayers(scene.layers)
    integ.iterations = list(scene.iterations)
    integ.customRigidSets = scene.custom_sets
    integ.precision = precision
    integ.contactResistance = scene.settings.get("contactResistance", integ.contactResistance)
    integ.contactColoring = bool(scene.settings.get("contactColoring", False))
    if residual:
        integ.computeResiduals = True
        integ.runUntilResSmallerThan = 1e-4
        integ.hangingStop = 15000
    return integ


def _gpu(scene, steps, state=None, residual=False, advance=0):
    m = scene.mesh
    sets = scene.custom_sets
    ls = find_boundary_vertices(m, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    s = Solver(m, precision=_lib.MLX_FP32, material="lame")
    if state is None:
        sim = ResidentSim(s, _integ(scene, _lib.MLX_FP32, residual), ls, scene.h, p0=m.p, v0=np.zeros_like(m.p))
        if scene.impulse is not None:
            sim.add_velocity(scene.impulse[0], scene.impulse[1])
    else:
        sim = ResidentSim(s, _integ(scene, _lib.MLX_FP32, residual), ls, scene.h, p0=state[0], v0=state[1])
    if scene.contact_finders:
        sim.set_obstacles(scene.contact_finders, restitution=1e-2)
    if advance:
        sim.step(advance, graph=True)
        start = tuple(a.copy() for a in sim.state()[:2])
        s.close()
        return _gpu(scene, steps, start, residual), start
    traj = []
    for _ in range(steps):
        sim.step(1, graph=True)
        traj.append(sim.state()[0])
    its = sim.monitor()[1] if residual else None
    s.close()
    return traj, its


def _oracle(scene, steps, oracle, state=None, residual=False):
    oracle.load().orc_set_threads(os.cpu_count() or 1)
    m = scene.mesh
    m.p = m.p.copy()
    m.v = np.zeros_like(m.p)
    if state is None:
        if scene.impulse is not None:
            m.v[scene.impulse[0] - 1] += scene.impulse[1]
    else:
        m.p, m.v = (a.copy() for a in state)
    integ = _integ(scene, _lib.MLX_FP64, residual)
    cache = StepCache()
    traj, its = [], None
    for frame in range(1, steps + 1):
        cs = oracle.find_contacts(scene.contact_finders, m.p) if scene.contact_finders else ContactSet()
        its = oracle.integrate(integ, m, scene.h, cs, cache, frame)[1]
        traj.append(m.p.copy())
    return traj, its


def _err(scene, got, ref, name):
    d = scene.mesh.bbox_diagonal()
    e = max(np.abs(a - b).max() / d for a, b in zip(got, ref))
    print(f"{name}: FP32 GPU vs FP64 oracle, max position error / bbox diagonal {e:.3e}")
    return e


def test_config2_full_size(gpu, oracle):
    got, _ = _gpu(scenes.config2(), 3)
    ref, _ = _oracle(scenes.config2(), 3, oracle)
    assert _err(scenes.config2(), got, ref, "config2, 3 steps") <= 1e-4


def test_config2_to_residual(gpu, oracle):
    got, its_gpu = _gpu(scenes.config2(), 1, residual=True)
    ref, its_ref = _oracle(scenes.config2(), 1, oracle, residual=True)
    print(f"config2 to residual 1e-4: projectGS iterations GPU {its_gpu}, oracle {its_ref}")
    # FP32 rounding moves the monitored residual, so the stop rules fire a few
    # per cent of the iterations apart (measured 1735 against 1665)
    assert abs(its_gpu - its_ref) <= 0.1 * its_ref
    assert _err(scenes.config2(), got, ref, "config2 to residual 1e-4, 1 step") <= 1e-4


def test_config3_full_size(gpu, oracle):
    sc = scenes.config3()
    got, _ = _gpu(sc, 2)
    ref, _ = _oracle(scenes.config3(), 2, oracle)
    assert _err(sc, got, ref, "config3 (256 scenes), 2 steps") <= 1e-4
    # every scene on its own scale: the worst scene's error over its own diagonal
    offs = sc.mesh.part_vertex_offsets
    worst = 0.0
    for k, part in enumerate(sc.settings["parts"]):
        sl = slice(3 * offs[k], 3 * offs[k + 1])
        worst = max(worst, max(np.abs(a[sl] - b[sl]).max() for a, b in zip(got, ref)) / part.bbox_diagonal())
    print(f"config3 worst scene error / its own diagonal {worst:.3e}")
    assert worst <= 1e-4


@pytest.mark.parametrize("coloring", [True, False])
def test_config4_full_size_landed(gpu, oracle, coloring):
    (got, _), start = _gpu(scenes.config4(contact_coloring=coloring), 3, advance=150)
    ref, _ = _oracle(scenes.config4(contact_coloring=coloring), 3, oracle, state=start)
    name = "config4 landed, 3 steps, contacts " + ("coloured" if coloring else "after the colours")
    assert _err(scenes.config4(), got, ref, name) <= 1e-4


def test_config5_full_size(gpu, oracle):
    got, _ = _gpu(scenes.config5(), 3)
    ref, _ = _oracle(scenes.config5(), 3, oracle)
    assert _err(scenes.config5(), got, ref, "config5, 3 steps") <= 1e-4
