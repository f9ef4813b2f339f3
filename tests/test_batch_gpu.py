"""Batched scenes (config 3): independent Neo-Hookean blocks merged into one
mesh as Mesh3D.mergeMesh does, stepped by one resident solver, and the
per-colour tile autotuner.

  * batch invariance, at the full config-3 size (256 scenes, 3.35 M tets) and
    on a small batch: every scene of the merged run is bit-identical to the
    same scene stepped alone (scenes share no vertex, tets of one colour are
    independent, bodies are reduced per body);
  * the autotuner changes no result bit (it only changes block sizes);
  * a small batch matches the FP64 oracle within the FP32 tolerance 1e-4 of
    each scene's bounding-box diagonal;
  * copies of the config-1 cantilever in one mesh: the copy at the origin is
    bit-identical to the cantilever stepped alone, and every copy matches the
    FP64 oracle's solo cantilever (shifted) within the FP32 tolerance 1e-3 of
    its bounding-box diagonal that the 200-step solo cantilever is held to.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import merge_meshes
from multilayersolver2024_b200.scenes import Scene

from test_step_gpu import _oracle_run, _resident_run

pytestmark = pytest.mark.gpu


def _solo_scene(batch: Scene, k: int) -> Scene:
    """Scene k of a batch as a scene of its own (same mesh, sets, impulse)."""
    m = batch.mesh
    v0, v1 = m.part_vertex_offsets[k], m.part_vertex_offsets[k + 1]
    t0, t1 = m.part_tet_offsets[k], m.part_tet_offsets[k + 1]
    part = batch.settings["parts"][k]
    solo = merge_meshes([part])
    sets = np.asfortranarray(batch.custom_sets[t0:t1].copy())
    ids = sets[:, 1]
    if (ids > 0).any():
        ids[ids > 0] -= ids[ids > 0].min() - 1
    dofs, dv = batch.impulse
    keep = (dofs > 3 * v0) & (dofs <= 3 * v1)
    return Scene(f"part{k}", solo, batch.h, batch.steps, batch.layers, batch.iterations, custom_sets=sets,
                 impulse=((dofs[keep] - 3 * v0).astype(np.int32), dv[keep]))


def _check_invariance(batch, steps, which):
    got, _ = _resident_run(batch, steps, _lib.MLX_FP32)
    m = batch.mesh
    for k in which:
        solo = _solo_scene(batch, k)
        ref, _ = _resident_run(solo, steps, _lib.MLX_FP32)
        a, b = 3 * m.part_vertex_offsets[k], 3 * m.part_vertex_offsets[k + 1]
        for s in range(steps):
            np.testing.assert_array_equal(got[s][a:b], ref[s], err_msg=f"scene {k} step {s}")


def test_small_batch_is_bitwise_invariant(gpu):
    batch = scenes.config3(seed=7, n_scenes=6, tmin=1500, tmax=6000)
    _check_invariance(batch, 3, range(6))


def test_config3_full_batch_is_bitwise_invariant(gpu):
    batch = scenes.config3()
    assert batch.mesh.T > 3_000_000
    ts = np.diff(batch.mesh.part_tet_offsets)
    # the smallest, the largest and one middle scene
    _check_invariance(batch, 2, [int(np.argmin(ts)), int(np.argmax(ts)), len(ts) // 2])


def test_small_batch_matches_oracle(gpu, oracle):
    batch = scenes.config3(seed=8, n_scenes=4, tmin=1500, tmax=4000)
    ref = _oracle_run(scenes.config3(seed=8, n_scenes=4, tmin=1500, tmax=4000), 3, oracle, threads=16)
    got, _ = _resident_run(batch, 3, _lib.MLX_FP32)
    m = batch.mesh
    for k, part in enumerate(batch.settings["parts"]):
        a, b = 3 * m.part_vertex_offsets[k], 3 * m.part_vertex_offsets[k + 1]
        d = part.bbox_diagonal()
        err = max(np.abs(g[a:b] - r[a:b]).max() / d for g, r in zip(got, ref))
        assert err <= 1e-4, f"scene {k}: {err:.3e}"


def test_autotuner_keeps_results(gpu):
    sc = scenes.config3(seed=9, n_scenes=8, tmin=2000, tmax=8000)
    ref, _ = _resident_run(sc, 3, _lib.MLX_FP32)
    sc2 = scenes.config3(seed=9, n_scenes=8, tmin=2000, tmax=8000)
    got, sim = _resident_run(sc2, 0, _lib.MLX_FP32)
    before, after = sim.autotune(reps=3)
    assert before > 0 and after > 0
    assert after <= before * 1.05
    for s in range(3):
        sim.step(1, graph=True)
        np.testing.assert_array_equal(sim.state()[0], ref[s])


def test_replicated_cantilevers(gpu, oracle):
    k, steps = 64, 10
    batch = scenes.config1_replicated(k, per_row=8)
    got, _ = _resident_run(batch, steps, _lib.MLX_FP32)
    solo, _ = _resident_run(scenes.config1_replicated(1), steps, _lib.MLX_FP32)
    n3 = solo[0].size
    for s in range(steps):
        np.testing.assert_array_equal(got[s][:n3], solo[s], err_msg=f"step {s}")
    ref = _oracle_run(scenes.config1(), steps, oracle)
    d = scenes.config1().mesh.bbox_diagonal()
    err = 0.0
    for c in range(k):
        shift = np.tile([0.0, 0.4 * (c % 8), 0.4 * (c // 8)], n3 // 3)
        err = max(err, max(np.abs(g[c * n3:(c + 1) * n3] - shift - r).max() / d for g, r in zip(got, ref)))
    assert err <= 1e-3, f"{err:.3e}"
