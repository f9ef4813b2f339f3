"""Edge cases of the layer solve and the resident stepper, against the
oracle (FP64 <= 1e-9 of the bounding-box diagonal) or bit-identity:

  * a single tet, one and two layers;
  * a layer whose tets are all rigid (one body, no elastic tet to sweep) and
    a layer at 0 % (all elastic);
  * zero iterations in a layer;
  * a mesh without pins;
  * obstacles that touch no vertex (empty device contact list, with and
    without contact colouring and the residual monitor);
  * a ragged batch (a single-tet scene merged with blocks) stepping
    bit-identically to its scenes alone;
  * the device layer builder on a single tet at 0 % and 100 %.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.contacts import PlaneContactFinder3D
from multilayersolver2024_b200.mesh3d import Mesh3D, merge_meshes, to_lame
from multilayersolver2024_b200.xpbd_layer3d import (ResidentSim, Solver, XpbdLayer3D, build_layers_device,
                                                    find_boundary_vertices, union_find_layers)

from helpers import Case, block_mesh, rel_pos_err

pytestmark = pytest.mark.gpu


def _one_tet(pin=False):
    V = np.array([[0, 0, 0], [0.1, 0, 0], [0, 0.1, 0], [0, 0, 0.1]], float)
    m = Mesh3D.from_arrays(V, np.array([[1, 2, 3, 4]]), *to_lame(0.3, 1e5), energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
    if pin:
        m.pin([1])
    return m


@pytest.mark.parametrize("layers,iterations", [([0], [5]), ([100, 0], [2, 3]), ([0], [0])])
def test_single_tet(gpu, layers, iterations):
    m = _one_tet()
    case = Case(m, layers, iterations, seed=3)
    ref, got = case.oracle(), case.product(_lib.MLX_FP64)
    assert rel_pos_err(got[0], ref[0], m) <= 1e-9


@pytest.mark.parametrize("energy", [_lib.MLX_ENERGY_STVK_VOIGT, _lib.MLX_ENERGY_NEOHOOKEAN])
def test_all_rigid_and_all_elastic_layers_without_pins(gpu, energy):
    m = block_mesh(dims=(4, 2, 2), energy=energy, seed=6, pin_x0=False)
    case = Case(m, [100, 0], [3, 4], seed=7)
    assert case.ls.numRigids.tolist() == [0, 1]  # sorted columns: 0 % then 100 % (one body)
    ref, got = case.oracle(), case.product(_lib.MLX_FP64)
    assert rel_pos_err(got[0], ref[0], m) <= 1e-9


def _resident(m, sets, finders, coloring, residuals, steps=3):
    it = XpbdLayer3D()
    it.setLayers([50, 0])
    it.iterations = [2, 3]
    it.customRigidSets = sets
    it.precision = _lib.MLX_FP64
    it.contactColoring = coloring
    it.computeResiduals = residuals
    ls = find_boundary_vertices(m, sets, [0, int(sets[:, 1].max())])
    s = Solver(m, precision=_lib.MLX_FP64, material="blocks")
    sim = ResidentSim(s, it, ls, 0.01, p0=m.p, v0=np.zeros_like(m.p))
    if finders:
        sim.set_obstacles(finders)
    out = []
    for _ in range(steps):
        sim.step(1, graph=True)
        out.append(sim.state()[0])
        if finders:
            assert sim.contact_count() == 0
    s.close()
    return out


@pytest.mark.parametrize("coloring", [False, True])
@pytest.mark.parametrize("residuals", [False, True])
def test_obstacles_touching_nothing(gpu, coloring, residuals):
    V, T, cube = scenes.generate_beam(4, 2, 2, 0.1)
    m = Mesh3D.from_arrays(V, T, *to_lame(0.3, 1e5), energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
    m.pin(np.nonzero(np.isclose(V[:, 0], 0.0))[0] + 1)
    forced = np.zeros(m.T, bool)
    forced[m.pinnedTets - 1] = True
    sets = np.asfortranarray(np.stack([np.zeros(m.T, np.int32),
                                       scenes.cluster_rigid_sets(cube, (4, 2, 2), 2, forced)], 1))
    far = [PlaneContactFinder3D([0, 0, 1.0], [0, 0, -10.0])]
    a = _resident(m, sets, far, coloring, residuals)
    b = _resident(m, sets, [], False, residuals)
    for k in range(len(a)):
        np.testing.assert_array_equal(a[k], b[k])


def test_ragged_batch_with_a_single_tet_scene(gpu):
    from test_step_gpu import _resident_run
    parts = [block_mesh(dims=(5, 2, 2), seed=1), _one_tet(pin=True), block_mesh(dims=(3, 3, 2), seed=2)]
    batch = merge_meshes(parts)
    got, _ = _resident_run(Scene_of(batch), 3, _lib.MLX_FP32)
    for k, part in enumerate(parts):
        solo, _ = _resident_run(Scene_of(merge_meshes([part])), 3, _lib.MLX_FP32)
        a, b = 3 * batch.part_vertex_offsets[k], 3 * batch.part_vertex_offsets[k + 1]
        for s in range(3):
            np.testing.assert_array_equal(got[s][a:b], solo[s], err_msg=f"scene {k} step {s}")


def Scene_of(mesh):
    return scenes.Scene("edge", mesh, 0.01, 3, [0], [4])


@pytest.mark.parametrize("pct", [0.0, 100.0])
def test_device_layer_builder_single_tet(gpu, pct):
    m = _one_tet()
    s = Solver(m, precision=_lib.MLX_FP32, material="lame")
    forced = np.zeros(1, np.uint8)
    p = m.p + 0.001
    got = build_layers_device(s, m, p, m.p, 0.01, [pct], forced)
    order = np.array([1], np.int32)
    sets, nr = union_find_layers(m, order, [pct], forced)
    np.testing.assert_array_equal(got.rigidBodySetsPerLayer, sets)
    np.testing.assert_array_equal(got.numRigids, nr)
    s.close()
