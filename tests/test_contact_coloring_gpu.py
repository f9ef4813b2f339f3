"""Contacts coloured together with the elastic constraints (mlx_solve_params
contact_coloring = 1; no counterpart in the reference, which projects them
after the colour sweep): each vertex's elastic contacts run in the first
colour phase whose tets do not touch it.  Checked against the oracle's
restatement of the same order (FP64 <= 1e-9, FP32 <= 1e-4 of the
bounding-box diagonal), on the colour launches (with a rigid-cluster layer
and rigid contacts) and on the component-group path (which must be
bit-identical to the colour launches); the order changes the result; host
contact lists are refused."""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200._lib import MlxError
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, ResidentSim, Solver, StepCache, XpbdLayer3D,
                                                    find_boundary_vertices)

from test_contacts_gpu import _falling_scene, _finders

pytestmark = pytest.mark.gpu


def _integ(sets, layers, iterations, precision, coloring, resistance=0.9):
    it = XpbdLayer3D()
    it.setLayers(layers)
    it.iterations = list(iterations)
    it.customRigidSets = sets
    it.precision = precision
    it.contactResistance = resistance
    it.boundaryCompliance = 1e-8
    it.contactColoring = coloring
    return it


def _oracle(oracle, mesh_fn, sets, layers, iterations, h, steps, finders, coloring, v0=None, resistance=0.9):
    oracle.load().orc_set_threads(8)
    m = mesh_fn()
    if v0 is not None:
        m.v = v0.copy()
    it = _integ(sets, layers, iterations, _lib.MLX_FP64, coloring, resistance)
    cache = StepCache()
    out = []
    for frame in range(1, steps + 1):
        cs = oracle.find_contacts(finders(), m.p)
        oracle.integrate(it, m, h, cs, cache, frame)
        out.append(m.p.copy())
    return out


def _resident(m, sets, layers, iterations, h, steps, finders, precision, coloring, v0, resistance=0.9):
    nr = [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])]
    ls = find_boundary_vertices(m, sets, nr)
    s = Solver(m, precision=precision, material="blocks" if precision == _lib.MLX_FP64 else "lame")
    sim = ResidentSim(s, _integ(sets, layers, iterations, precision, coloring, resistance), ls, h, p0=m.p, v0=v0)
    sim.set_obstacles(finders(), restitution=1e-2)
    out = []
    for _ in range(steps):
        sim.step(1, graph=True)
        out.append(sim.state()[0])
    path = s.launch_path
    s.close()
    return out, path


@pytest.mark.parametrize("precision,tol", [(_lib.MLX_FP64, 1e-9), (_lib.MLX_FP32, 1e-4)])
def test_colour_launches_match_oracle(gpu, oracle, monkeypatch, precision, tol):
    monkeypatch.setenv("MLXPBD_GROUPS", "0")
    h, steps = 0.01, 8
    m, sets, v0 = _falling_scene()
    ref = _oracle(oracle, lambda: _falling_scene()[0], sets, [50, 0], [3, 6], h, steps, _finders, True, v0)
    got, path = _resident(m, sets, [50, 0], [3, 6], h, steps, _finders, precision, True, v0)
    assert "one launch per colour" in path
    d = m.bbox_diagonal()
    for k in range(steps):
        err = np.abs(got[k] - ref[k]).max() / d
        assert err <= tol, f"step {k}: {err:.3e}"
    # the colouring changes the order, hence the result
    plain = _oracle(oracle, lambda: _falling_scene()[0], sets, [50, 0], [3, 6], h, steps, _finders, False, v0)
    assert np.abs(plain[-1] - ref[-1]).max() / d > 1e-7


def _small_drop():
    return scenes.config4(seed=11, n_boxes=2, cubes=4, grid=(2, 1), spacing=1.5, n_spheres=1, coarse=2, mid=2,
                          drop=(0.005, 0.015))


def test_group_path_matches_oracle_and_colour_launches(gpu, oracle, monkeypatch):
    h, steps = 1.0 / 120.0, 24
    sc = _small_drop()
    v0 = np.zeros_like(sc.mesh.p)
    v0[2::3] = -1.0
    finders = lambda: _small_drop().contact_finders
    ref = _oracle(oracle, lambda: _small_drop().mesh, sc.custom_sets, sc.layers, sc.iterations, h, steps, finders,
                  True, v0, 0.9)
    runs = {}
    for groups in ("0", "1"):
        monkeypatch.setenv("MLXPBD_GROUPS", groups)
        runs[groups] = _resident(_small_drop().mesh, sc.custom_sets, sc.layers, sc.iterations, h, steps, finders,
                                 _lib.MLX_FP64, True, v0, 0.9)
    assert "CTAs each owning whole components" in runs["1"][1]
    d = sc.mesh.bbox_diagonal()
    for k in range(steps):
        np.testing.assert_array_equal(runs["1"][0][k], runs["0"][0][k], err_msg=f"step {k}")
        err = np.abs(runs["1"][0][k] - ref[k]).max() / d
        assert err <= 1e-9, f"step {k}: {err:.3e}"


def test_host_contact_lists_are_refused(gpu):
    m, sets, v0 = _falling_scene()
    m.v = v0
    it = _integ(sets, [50, 0], [3, 6], _lib.MLX_FP32, True)
    from oracle import oracle as O
    cs = O.find_contacts(_finders(), m.p)
    assert cs.vertex_ids.size > 0
    with pytest.raises(MlxError):
        it.integrate(m, 0.01, cs, StepCache(), 1)
