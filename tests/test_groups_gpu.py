"""The component-group path (one launch per body-free layer, one CTA per group
of vertex-disconnected components, vertex records in shared memory) against
the colour launches: positions bit-identical at every step, for

  * a batch of Neo-Hookean blocks with pinned bases and a coarse cluster
    layer (the cluster layer keeps the colour launches, the fine layer takes
    the group path), FP32;
  * the contact-heavy drop at reduced size (device contacts in the group
    kernel's contact phase), FP32, and the same drop through the host API
    (the finders' contact list grouped by vertex in the group kernel);
  * damped StVK blocks (step-start positions read for the damping term),
    FP32 and FP64;
  * the single-component cantilever of config 1 with the path forced, FP64,
    which also matches the oracle;
  * 64 copies of that cantilever in one mesh, FP32;
  * batches of blocks on clusters of 2 and 4 CTAs per group (records in
    distributed shared memory), with colours that fit one pass of the
    cluster and colours that need several: FP32 bit-identical; FP64
    Neo-Hookean within 1e-12 m (measured 8.5e-14: the same projection
    inlined into two kernels contracts its FP64 multiply-adds differently).
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import merge_meshes
from multilayersolver2024_b200.scenes import Scene
from multilayersolver2024_b200.xpbd_layer3d import ResidentSim, Solver, XpbdLayer3D, find_boundary_vertices

from helpers import block_mesh

pytestmark = pytest.mark.gpu

GROUP_PATH = "CTAs each owning whole components"


def _integ(sc, precision):
    it = XpbdLayer3D()
    it.Gravity = sc.gravity
    it.setLayers(sc.layers)
    it.iterations = list(sc.iterations)
    it.customRigidSets = sc.custom_sets
    it.precision = precision
    it.contactResistance = sc.settings.get("contactResistance", it.contactResistance)
    return it


def _run(monkeypatch, make_scene, groups, steps, precision, v0z=0.0):
    monkeypatch.setenv("MLXPBD_GROUPS", groups)
    for var in ("MLXPBD_CLUSTER", "MLXPBD_PERSISTENT"):
        monkeypatch.delenv(var, raising=False)
    sc = make_scene()
    m = sc.mesh
    if sc.custom_sets is not None:
        sets = sc.custom_sets
        nr = [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])]
    else:
        sets = np.zeros((m.T, 1), np.int32, order="F")
        nr = [0]
    ls = find_boundary_vertices(m, sets, nr)
    s = Solver(m, precision=precision, material="blocks" if precision == _lib.MLX_FP64 else "lame")
    v0 = np.zeros_like(m.p)
    v0[2::3] = v0z
    sim = ResidentSim(s, _integ(sc, precision), ls, sc.h, p0=m.p, v0=v0)
    if sc.impulse is not None:
        sim.add_velocity(sc.impulse[0], sc.impulse[1])
    if sc.contact_finders:
        sim.set_obstacles(sc.contact_finders, restitution=1e-2)
    traj = []
    for _ in range(steps):
        sim.step(1, graph=True)
        traj.append(sim.state()[0])
    path = s.launch_path
    s.close()
    return traj, path


def _same(monkeypatch, make_scene, steps, precision, v0z=0.0, atol=0.0):
    ref, p0 = _run(monkeypatch, make_scene, "0", steps, precision, v0z)
    got, p1 = _run(monkeypatch, make_scene, "1", steps, precision, v0z)
    assert GROUP_PATH not in p0
    assert GROUP_PATH in p1, p1
    for k in range(steps):
        if atol == 0.0:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"step {k}")
        else:
            np.testing.assert_allclose(got[k], ref[k], rtol=0.0, atol=atol, err_msg=f"step {k}")
    return got


def test_batch_of_blocks(gpu, monkeypatch):
    _same(monkeypatch, lambda: scenes.config3(seed=7, n_scenes=6, tmin=1500, tmax=6000), 4, _lib.MLX_FP32)


def test_drop_with_device_contacts(gpu, monkeypatch):
    def small():
        return scenes.config4(seed=11, n_boxes=3, cubes=4, grid=(3, 1), spacing=1.5, n_spheres=1, coarse=2, mid=2,
                              drop=(0.005, 0.015))
    _same(monkeypatch, small, 30, _lib.MLX_FP32, v0z=-1.0)


def test_replicated_cantilevers(gpu, monkeypatch):
    """64 copies of the config-1 cantilever: one CTA owns many whole copies."""
    _same(monkeypatch, lambda: scenes.config1_replicated(64, per_row=8), 5, _lib.MLX_FP32)


def test_host_contact_lists_on_the_group_path(gpu, monkeypatch):
    """simulate3D's loop through the host API (finders, then integrate ->
    mlx_layer_solve with the contact list): the body-free layer runs on the
    group path with the list's vertex groups, and every frame's positions
    and velocities equal the colour launches' bit for bit."""
    from multilayersolver2024_b200.contacts import find_contacts
    from multilayersolver2024_b200.xpbd_layer3d import StepCache

    def run(flag):
        monkeypatch.setenv("MLXPBD_GROUPS", flag)
        sc = scenes.config4(seed=11, n_boxes=3, cubes=4, grid=(3, 1), spacing=1.5, n_spheres=1, coarse=2, mid=2,
                            drop=(0.005, 0.015))
        m = sc.mesh
        m.v[2::3] = -1.0
        it = _integ(sc, _lib.MLX_FP32)
        cache = StepCache()
        out, counts = [], []
        for frame in range(1, 31):
            cs = find_contacts(it.solver(m), sc.contact_finders, m.p)
            counts.append(int(cs.vertex_ids.size))
            it.integrate(m, sc.h, cs, cache, frame)
            out.append((m.p.copy(), m.v.copy()))
        paths = [s.launch_path for s in it._solvers.values()]
        for s in it._solvers.values():
            s.close()
        return out, counts, paths

    a, ca, pa = run("1")
    b, cb, pb = run("0")
    assert any(GROUP_PATH in p for p in pa) and not any(GROUP_PATH in p for p in pb)
    assert max(ca) > 20 and ca == cb
    for k in range(len(a)):
        np.testing.assert_array_equal(a[k][0], b[k][0], err_msg=f"positions, frame {k + 1}")
        np.testing.assert_array_equal(a[k][1], b[k][1], err_msg=f"velocities, frame {k + 1}")


def _damped_blocks():
    parts = [block_mesh(dims=d, energy=_lib.MLX_ENERGY_STVK_VOIGT, seed=k, alpha1=0.02)
             for k, d in enumerate([(6, 3, 3), (4, 2, 2), (5, 3, 2)])]
    m = merge_meshes(parts)
    m.v[2::3] = -0.5
    return Scene("damped_blocks", m, 1.0 / 60.0, 10, [0], [6])


@pytest.mark.parametrize("precision", [_lib.MLX_FP32, _lib.MLX_FP64])
def test_damped_stvk_blocks(gpu, monkeypatch, precision):
    _same(monkeypatch, _damped_blocks, 5, precision)


def test_forced_single_component_matches_oracle(gpu, monkeypatch, oracle):
    from test_step_gpu import _oracle_run
    got = _same(monkeypatch, scenes.config1, 20, _lib.MLX_FP64)
    ref = _oracle_run(scenes.config1(), 20, oracle)
    d = scenes.config1().mesh.bbox_diagonal()
    assert max(np.abs(a - b).max() / d for a, b in zip(got, ref)) <= 1e-9


def test_host_layer_solve_graph_replay_is_bit_identical(gpu, monkeypatch):
    """mlx_layer_solve replays its layer loop from a CUDA graph while calls
    keep one shape (fixed iterations, no contacts, same masks): integrate
    over several frames equals the uncaptured loop bit for bit, with
    bodies, boundary glue and pins (config 2 class at reduced size)."""
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet, StepCache

    def run(flag):
        monkeypatch.setenv("MLXPBD_HOST_GRAPH", flag)
        sc = scenes.config2(seed=4, nx=16, ny=4, nz=4, cluster=4)
        m = sc.mesh
        m.v[sc.impulse[0] - 1] += sc.impulse[1]
        it = _integ(sc, _lib.MLX_FP32)
        cache = StepCache()
        out = []
        for frame in range(1, 7):
            it.integrate(m, sc.h, ContactSet(), cache, frame)
            out.append(m.p.copy())
        for s in it._solvers.values():
            s.close()
        return out
    a, b = run("1"), run("0")
    for k in range(len(a)):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"frame {k + 1}")


@pytest.mark.parametrize("cs,precision,dims", [
    (2, _lib.MLX_FP32, (1500, 6000)),
    (4, _lib.MLX_FP32, (1500, 6000)),
    (2, _lib.MLX_FP32, (30000, 40000)),   # colours of a group exceed one pass of the cluster
    (4, _lib.MLX_FP64, (1500, 6000)),
])
def test_batch_on_thread_block_clusters(gpu, monkeypatch, cs, precision, dims):
    monkeypatch.setenv("MLXPBD_GROUP_CS", str(cs))
    got = _same(monkeypatch, lambda: scenes.config3(seed=7, n_scenes=5, tmin=dims[0], tmax=dims[1]), 3, precision,
                atol=0.0 if precision == _lib.MLX_FP32 else 1e-12)
    _, path = _run(monkeypatch, lambda: scenes.config3(seed=7, n_scenes=5, tmin=dims[0], tmax=dims[1]), "1", 1,
                   precision)
    assert f"clusters of {cs} CTAs" in path, path
    assert np.all(np.isfinite(got[-1]))
