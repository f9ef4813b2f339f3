"""Config 4 (contact-heavy drop, three cluster layers) at reduced size:
2 boxes of 4^3 cubes dropped from just above a ground plane and spheres,
contacts detected on the device every step, against the oracle integrate fed
with the oracle finders' lists (FP64 <= 1e-9, FP32 <= 1e-4 of the
bounding-box diagonal over 32 steps); and the full-size scene steps stay
finite with contacts."""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.xpbd_layer3d import ResidentSim, Solver, StepCache, XpbdLayer3D, find_boundary_vertices

pytestmark = pytest.mark.gpu


def _small():
    # the boxes start 5-15 mm above the ground / sphere tops and fall with
    # an initial 1 m/s (set by the test), so contacts begin within a few steps
    return scenes.config4(seed=11, n_boxes=2, cubes=4, grid=(2, 1), spacing=1.5, n_spheres=1, coarse=2, mid=2,
                          drop=(0.005, 0.015))


def _integ(sc, precision):
    it = XpbdLayer3D()
    it.Gravity = sc.gravity
    it.setLayers(sc.layers)
    it.iterations = list(sc.iterations)
    it.customRigidSets = sc.custom_sets
    it.precision = precision
    it.contactResistance = sc.settings["contactResistance"]
    return it


@pytest.mark.parametrize("precision,tol", [(_lib.MLX_FP64, 1e-9), (_lib.MLX_FP32, 1e-4)])
def test_small_drop_matches_oracle(gpu, oracle, precision, tol):
    steps = 32
    so = _small()
    oracle.load().orc_set_threads(8)
    mo = so.mesh
    mo.v[2::3] = -1.0
    integ = _integ(so, _lib.MLX_FP64)
    cache = StepCache()
    ref, nref = [], []
    for frame in range(1, steps + 1):
        cs = oracle.find_contacts(so.contact_finders, mo.p)
        nref.append(np.unique(cs.vertex_ids).size)
        oracle.integrate(integ, mo, so.h, cs, cache, frame)
        ref.append(mo.p.copy())
    assert max(nref) > 20
    sc = _small()
    m = sc.mesh
    sets = sc.custom_sets
    ls = find_boundary_vertices(m, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    s = Solver(m, precision=precision, material="blocks" if precision == _lib.MLX_FP64 else "lame")
    v0 = np.zeros_like(m.p)
    v0[2::3] = -1.0
    sim = ResidentSim(s, _integ(sc, precision), ls, sc.h, p0=m.p, v0=v0)
    sim.set_obstacles(sc.contact_finders, restitution=1e-2)
    d = m.bbox_diagonal()
    for k in range(steps):
        sim.step(1, graph=True)
        err = np.abs(sim.state()[0] - ref[k]).max() / d
        assert err <= tol, f"step {k}: {err:.3e}"


def test_full_scene_runs_with_contacts(gpu):
    sc = scenes.config4(drop=(0.0, 0.02))
    m = sc.mesh
    sets = sc.custom_sets
    ls = find_boundary_vertices(m, sets, [int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])])
    s = Solver(m, precision=_lib.MLX_FP32, material="lame")
    sim = ResidentSim(s, _integ(sc, _lib.MLX_FP32), ls, sc.h, p0=m.p, v0=np.zeros_like(m.p))
    sim.set_obstacles(sc.contact_finders, restitution=1e-2)
    counts = []
    for _ in range(45):
        sim.step(1, graph=True)
        counts.append(sim.contact_count())
    p = sim.state()[0]
    assert np.all(np.isfinite(p))
    assert max(counts) > 100
    assert p[2::3].min() > -0.05  # nothing falls through the ground
