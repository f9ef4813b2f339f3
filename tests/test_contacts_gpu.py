"""Contact detection on the device (a18) and the resident stepper with
analytic obstacles, against the oracle's finders and integrate.

  * mlx_find_contacts: the concatenated contact list (ids, normals, collider
    points, compliances) is bit-identical to the oracle finders', FP64, for
    planes, spheres and rotated boxes with overlapping obstacles;
  * resident stepper with obstacles (contacts detected on the device every
    step, projected in every layer, contactVelocityUpdate after the step)
    against the oracle integrate fed with the oracle finders' lists of the
    step-start positions: FP64 <= 1e-9, FP32 <= 1e-4 of the bounding-box
    diagonal over 8 steps, rigid contacts on and off;
  * the residual monitor (device and host) with those contacts: residual
    arrays, iteration counts and positions against the oracle, FP64.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.contacts import (PlaneContactFinder3D, PlatformContactDetector, SphereContactFinder,
                                                find_contacts)
from multilayersolver2024_b200.mesh3d import Mesh3D, to_lame
from multilayersolver2024_b200.xpbd_layer3d import (ResidentSim, Solver, StepCache, XpbdLayer3D,
                                                    find_boundary_vertices)

pytestmark = pytest.mark.gpu


def _finders():
    return [PlaneContactFinder3D([0, 0, 1.0], [0, 0, 0]),
            SphereContactFinder(0.12, [0.3, 0.15, 0.12]),
            PlatformContactDetector([0, 8, 20], [0.3, 0.5, 0.1], [0.55, 0.15, 0.02], 2e-5),
            PlaneContactFinder3D([0.1, 0, 2.0], [0.7, 0, 0.0], 5e-5)]


@pytest.mark.parametrize("precision", [_lib.MLX_FP64, _lib.MLX_FP32])
def test_device_detection_matches_oracle_finders(gpu, oracle, precision):
    rng = np.random.default_rng(5)
    V, T, _ = scenes.generate_beam(8, 3, 3, 0.1, origin=(0.0, 0.0, -0.03))
    m = Mesh3D.from_arrays(V, T, *to_lame(0.3, 1e5), energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
    s = Solver(m, precision=precision, material="lame")
    for trial in range(3):
        p = m.p + rng.normal(0, 0.02, m.p.size)
        got = find_contacts(s, _finders(), p)
        ref = oracle.find_contacts(_finders(), p)
        assert ref.vertex_ids.size > 20
        np.testing.assert_array_equal(got.vertex_ids, ref.vertex_ids)
        np.testing.assert_array_equal(got.normals, ref.normals)
        np.testing.assert_array_equal(got.points, ref.points)
        np.testing.assert_array_equal(got.compliance, ref.compliance)


def _falling_scene():
    V, T, cube = scenes.generate_beam(6, 3, 3, 0.1, origin=(0.05, 0.0, 0.004))
    m = Mesh3D.from_arrays(V, T, *to_lame(0.3, 2e5), energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
    coarse = scenes.cluster_rigid_sets(cube, (6, 3, 3), 2, np.zeros(m.T, bool))
    sets = np.asfortranarray(np.stack([np.zeros(m.T, np.int32), coarse], 1))
    v0 = np.zeros_like(m.p)
    v0[2::3] = -0.8
    v0[0::3] = 0.3
    return m, sets, v0


def _integ(sets, precision, rigid_contacts):
    it = XpbdLayer3D()
    it.setLayers([50, 0])
    it.iterations = [3, 6]
    it.customRigidSets = sets
    it.precision = precision
    it.useRigidContacts = rigid_contacts
    it.contactResistance = 0.9
    it.boundaryCompliance = 1e-8
    return it


@pytest.mark.parametrize("precision,tol", [(_lib.MLX_FP64, 1e-9), (_lib.MLX_FP32, 1e-4)])
@pytest.mark.parametrize("rigid_contacts", [True, False])
def test_resident_stepper_with_obstacles_matches_oracle(gpu, oracle, precision, tol, rigid_contacts):
    h, steps = 0.01, 8
    m, sets, v0 = _falling_scene()
    # oracle: simulate3D's loop -- finders on the step-start positions, then integrate
    oracle.load().orc_set_threads(8)
    mo, _, _ = _falling_scene()
    mo.v = v0.copy()
    integ = _integ(sets, _lib.MLX_FP64, rigid_contacts)
    cache = StepCache()
    ref, nref = [], []
    for frame in range(1, steps + 1):
        cs = oracle.find_contacts(_finders(), mo.p)
        nref.append(np.unique(cs.vertex_ids).size)
        oracle.integrate(integ, mo, h, cs, cache, frame)
        ref.append(mo.p.copy())
    assert max(nref) > 10
    # device-resident stepper
    ls = find_boundary_vertices(m, sets, [0, int(sets[:, 1].max())])
    s = Solver(m, precision=precision, material="blocks" if precision == _lib.MLX_FP64 else "lame")
    sim = ResidentSim(s, _integ(sets, precision, rigid_contacts), ls, h, p0=m.p, v0=v0)
    sim.set_obstacles(_finders(), restitution=1e-2)
    d = m.bbox_diagonal()
    for k in range(steps):
        sim.step(1, graph=True)
        if precision == _lib.MLX_FP64:
            assert sim.contact_count() == nref[k]
        else:  # FP32 positions may put a vertex on the other side of a surface
            assert abs(sim.contact_count() - nref[k]) <= max(2, nref[k] // 10)
        err = np.abs(sim.state()[0] - ref[k]).max() / d
        assert err <= tol, f"step {k}: {err:.3e}"


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("run_until,hanging_stop", [(-1.0, 400), (0.03, 400), (1e-7, 60)])
def test_monitored_steps_with_obstacles_match_oracle(gpu, oracle, graph, run_until, hanging_stop):
    """Residual monitor with device contacts (the contact rows of
    simpleEvaluateAllConstraintResiduals, K x K expansion included): the
    residual array, the iteration count, runUntil and the positions of every
    step against the oracle fed with its finders' lists, FP64, graph (device
    monitor) and host monitor."""
    h, steps = 0.01, 6
    m, sets, v0 = _falling_scene()

    def integ():
        it = _integ(sets, _lib.MLX_FP64, True)
        it.computeResiduals = True
        it.runUntilResSmallerThan = run_until
        it.hangingStop = hanging_stop
        return it

    oracle.load().orc_set_threads(8)
    mo, _, _ = _falling_scene()
    mo.v = v0.copy()
    io = integ()
    cache = StepCache()
    ref = []
    for frame in range(1, steps + 1):
        cs = oracle.find_contacts(_finders(), mo.p)
        ra, iters = oracle.integrate(io, mo, h, cs, cache, frame)
        ref.append((mo.p.copy(), np.asarray(ra, float), int(iters), float(io.runUntilResSmallerThan),
                    np.unique(cs.vertex_ids).size))
    assert max(r[4] for r in ref) > 10
    ls = find_boundary_vertices(m, sets, [0, int(sets[:, 1].max())])
    s = Solver(m, precision=_lib.MLX_FP64, material="blocks")
    sim = ResidentSim(s, integ(), ls, h, p0=m.p, v0=v0)
    sim.set_obstacles(_finders(), restitution=1e-2)
    d = m.bbox_diagonal()
    for k in range(steps):
        sim.step(1, graph=graph)
        ra, iters, ru, status = sim.monitor()
        p_ref, ra_ref, it_ref, ru_ref, _ = ref[k]
        assert status == 0
        assert iters == it_ref, f"step {k}: {iters} iterations, oracle {it_ref}"
        assert ra.size == ra_ref.size
        np.testing.assert_allclose(ra, ra_ref, rtol=0, atol=1e-9 * max(np.abs(ra_ref).max(), 1e-300))
        assert ru == pytest.approx(ru_ref, rel=1e-9, abs=0)
        err = np.abs(sim.state()[0] - p_ref).max() / d
        assert err <= 1e-9, f"step {k}: {err:.3e}"
