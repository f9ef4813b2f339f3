"""The residual monitor and stop rules in resident steps (simpleMonitorError,
xpbdLayer3D.m:515-544): on the device inside one captured graph (layers as
conditional IF nodes, projectGS loops as conditional WHILE nodes) and on the
host without a graph, against the oracle integrate over three steps.

Compared per step: positions (FP64, <= 1e-9 of the bounding-box diagonal),
the residual array (entries within 1e-9 of its largest entry), the total
projectGS iterations (equal) and runUntilResSmallerThan (equal), which
carries over from step to step.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, to_lame
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, ResidentSim, Solver, StepCache, XpbdLayer3D,
                                                    find_boundary_vertices)

pytestmark = pytest.mark.gpu

CASES = {
    # name: (iterations, runUntil, hangingStop, StopAtImprovementPercent, giveUp)
    "fixed_with_residuals": ([2, 3], -1.0, 30, 0.0, False),
    "run_until_early": ([2, 3], 1e-6, 400, 0.0, False),
    "run_until_extends_last_layer": ([2, 1], 1e-13, 400, 0.0, False),
    "hanging_stop": ([2, 1], 1e-30, 4, 0.0, False),
    "improvement_percent": ([2, 3], -1.0, 400, 90.0, False),
    "give_up": ([4, 3], -1.0, 400, 0.0, True),
}

_V, _T, _CUBE = scenes.generate_beam(6, 3, 3, 0.1)


def _mesh():
    m = Mesh3D.from_arrays(_V, _T, *to_lame(0.35, 2e4), energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
    m.pin(np.nonzero(np.isclose(_V[:, 0], 0.0))[0] + 1)
    m.v[2::3] = -2.0 * (_V[:, 0] / _V[:, 0].max())
    return m


def _integ(name, sets):
    iters, ru, hs, pct, give_up = CASES[name]
    it = XpbdLayer3D()
    it.setLayers([50, 0])
    it.iterations = list(iters)
    it.customRigidSets = sets
    it.computeResiduals = True
    it.runUntilResSmallerThan = ru
    it.hangingStop = hs
    it.StopAtImprovementPercent = pct
    it.giveUpEnabled = give_up
    it.giveUpThreshold = -1.0  # any change once the residual has decreased ends a (non-last) layer
    it.LastLayerGiveUpEnabled = False
    it.precision = _lib.MLX_FP64
    return it


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("name", list(CASES))
def test_monitored_steps_match_oracle(gpu, oracle, name, graph):
    h, steps = 1.0 / 60.0, 3
    m = _mesh()
    forced = np.zeros(m.T, bool)
    forced[m.pinnedTets - 1] = True
    coarse = scenes.cluster_rigid_sets(_CUBE, (6, 3, 3), 2, forced)
    sets = np.asfortranarray(np.stack([np.zeros(m.T, np.int32), coarse], 1))
    # oracle
    mo = _mesh()
    io = _integ(name, sets)
    cache = StepCache()
    ref = []
    for frame in range(1, steps + 1):
        ra, iters = oracle.integrate(io, mo, h, ContactSet(), cache, frame)
        ref.append((mo.p.copy(), np.asarray(ra, float), int(iters), float(io.runUntilResSmallerThan)))
    # resident stepper
    ls = find_boundary_vertices(m, sets, [0, int(sets[:, 1].max())])
    s = Solver(m, precision=_lib.MLX_FP64, material="blocks")
    sim = ResidentSim(s, _integ(name, sets), ls, h, p0=m.p, v0=m.v)
    d = m.bbox_diagonal()
    for k in range(steps):
        sim.step(1, graph=graph)
        ra, iters, run_until, status = sim.monitor()
        p_ref, ra_ref, it_ref, ru_ref = ref[k]
        assert status == 0
        assert iters == it_ref, f"step {k}: {iters} iterations, oracle {it_ref}"
        assert ra.size == ra_ref.size
        np.testing.assert_allclose(ra, ra_ref, rtol=0, atol=1e-9 * max(np.abs(ra_ref).max(), 1e-300))
        assert run_until == pytest.approx(ru_ref, rel=1e-9, abs=0)
        err = np.abs(sim.state()[0] - p_ref).max() / d
        assert err <= 1e-9, f"step {k}: {err:.3e}"
