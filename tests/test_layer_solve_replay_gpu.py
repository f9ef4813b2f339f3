"""mlx_layer_solve with residual monitoring, replayed as a graph.

The second call of a shape (the same layers and parameters, no host contact
list) runs the loop recorded once, with simpleMonitorError's stop rules
(xpbdLayer3D.m:515-544) on the device: layers as conditional IF nodes,
projectGS as conditional WHILE nodes, the residual array going in and out
through the device monitor's state.  The first call runs the same kernels
with the rules on the host.  Given the same inputs, every call returns the
same positions, multipliers, residual array, runUntil and iteration count,
bit for bit (the device monitor sums the residual's partials in the order
the host path does); sum_non_monitored_time passes through a replay.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib
from multilayersolver2024_b200.xpbd_layer3d import Solver, XpbdLayer3D

from helpers import Case, block_mesh

pytestmark = pytest.mark.gpu

CASES = {
    # name: (iterations, runUntil, hangingStop, StopAtImprovementPercent, giveUp, energy, layer PCG)
    "fixed_with_residuals": ([2, 3], -1.0, 30, 0.0, False, _lib.MLX_ENERGY_STVK_VOIGT, None),
    "run_until": ([2, 3], 1e-6, 400, 0.0, False, _lib.MLX_ENERGY_STVK_VOIGT, None),
    "hanging_stop": ([2, 1], 1e-30, 6, 0.0, False, _lib.MLX_ENERGY_STVK_VOIGT, None),
    "improvement_percent": ([2, 3], -1.0, 400, 90.0, False, _lib.MLX_ENERGY_STVK_VOIGT, None),
    "give_up": ([4, 3], -1.0, 400, 0.0, True, _lib.MLX_ENERGY_STVK_VOIGT, None),
    "neo_hookean_layer_pcg": ([0], 1e-6, 5000, 0.0, False, _lib.MLX_ENERGY_NEOHOOKEAN, (30, 20)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_replay_matches_host_rules(gpu, name):
    iters, ru, hs, pct, give_up, energy, pcg = CASES[name]
    m = block_mesh(dims=(8, 3, 3), energy=energy, seed=5)
    integ = XpbdLayer3D()
    integ.computeResiduals = True
    integ.runUntilResSmallerThan = ru
    integ.hangingStop = hs
    integ.StopAtImprovementPercent = pct
    integ.giveUpEnabled = give_up
    integ.giveUpThreshold = -1.0
    integ.LastLayerGiveUpEnabled = False
    layers = [0] if len(iters) == 1 else [50, 0]
    iterations = [10] if len(iters) == 1 else iters
    case = Case(m, layers, iterations, seed=7, integ=integ, h=1.0 / 60.0)
    s = Solver(m, precision=_lib.MLX_FP64, material="lame")
    if pcg:
        s.layer_pcg(*pcg)
    first = case.product(_lib.MLX_FP64, "lame", solver=s)   # host rules (builds the layer statics)
    second = case.product(_lib.MLX_FP64, "lame", solver=s)  # recorded, then replayed
    third = case.product(_lib.MLX_FP64, "lame", solver=s)   # replayed
    s.close()
    xi1, snm1, ra1, ru1, lam1, it1 = first
    assert it1 > 0
    assert snm1 > 0.0  # the host rules time their residuals; a replay passes the input (0) through
    for xi, snm, ra, ru_, lam, it in (second, third):
        assert it == it1
        assert ru_ == ru1
        np.testing.assert_array_equal(ra, ra1)
        np.testing.assert_array_equal(xi, xi1)
        np.testing.assert_array_equal(lam, lam1)
        assert snm == 0.0
