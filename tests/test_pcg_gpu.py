"""PCG on the device (mlx_pcg_solve) against the restatement of solvePCG.m
on the assembled system: the same iterates to 1e-9 (relative to ||x||) and
the same residual history (rtol 1e-7), FP64 and FP32 solvers (the PCG runs
in FP64 in both)."""
import ctypes as C

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib
from multilayersolver2024_b200._lib import check, f64
from multilayersolver2024_b200.xpbd_layer3d import Solver
from oracle import pcg as P

from helpers import block_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.MLX_FP64, _lib.MLX_FP32])
@pytest.mark.parametrize("iterations", [1, 25])
def test_device_pcg_matches_solvepcg(gpu, precision, iterations):
    m = block_mesh(dims=(6, 3, 3), energy=_lib.MLX_ENERGY_NEOHOOKEAN, seed=4)
    h = 1.0 / 60.0
    s = Solver(m, precision=precision, material="lame")
    b = np.random.default_rng(iterations).normal(0, 1, 3 * m.N)
    x = np.zeros(3 * m.N)
    res = np.zeros(iterations)
    lib = s._lib
    check("mlx_pcg_solve", lib.mlx_pcg_solve(s.handle, h, f64(b), iterations, f64(x), f64(res)), lib)
    A, prec, free = P.system(m, h)
    xr, rr = P.solve_pcg(iterations, A, b[free], np.zeros(free.size), prec)
    pinned = np.asarray(m.pinnedDOFs, np.int64) - 1
    assert np.all(x[pinned] == 0)
    assert np.abs(x[free] - xr).max() <= 1e-9 * np.abs(xr).max()
    np.testing.assert_allclose(res, rr, rtol=1e-7)
