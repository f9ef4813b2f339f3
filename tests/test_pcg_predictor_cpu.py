"""The PCG in the layer solve, measured (CPU, FP64 oracle).

Predictor experiment: before the fine layer's Gauss-Seidel, solve the XPBD
step linearised at the released positions with solvePCG's iteration
(oracle/pcg.py: (M + J^T W J) dx = -J^T W C, 3x3 block-Jacobi, the
multipliers then lam = -W (C + J dx), a state that keeps M dx = J^T lam) and
start projectGS from (x~ + dx, lam).  On a single-layer Neo-Hookean block
(E log-uniform in [1e4, 1e7]) after three steps of motion the predictor cuts
the first residual of the layer by more than 2x, yet the Gauss-Seidel
iterations to residual 1e-4 fall by well under half (measured here: 803
plain, 664 from the predicted start, a 17 % saving; 9-28 % over other seeds
and block sizes): most iterations are spent in the slow tail of the
nonlinear solve, not in the start.  The same correction repeated during the
sweep is what removes that tail (tests/test_layer_pcg_gpu.py).  The
converged positions move by ~1.5e-4 of the bounding-box diagonal.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import XpbdLayer3D, _lib, scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, to_lame
from multilayersolver2024_b200.xpbd_layer3d import ContactSet, StepCache, find_boundary_vertices
from oracle import pcg as PCG


def test_linearised_pcg_predictor_saves_few_iterations(oracle):
    oracle.load().orc_set_threads(8)
    nx, ny, nz = 16, 4, 4
    rng = np.random.default_rng(2)
    V, T, _ = scenes.generate_beam(nx, ny, nz, 0.1)
    nt = T.shape[0]
    mu, lam = to_lame(rng.uniform(0.25, 0.45, nt), np.exp(rng.uniform(np.log(1e4), np.log(1e7), nt)))
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, energy_type=_lib.MLX_ENERGY_NEOHOOKEAN)
    m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
    h = 1.0 / 60.0
    integ = XpbdLayer3D()
    integ.setLayers([0])
    integ.iterations = [10]
    integ.customRigidSets = np.zeros((nt, 1), np.int32, order="F")
    integ.computeResiduals, integ.hangingStop = True, 20000
    ls = find_boundary_vertices(m, integ.customRigidSets, [0])
    top = np.nonzero(np.isclose(V[:, 2], nz * 0.1))[0]
    m.v = np.zeros(3 * m.N)
    m.v[3 * top + 2] = -2.0
    cache = StepCache()
    for frame in range(1, 4):
        integ.runUntilResSmallerThan = 1e-4
        oracle.integrate(integ, m, h, ContactSet(), cache, frame, material="lame")
    f = np.zeros(3 * m.N)
    f[2::3] = m.mass[2::3] * integ.Gravity
    free = np.setdiff1d(np.arange(3 * m.N), m.pinnedDOFs - 1)
    resv = m.v.copy()
    resv[free] += h * f[free] / m.mass[free]
    xt = m.p.copy()
    xt[free] += h * resv[free]  # the released positions of the single elastic layer
    P = oracle.params(integ, h)
    P.run_until = 1e-4

    def solve(xi, rv, lam0):
        return oracle.layer_solve(m, ls, integ.layersMap, integ.iterations, P, oracle.ContactList(), xi, lam0, m.p,
                                  m.p, f, rv, m.p[m.pinnedDOFs - 1], np.array([0.0]), 0.0, "lame", True)

    x_pl, _, ra_pl, _, _, it_pl = solve(m.p.copy(), resv, np.zeros((nt, 6), order="F"))
    A, b, prec, J, W, C = PCG.nh_linearized_step(m, xt, h, np.zeros(2 * nt), free)
    dxf, _ = PCG.solve_pcg(100, A, b, np.zeros(free.size), prec)
    dx = np.zeros(3 * m.N)
    dx[free] = dxf
    lam_new = -(W @ (C + J @ dx))
    # the predicted state keeps XPBD's relation M dx = J^T lam on the free
    # DOFs up to the PCG residual (M dx - J^T lam = A dx - b)
    r = (m.mass * dx - J.T @ lam_new)[free]
    assert np.linalg.norm(r) <= 1e-2 * np.linalg.norm(b)
    lam0 = np.zeros((nt, 6), order="F")
    lam0[:, 0], lam0[:, 1] = lam_new[0::2], lam_new[1::2]
    x_pr, _, ra_pr, _, _, it_pr = solve(xt + dx, np.zeros(3 * m.N), lam0)
    assert ra_pr[-1] <= 1e-4 and ra_pl[-1] <= 1e-4
    assert ra_pr[1] < 0.5 * ra_pl[1]          # a much better start ...
    assert it_pr > 0.6 * it_pl, (it_pr, it_pl)  # ... saves well under half of the iterations
    assert np.abs(x_pr - x_pl).max() / m.bbox_diagonal() <= 1e-3
