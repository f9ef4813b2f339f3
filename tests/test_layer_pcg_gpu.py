"""The PCG in the layer solve (mlx_layer_pcg): Newton-PCG corrections of the
last (fine) Neo-Hookean layer between Gauss-Seidel sweeps.

  * FP64, one layerSolve through mlx_layer_solve (host stop rules) against
    the same algorithm restated on the CPU (oracle/pcg.py
    nh_linearized_step + solve_pcg for the corrections, the oracle's
    projectGS for the sweeps in between): positions within 1e-8 of the
    bounding-box diagonal, multipliers within 1e-6 relative, the same
    number of projectGS iterations;
  * the resident stepper with the stop rules on the device (the corrections
    as a conditional node inside the WHILE node of projectGS) and without a
    graph (host rules): the same iterations and positions (FP64, 1e-9);
  * the gain: on a Neo-Hookean block (E log-uniform in [1e4, 1e7]) FP32 steps
    to residual 1e-4 take under half the projectGS iterations of the plain
    solve, reach the residual, and stay within 5e-3 of the bounding-box
    diagonal of the plain solve's positions (measured 1.2e-3 after 4 steps
    on this small, soft block; 1.4e-4 on config 2 and 2.5e-4 on config 5:
    the converged positions of Gauss-Seidel on these constraints depend on
    its path, and the corrections change the path).
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, to_lame
from multilayersolver2024_b200.xpbd_layer3d import ResidentSim, Solver, XpbdLayer3D, find_boundary_vertices

from helpers import Case

pytestmark = pytest.mark.gpu


def _nh_block(dims=(12, 4, 4), seed=2, pin_z0=True):
    rng = np.random.default_rng(seed)
    V, T, _ = scenes.generate_beam(*dims, 0.1)
    nt = T.shape[0]
    mu, lam = to_lame(rng.uniform(0.25, 0.45, nt), np.exp(rng.uniform(np.log(1e4), np.log(1e7), nt)))
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, energy_type=_lib.MLX_ENERGY_NEOHOOKEAN)
    if pin_z0:
        m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
    return m


def test_fp64_layer_solve_matches_cpu_restatement(gpu, oracle):
    from oracle import pcg as PCG
    m = _nh_block()
    case = Case(m, [0], [10], seed=3, h=1.0 / 60.0, perturb=0.002, vel=0.5)
    case.integ.computeResiduals = True
    case.integ.runUntilResSmallerThan = 1e-4
    case.integ.hangingStop = 20000
    k_pcg, every = 60, 40
    s = Solver(m, precision=_lib.MLX_FP64, material="lame")
    s.layer_pcg(k_pcg, every)
    xi_g, _, ra_g, _, lam_g, it_g = case.product(_lib.MLX_FP64, "lame", solver=s)
    s.close()
    # the same algorithm on the CPU: release, correction, then sweeps of
    # `every` iterations (stop rules every iteration) with a correction
    # between them
    h, nt = case.h, m.T
    free = np.setdiff1d(np.arange(3 * m.N), m.pinnedDOFs - 1)
    x = case.xi + h * case.resv
    lam = np.asfortranarray(case.lam.copy())

    def correct(x, lam):
        A, b, prec, J, W, C = PCG.nh_linearized_step(m, x, h, np.stack([lam[:, 0], lam[:, 1]], 1).ravel(), free)
        dxf, _ = PCG.solve_pcg(k_pcg, A, b, np.zeros(free.size), prec)
        dx = np.zeros(3 * m.N)
        dx[free] = dxf
        ln = -(W @ (C + J @ dx))
        out = np.zeros_like(lam)
        out[:, 0], out[:, 1] = ln[0::2], ln[1::2]
        return x + dx, out

    x, lam = correct(x, lam)
    P = oracle.params(case.integ, h)
    total = 0
    while True:
        P.hanging_stop = every
        x, _, ra, _, lam, its = oracle.layer_solve(m, case.ls, case.integ.layersMap, case.integ.iterations, P,
                                                   oracle.ContactList(), x, lam, case.oldp, case.oldOldp, case.f,
                                                   np.zeros(3 * m.N), case.pinnedx, np.array([0.0]), 0.0, "lame",
                                                   True)
        total += its
        if ra[-1] <= 1e-4 or total > 20000:
            break
        x, lam = correct(x, lam)
    d = m.bbox_diagonal()
    assert ra_g[-1] <= 1e-4 and ra[-1] <= 1e-4
    assert it_g == total, (it_g, total)
    assert np.abs(xi_g - x).max() / d <= 1e-8
    assert np.abs(lam_g[:, :2] - lam[:, :2]).max() <= 1e-6 * np.abs(lam[:, :2]).max()


def _stepper(m, precision, pcg=(0, 0), layers=([0], [10]), graph_ok=True):
    it = XpbdLayer3D()
    it.setLayers(layers[0])
    it.iterations = list(layers[1])
    sets = np.zeros((m.T, 1), np.int32, order="F")
    it.customRigidSets = sets
    it.precision = precision
    it.computeResiduals = True
    it.runUntilResSmallerThan = 1e-4
    it.hangingStop = 20000
    ls = find_boundary_vertices(m, sets, [0])
    s = Solver(m, precision=precision, material="lame")
    if pcg[0]:
        s.layer_pcg(*pcg)
    v0 = np.zeros_like(m.p)
    top = np.isclose(m.p[2::3], m.p[2::3].max())
    v0[2::3][top] = -2.0
    return ResidentSim(s, it, ls, 1.0 / 60.0, p0=m.p, v0=v0)


def test_device_and_host_stop_rules_agree(gpu):
    m = _nh_block(dims=(8, 4, 4), seed=4)
    dev = _stepper(m, _lib.MLX_FP64, pcg=(40, 30))
    host = _stepper(m, _lib.MLX_FP64, pcg=(40, 30))
    d = m.bbox_diagonal()
    for _ in range(3):
        dev.step(1, graph=True)
        host.step(1, graph=False)
        ra_d, it_d, _, st_d = dev.monitor()
        ra_h, it_h, _, st_h = host.monitor()
        assert st_d == 0 and st_h == 0 and it_d == it_h
        assert np.abs(dev.state()[0] - host.state()[0]).max() / d <= 1e-9
        np.testing.assert_allclose(ra_d, ra_h, rtol=1e-7, atol=1e-12)


def test_gain_over_the_plain_solve(gpu):
    m = _nh_block(dims=(24, 6, 6), seed=2)
    plain = _stepper(m, _lib.MLX_FP32)
    fast = _stepper(m, _lib.MLX_FP32, pcg=(100, 50))
    d = m.bbox_diagonal()
    it_p = it_f = 0
    for _ in range(4):
        plain.step(1, graph=True)
        fast.step(1, graph=True)
        ra_p, ip, _, _ = plain.monitor()
        ra_f, iff, _, st = fast.monitor()
        assert st == 0 and abs(ra_f[-1]) <= 1e-4
        it_p += ip
        it_f += iff
        assert np.abs(fast.state()[0] - plain.state()[0]).max() / d <= 5e-3
    print(f"projectGS iterations to residual 1e-4 over 4 steps: plain {it_p}, with the layer PCG {it_f}")
    assert it_f < 0.5 * it_p
