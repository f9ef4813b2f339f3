"""The PCG oracle (CPU): the assembled stiffness annihilates rigid
translations and is symmetric; solvePCG's restatement converges to the
direct solution."""
import numpy as np
import scipy.sparse.linalg as spla

from multilayersolver2024_b200 import _lib
from oracle import pcg as P

from helpers import block_mesh


def test_stiffness_and_pcg_convergence():
    m = block_mesh(dims=(4, 2, 2), energy=_lib.MLX_ENERGY_NEOHOOKEAN, seed=3)
    K = P.stiffness(m)
    assert abs(K - K.T).max() < 1e-9 * abs(K).max()
    for d in range(3):
        u = np.zeros(3 * m.N)
        u[d::3] = 1.0
        assert np.abs(K @ u).max() < 1e-9 * abs(K).max()
    A, prec, free = P.system(m, 1.0 / 60.0)
    b = np.random.default_rng(0).normal(0, 1, free.size)
    x, res = P.solve_pcg(200, A, b, np.zeros(free.size), prec)
    ref = spla.spsolve(A.tocsc(), b)
    assert np.abs(x - ref).max() <= 1e-8 * np.abs(ref).max()
    assert res[-1] < 1e-8 * np.linalg.norm(b)
