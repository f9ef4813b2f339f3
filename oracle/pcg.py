"""Oracle of the device PCG (test infrastructure only).

`solve_pcg` restates the reference's solvePCG.m (2d/tools/solver/solvePCG.m:
1-56) line by line for a matrix A and a preconditioner function; `system`
assembles the linearly implicit system A = M + h^2 K0 of a tet mesh
(lumped masses, linear-elasticity stiffness at the rest shape from DmInv,
volume, mu, lambda), restricted to the unpinned DOFs, and its 3x3
block-Jacobi preconditioner.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def element_gradients(DmInv_rows):
    """Shape-function gradients g_0..g_3 of one tet (DmInv page, column-major
    9-vector): rows of DmInv for corners 1..3, minus their sum for corner 0."""
    G = np.asarray(DmInv_rows, float).reshape(3, 3, order="F")
    g = [G[0], G[1], G[2]]
    return [-(g[0] + g[1] + g[2])] + g


def stiffness(mesh):
    """K0 (3N x 3N, sparse): K_ab = vol (mu (g_a.g_b) I + mu g_b g_a^T + lambda g_a g_b^T)."""
    N = mesh.N
    rows, cols, vals = [], [], []
    t = np.asarray(mesh.t, np.int64) - 1
    for e in range(mesh.T):
        g = element_gradients(mesh.DmInv[e])
        mu, lm, V = mesh.mu[e], mesh.lam[e], mesh.elV[e]
        for a in range(4):
            for b in range(4):
                Kab = V * (mu * np.dot(g[a], g[b]) * np.eye(3) + mu * np.outer(g[b], g[a]) + lm * np.outer(g[a], g[b]))
                va, vb = t[e, a], t[e, b]
                for i in range(3):
                    for j in range(3):
                        rows.append(3 * va + i); cols.append(3 * vb + j); vals.append(Kab[i, j])
    return sp.csr_matrix((vals, (rows, cols)), shape=(3 * N, 3 * N))


def system(mesh, h):
    """(A restricted to the unpinned DOFs, preconditioner function, unpinned DOF indices)."""
    K = stiffness(mesh)
    A = sp.diags(mesh.mass) + h * h * K
    free = np.setdiff1d(np.arange(3 * mesh.N), np.asarray(mesh.pinnedDOFs, np.int64) - 1)
    Af = A[free][:, free].tocsr()
    # 3x3 block-Jacobi on the free DOFs of every vertex
    blocks = {}
    for k, dof in enumerate(free):
        blocks.setdefault(dof // 3, []).append(k)
    P = sp.lil_matrix(Af.shape)
    Ad = Af.toarray() if Af.shape[0] < 4000 else None
    for v, ks in blocks.items():
        sub = (Ad[np.ix_(ks, ks)] if Ad is not None else Af[ks][:, ks].toarray())
        inv = np.linalg.inv(sub)
        for i, ki in enumerate(ks):
            for j, kj in enumerate(ks):
                P[ki, kj] = inv[i, j]
    P = P.tocsr()
    return Af, (lambda r: P @ r), free


def solve_pcg(iterations, A, b, x0, preconditioner):
    """solvePCG.m: returns x and resvec (||A x - b|| after every iteration)."""
    x = np.array(x0, float)
    r = b - A @ x
    z = preconditioner(r)
    d = z.copy()
    rTz = r @ z
    resvec = np.zeros(iterations)
    for i in range(iterations):
        Ap = A @ d
        qAp = d @ Ap
        alpha = 0.0 if qAp == 0 else rTz / (d @ Ap)
        x = x + alpha * d
        r = r - alpha * Ap
        z = preconditioner(r)
        rTznew = r @ z
        beta = rTznew / rTz
        rTz = rTznew
        d = z + beta * d
        resvec[i] = np.linalg.norm(A @ x - b)
    return x, resvec
