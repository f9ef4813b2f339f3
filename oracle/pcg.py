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


def nh_linearized_step(mesh, x, h, lam_c, free):
    """The XPBD layer step of a Neo-Hookean mesh linearised at x (test
    infrastructure: the predictor experiment).  With J the Jacobian of the
    per-tet constraints C = (C_D, C_H) = (sqrt(B), det F - 1) (the pair the
    library projects), W = alpha~^-1 = diag(h^2 vol mu, h^2 vol (lambda - mu))
    and lam_c (2T) the multipliers the layer starts from, the linear system
        [M  -J^T] [dx]   [0            ]
        [J  W^-1] [dl] = [-C - W^-1 lam_c]
    reduces to (M + J^T W J) dx = -J^T (W C + lam_c) on the free DOFs, and the
    multipliers become lam = -W (C + J dx).  Returns (A_free, b_free,
    preconditioner, J, W, C): the system, its 3x3 block-Jacobi
    preconditioner, and the pieces that give lam."""
    t = np.asarray(mesh.t, np.int64) - 1
    nt, N = t.shape[0], mesh.N
    X = np.asarray(x, float).reshape(-1, 3)
    Gm = np.asarray(mesh.DmInv, float).reshape(nt, 3, 3).transpose(0, 2, 1)  # Gm[e, r, c] = DmInv(r, c)
    Ds = np.stack([X[t[:, k]] - X[t[:, 0]] for k in (1, 2, 3)], 2)
    F = Ds @ Gm
    f0, f1, f2 = F[:, :, 0], F[:, :, 1], F[:, :, 2]
    cf = np.stack([np.cross(f1, f2), np.cross(f2, f0), np.cross(f0, f1)], 2)
    Jd = np.einsum("ei,ei->e", f0, cf[:, :, 0])
    B = (F ** 2).sum((1, 2)) + Jd * Jd - 4 * Jd
    CD = np.sqrt(np.maximum(B, 0.0))
    mu, lam = np.asarray(mesh.mu, float), np.asarray(mesh.lam, float)
    hasH = lam > mu
    CH = np.where(hasH, Jd - 1.0, 0.0)
    dD = (F + (Jd - 2.0)[:, None, None] * cf) / np.where(CD > 1e-12, CD, np.inf)[:, None, None]
    dH = cf * hasH[:, None, None]

    def grad_x(dF):
        g = np.einsum("erc,ekc->ekr", dF, Gm)
        return np.concatenate([-g.sum(1, keepdims=True), g], 1)

    rows, cols, vals = [], [], []
    for q, g in enumerate((grad_x(dD), grad_x(dH))):
        for k in range(4):
            for d in range(3):
                rows.append(2 * np.arange(nt) + q)
                cols.append(3 * t[:, k] + d)
                vals.append(g[:, k, d])
    J = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(2 * nt, 3 * N))
    vol = np.asarray(mesh.elV, float)
    W = sp.diags(np.stack([h * h * vol * mu, np.where(hasH, h * h * vol * (lam - mu), 0.0)], 1).ravel())
    C = np.stack([CD, CH], 1).ravel()
    A = (sp.diags(np.asarray(mesh.mass, float)) + J.T @ W @ J).tocsr()[free][:, free].tocsr()
    b = -(J.T @ (W @ C + np.asarray(lam_c, float)))[free]
    # 3x3 block-Jacobi on the free DOFs of every vertex
    blocks = {}
    for k, dof in enumerate(free):
        blocks.setdefault(int(dof) // 3, []).append(k)
    P = sp.lil_matrix(A.shape)
    for ks in blocks.values():
        inv = np.linalg.inv(A[ks][:, ks].toarray())
        for i, ki in enumerate(ks):
            for j, kj in enumerate(ks):
                P[ki, kj] = inv[i, j]
    P = P.tocsr()
    return A, b, (lambda r: P @ r), J, W, C
