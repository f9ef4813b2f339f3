"""Tet-mesh files of the reference's assets: TetGen ``.node`` / ``.ele`` (read
by polyLoader.m through gptoolbox's readNODE / readELE) and Medit ``.mesh``
(meshLoader.m through readMESH).

``.node``: a header ``<points> <dim> <attributes> <boundary marker flag>``,
then ``<index> <x> <y> <z> [attributes] [marker]`` per point.  ``.ele``: a
header ``<tets> <nodes per tet> <attributes>``, then ``<index> <n1> ... <nk>
[attributes]`` per tet; the node numbers follow the ``.node`` file's first
index (0 or 1).  ``#`` starts a comment.  ``.mesh``: keyword sections
(``Vertices``, ``Tetrahedra``, ``Triangles``, ...) each followed by a count
and one entity per line, the last value of an entity being its reference
label.

The loaders return 1-based tets as the reference's Mesh3D holds them.  The
solver needs det(Dm) > 0; with ``orient=True`` (default) tets of the other
orientation get their last two corners swapped, which is the same tet.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import _lib
from .mesh3d import Mesh3D


def _rows(path):
    for line in Path(path).read_text().splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            yield line.split()


def read_node(path):
    """(V (n x 3), attributes (n x a), markers (n,) or None, first index)."""
    rows = _rows(path)
    head = next(rows)
    n, dim, na, nb = (int(x) for x in (head + ["0", "0", "0"])[:4])
    if dim != 3:
        raise ValueError(f"{path}: {dim}-dimensional points")
    V = np.zeros((n, 3))
    A = np.zeros((n, na))
    B = np.zeros(n, np.int32) if nb else None
    first = None
    for k in range(n):
        r = next(rows)
        if first is None:
            first = int(r[0])
        V[k] = [float(x) for x in r[1:4]]
        if na:
            A[k] = [float(x) for x in r[4:4 + na]]
        if nb:
            B[k] = int(r[4 + na])
    return V, A, B, 0 if first is None else first


def read_ele(path, first_index=None):
    """(T (m x 4), 1-based, attributes (m x a)).  `first_index` is the node
    numbering base (the .node file's first index); by default the smallest
    node number in the file."""
    rows = _rows(path)
    head = next(rows)
    m, npt, na = (int(x) for x in (head + ["0", "0"])[:3])
    if npt not in (4, 10):
        raise ValueError(f"{path}: {npt} nodes per tet")
    T = np.zeros((m, 4), np.int64)
    A = np.zeros((m, na))
    for k in range(m):
        r = next(rows)
        T[k] = [int(x) for x in r[1:5]]  # corners; quadratic tets keep their 4 vertices
        if na:
            A[k] = [float(x) for x in r[1 + npt:1 + npt + na]]
    base = int(T.min()) if first_index is None and m else (first_index or 0)
    return (T - base + 1).astype(np.int32), A


def read_mesh(path):
    """Medit .mesh: (V (n x 3), T (m x 4) 1-based, tet labels (m,),
    triangles (k x 3) 1-based)."""
    toks = []
    for line in Path(path).read_text().splitlines():
        line = line.split("#", 1)[0].strip()
        if line:
            toks.extend(line.split())
    i, V, T, TL, F = 0, np.zeros((0, 3)), np.zeros((0, 4), np.int32), np.zeros(0, np.int32), np.zeros((0, 3), np.int32)
    width = {"Vertices": 4, "Tetrahedra": 5, "Triangles": 4, "Edges": 3, "Corners": 1, "Ridges": 1,
             "RequiredVertices": 1, "Quadrilaterals": 5, "Hexahedra": 9}
    while i < len(toks):
        kw = toks[i]
        i += 1
        if kw in ("MeshVersionFormatted", "Dimension"):
            i += 1
        elif kw == "End":
            break
        elif kw in width:
            n = int(toks[i])
            i += 1
            w = width[kw]
            block = np.array(toks[i:i + n * w], dtype=np.float64).reshape(n, w)
            i += n * w
            if kw == "Vertices":
                V = block[:, :3].copy()
            elif kw == "Tetrahedra":
                T, TL = block[:, :4].astype(np.int32), block[:, 4].astype(np.int32)
            elif kw == "Triangles":
                F = block[:, :3].astype(np.int32)
        else:
            raise ValueError(f"{path}: unknown keyword {kw!r}")
    return V, T, TL, F


def orient_tets(V, T):
    """Tets with det(Dm) < 0 get their last two corners swapped (1-based T)."""
    T = np.array(T, np.int32, copy=True)
    P = V[T - 1]
    D = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)
    neg = np.linalg.det(D) < 0
    T[neg, 2], T[neg, 3] = T[neg, 3].copy(), T[neg, 2].copy()
    return T


def _materials(attr, mu, lam):
    """Per-tet (mu, lam) from scalars or from per-attribute tables."""
    mu, lam = np.asarray(mu, np.float64), np.asarray(lam, np.float64)
    if mu.ndim == 0:
        return mu, lam
    idx = np.asarray(attr, np.int64).ravel()
    return mu[idx - idx.min()], lam[idx - idx.min()]


def load_poly(base, mu, lam, scale=(1.0, 1.0, 1.0), rho=1000.0, energy_type=_lib.MLX_ENERGY_STVK_VOIGT,
              orient=True) -> Mesh3D:
    """polyLoader.m:21-31: `base`.node / `base`.ele, coordinates scaled per
    axis.  mu / lam: scalars, or tables indexed by the .ele attribute."""
    V, _, _, first = read_node(f"{base}.node")
    T, A = read_ele(f"{base}.ele", first)
    V = V * np.asarray(scale, np.float64)[None, :]
    if orient:
        T = orient_tets(V, T)
    m_mu, m_lam = _materials(A[:, 0] if A.shape[1] else np.zeros(T.shape[0]), mu, lam)
    return Mesh3D.from_arrays(V, T, m_mu, m_lam, rho=rho, energy_type=energy_type)


def load_mesh(path, mu, lam, scale=(1.0, 1.0, 1.0), rho=1000.0, energy_type=_lib.MLX_ENERGY_STVK_VOIGT,
              orient=True) -> Mesh3D:
    """meshLoader.m:22-33: a Medit .mesh file, coordinates scaled per axis;
    mu / lam scalars or tables indexed by the tets' reference labels."""
    V, T, TL, _ = read_mesh(path)
    V = V * np.asarray(scale, np.float64)[None, :]
    if orient:
        T = orient_tets(V, T)
    m_mu, m_lam = _materials(TL, mu, lam)
    return Mesh3D.from_arrays(V, T, m_mu, m_lam, rho=rho, energy_type=energy_type)


def write_node(path, V, first_index=0):
    lines = [f"{len(V)} 3 0 0"] + [f"{k + first_index} {float(x)!r} {float(y)!r} {float(z)!r}"
                                   for k, (x, y, z) in enumerate(V)]
    Path(path).write_text("\n".join(lines) + "\n")


def write_ele(path, T, first_index=0):
    """T 1-based; written with node numbers starting at `first_index`."""
    T = np.asarray(T, np.int64) - 1 + first_index
    lines = [f"{len(T)} 4 0"] + [f"{k + first_index} " + " ".join(str(int(v)) for v in t) for k, t in enumerate(T)]
    Path(path).write_text("\n".join(lines) + "\n")
