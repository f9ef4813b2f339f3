"""Host-side mirror of the reference's tet-mesh precompute (``Mesh3D``).

Builds, with numpy, exactly the arrays ``xpbdLayer3D.layerSolve`` consumes
(3d/@Mesh3D/Mesh3D.m:123-298 and :408-461): positions in MATLAB's interleaved
layout, 1-based tets, greedy colours (through the native colouring of the C
ABI), DmInv pages, signed volumes, lumped masses and the per-tet compliance
blocks, plus ``pin`` (3d/@Mesh3D/pin.m:1-39).  Array memory layouts match the
MATLAB arrays so they can be handed to the C ABI as they are:
  t        (T, 4)  int32, column-major (Fortran) -- Mesh3D.t
  DmInv    (T, 9)  float64, row e = page e in column-major order
  alpha    (T, 36) float64, row e = 6x6 page e in column-major order
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, i32, load


def to_lame(nu, E):
    """util/toLame.m:1-6 (argument order nu, E as in the reference)."""
    nu = np.asarray(nu, dtype=np.float64)
    E = np.asarray(E, dtype=np.float64)
    return E / (2 * (1 + nu)), (E * nu) / ((1 + nu) * (1 - 2 * nu))


_COLORING = None


def use_coloring(fn):
    """Replace the colouring used by Mesh3D (fn(t, N) -> (colours, count));
    None restores the native one.  A CPU-only caller that must not load the
    native library passes its own first-fit colouring here."""
    global _COLORING
    _COLORING = fn


def greedy_coloring(t: np.ndarray, N: int):
    """naiveGraphColoring via the native first-fit colouring (1-based colours)."""
    if _COLORING is not None:
        col, nc = _COLORING(t, N)
        return np.ascontiguousarray(col, np.int32), int(nc)
    lib = load()
    tf = np.asfortranarray(t, dtype=np.int32)
    T = tf.shape[0]
    color = np.zeros(T, dtype=np.int32)
    nc = C.c_int32(0)
    check("mlx_greedy_coloring", lib.mlx_greedy_coloring(i32(tf), T, N, i32(color), C.byref(nc)))
    return color, int(nc.value)


def rest_state(p: np.ndarray, t: np.ndarray):
    """DmInv = inv([p1-p0, p2-p0, p3-p0]) (computeB3D.m:23-24) and the signed
    volume det(Dm)/6 (makeElements3D.m:11)."""
    V = p.reshape(-1, 3)
    ids = np.asarray(t, dtype=np.int64) - 1
    Dm = np.stack([V[ids[:, 1]] - V[ids[:, 0]], V[ids[:, 2]] - V[ids[:, 0]], V[ids[:, 3]] - V[ids[:, 0]]],
                  axis=2)  # (T, 3 rows, 3 cols): column k = p_{k+1} - p0
    DmInv = np.linalg.inv(Dm)
    vol = np.linalg.det(Dm) / 6.0
    # page e in column-major order: entry (r, c) at r + 3c
    return np.ascontiguousarray(DmInv.transpose(0, 2, 1).reshape(-1, 9)), vol


def material_blocks(mu, lam, alpha1):
    """Mesh3D.updateMaterials compliance (Mesh3D.m:445-460): K = [lam+4mu lam
    lam; ...] (+) 2mu I, alpha = inv(K), alphaInv = K, beta = alpha1 K."""
    T = mu.shape[0]
    K = np.zeros((T, 6, 6))
    diag_mu = 2 * mu
    diag_val = lam + 2 * diag_mu
    for r in range(3):
        for c in range(3):
            K[:, r, c] = diag_val if r == c else lam
    for r in range(3, 6):
        K[:, r, r] = diag_mu
    alpha = np.linalg.inv(K)
    beta = K * alpha1[:, None, None]
    cm = lambda a: np.ascontiguousarray(a.transpose(0, 2, 1).reshape(T, 36))
    return cm(alpha), cm(K), cm(beta)


@dataclass
class Mesh3D:
    """The simulation state and precompute of one tet mesh."""

    p: np.ndarray                 # 3N positions, [x1 y1 z1 x2 ...]
    t: np.ndarray                 # (T, 4) int32, 1-based, Fortran order
    mu: np.ndarray                # (T,) Lame mu
    lam: np.ndarray               # (T,) Lame lambda
    rho: np.ndarray               # (T,) density
    alpha1: np.ndarray            # (T,) Rayleigh stiffness factor
    energy_type: int = _lib.MLX_ENERGY_STVK_VOIGT
    v: np.ndarray = None
    f: np.ndarray = None
    N: int = 0
    T: int = 0
    elementColor: np.ndarray = None
    numColors: int = 0
    DmInv: np.ndarray = None
    elV: np.ndarray = None
    mass: np.ndarray = None
    pinnedInds: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    pinnedDOFs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    unpinnedDOFs: np.ndarray = None
    pinnedTets: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    @classmethod
    def from_arrays(cls, V, T, mu, lam, rho=1000.0, alpha1=0.0,
                    energy_type=_lib.MLX_ENERGY_STVK_VOIGT) -> "Mesh3D":
        V = np.asarray(V, dtype=np.float64)
        T = np.asfortranarray(np.asarray(T, dtype=np.int32))
        nt = T.shape[0]
        bc = lambda x: np.broadcast_to(np.asarray(x, dtype=np.float64), (nt,)).copy()
        m = cls(p=np.ascontiguousarray(V.reshape(-1)), t=T, mu=bc(mu), lam=bc(lam), rho=bc(rho),
                alpha1=bc(alpha1), energy_type=energy_type)
        m._precompute()
        return m

    def _precompute(self):
        self.N = self.p.size // 3
        self.T = self.t.shape[0]
        self.v = np.zeros(3 * self.N)
        self.f = np.zeros(3 * self.N)
        self.elementColor, self.numColors = greedy_coloring(self.t, self.N)
        self.DmInv, self.elV = rest_state(self.p, self.t)
        if np.any(self.elV <= 0):
            raise ValueError("tets must be positively oriented (det(Dm) > 0)")
        # computeMass density branch (computeMass.m:20-37): vol*rho/4 per corner
        m = np.zeros(self.N)
        # tet-major accumulation order, as the reference's loop over tets
        np.add.at(m, (np.asarray(self.t, np.int64) - 1).reshape(-1, order="C"),
                  np.repeat(self.elV * self.rho / 4.0, 4))
        self.mass = np.repeat(m, 3)
        self._blocks = None
        self.unpinnedDOFs = np.arange(1, 3 * self.N + 1, dtype=np.int32)

    # The 6x6 compliance pages (Mesh3D.updateMaterials) are formed on first
    # use: a Neo-Hookean mesh never needs them, and for a few million tets
    # they take gigabytes.
    def _material_blocks(self):
        if self._blocks is None:
            self._blocks = material_blocks(self.mu, self.lam, self.alpha1)
        return self._blocks

    @property
    def perElementXPBDalphaMatrix(self):
        return self._material_blocks()[0]

    @property
    def perElementXPBDalphaInvMatrix(self):
        return self._material_blocks()[1]

    @property
    def perElementXPBDbeta(self):
        return self._material_blocks()[2]

    def pin(self, pinned_inds):
        """Mesh3D.pin (pin.m:1-39): pinned DOFs sorted, pinned tets = tets with
        at least one pinned vertex."""
        ids = np.concatenate([self.pinnedInds, np.asarray(pinned_inds, dtype=np.int32).ravel()])
        self.pinnedInds = ids.astype(np.int32)
        dofs = np.sort(np.concatenate([ids * 3 - 2, ids * 3 - 1, ids * 3])).astype(np.int32)
        self.pinnedDOFs = dofs
        pinned = np.zeros(self.N + 1, dtype=bool)
        pinned[ids] = True
        self.pinnedTets = (np.nonzero(pinned[self.t].any(axis=1))[0] + 1).astype(np.int32)
        self.unpinnedDOFs = np.setdiff1d(np.arange(1, 3 * self.N + 1), dofs).astype(np.int32)

    @property
    def elementDOFs(self):
        tt = np.asarray(self.t, np.int64)
        return np.stack([tt[:, k] * 3 - 2 + d for k in range(4) for d in range(3)], axis=1).astype(np.int32)

    def bbox_diagonal(self) -> float:
        V = self.p.reshape(-1, 3)
        return float(np.linalg.norm(V.max(0) - V.min(0)))


def merge_meshes(meshes) -> "Mesh3D":
    """Mesh3D.mergeMesh (3d/@Mesh3D/Mesh3D.m:300-338) applied in order: the
    vertices, tets (offset by the vertices before them), materials and pins
    are concatenated and the colours of the parts are overlaid (colour c of
    every part is one colour of the result, numColors = max).  First-fit
    colouring of the merged mesh gives exactly that overlay, because parts
    share no vertex; it is checked here."""
    meshes = list(meshes)
    first = meshes[0]
    offs = np.cumsum([0] + [m.N for m in meshes])
    V = np.concatenate([m.p.reshape(-1, 3) for m in meshes])
    T = np.concatenate([np.asarray(m.t, np.int64) + o for m, o in zip(meshes, offs[:-1])]).astype(np.int32)
    cat = lambda name: np.concatenate([getattr(m, name) for m in meshes])
    out = Mesh3D.from_arrays(V, T, cat("mu"), cat("lam"), rho=cat("rho"), alpha1=cat("alpha1"),
                             energy_type=first.energy_type)
    overlay = cat("elementColor")
    if not np.array_equal(out.elementColor, overlay):
        raise AssertionError("merged colouring differs from the overlay of the parts' colourings")
    pins = [m.pinnedInds.astype(np.int64) + o for m, o in zip(meshes, offs[:-1]) if m.pinnedInds.size]
    if pins:
        out.pin(np.concatenate(pins).astype(np.int32))
    out.v = cat("v")
    out.f = cat("f")
    out.part_vertex_offsets = offs
    out.part_tet_offsets = np.cumsum([0] + [m.T for m in meshes])
    return out
