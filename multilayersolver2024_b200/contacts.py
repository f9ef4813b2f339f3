"""Analytic contact finders (the reference's 3d/contact classes) on the device.

``PlaneContactFinder3D``, ``SphereContactFinder`` and
``PlatformContactDetector`` keep the reference constructors' arguments
(3d/contact/PlaneContactFinder3D.m:16-32, SphereContactFinder.m:13-21,
PlatformContactDetector.m:22-63); ``find_contacts`` runs simulate3D's finder
loop (3d/simulate3D.m:156-171) on the GPU through ``mlx_find_contacts`` and
returns the concatenated contact list as a ``ContactSet``.  A ``ResidentSim``
takes the same finders (``ResidentSim.set_obstacles``) and detects contacts on
the device every step.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, f64, i32


def rotation_matrix_degrees(degrees):
    """RotationMatrixDegrees (3d/tools/math/RotationMatrixDegrees.m):
    eul2rotm(deg2rad(degrees), 'XYZ') = Rx(a) Ry(b) Rz(c)."""
    a, b, c = np.deg2rad(np.asarray(degrees, dtype=np.float64))
    Rx = np.array([[1, 0, 0], [0, np.cos(a), -np.sin(a)], [0, np.sin(a), np.cos(a)]])
    Ry = np.array([[np.cos(b), 0, np.sin(b)], [0, 1, 0], [-np.sin(b), 0, np.cos(b)]])
    Rz = np.array([[np.cos(c), -np.sin(c), 0], [np.sin(c), np.cos(c), 0], [0, 0, 1]])
    return Rx @ Ry @ Rz


@dataclass
class Finder:
    kind: int
    normal: np.ndarray = field(default_factory=lambda: np.zeros(3))
    center: np.ndarray = field(default_factory=lambda: np.zeros(3))
    radius: float = 0.0
    rotation: np.ndarray = field(default_factory=lambda: np.eye(3))
    scale: np.ndarray = field(default_factory=lambda: np.zeros(3))
    compliance: float = 1e-4  # ContactFinder.xpbdContactCompliance default

    def to_c(self) -> _lib.mlx_obstacle:
        o = _lib.mlx_obstacle()
        o.type = self.kind
        o.normal[:] = [float(x) for x in np.asarray(self.normal, float)]
        o.center[:] = [float(x) for x in np.asarray(self.center, float)]
        o.radius = float(self.radius)
        o.rotation[:] = [float(x) for x in np.asarray(self.rotation, float).reshape(9)]
        o.scale[:] = [float(x) for x in np.asarray(self.scale, float)]
        o.compliance = float(self.compliance)
        return o


def PlaneContactFinder3D(normal, position, compliance=1e-4) -> Finder:
    return Finder(_lib.MLX_OBSTACLE_PLANE, normal=np.asarray(normal, float), center=np.asarray(position, float),
                  compliance=compliance)


def SphereContactFinder(radius, position) -> Finder:
    return Finder(_lib.MLX_OBSTACLE_SPHERE, radius=float(radius), center=np.asarray(position, float))


def PlatformContactDetector(degrees, scale, position, compliance=1e-4) -> Finder:
    return Finder(_lib.MLX_OBSTACLE_BOX, rotation=rotation_matrix_degrees(degrees), scale=np.asarray(scale, float),
                  center=np.asarray(position, float), compliance=compliance)


def pack_finders(finders):
    finders = list(finders)
    if len(finders) > _lib.MLX_MAX_OBSTACLES:
        raise ValueError(f"at most {_lib.MLX_MAX_OBSTACLES} finders")
    arr = (_lib.mlx_obstacle * max(len(finders), 1))()
    for k, f in enumerate(finders):
        arr[k] = f.to_c()
    return arr, len(finders)


def find_contacts(solver, finders, p):
    """simulate3D's contact loop on the device: the finders' contact lists
    concatenated in order (``mlx_find_contacts``)."""
    from .xpbd_layer3d import ContactSet
    lib = solver._lib
    arr, n = pack_finders(finders)
    p = np.ascontiguousarray(p, dtype=np.float64)
    N = p.size // 3
    cap = max(N * n, 1)
    # only the first K rows (3K values) are written and read
    ids = np.empty(cap, np.int32)
    nrm = np.empty(3 * cap)
    pts = np.empty(3 * cap)
    comp = np.empty(cap)
    K = C.c_int32(0)
    check("mlx_find_contacts", lib.mlx_find_contacts(solver.handle, C.cast(arr, C.c_void_p), n, f64(p), cap, i32(ids),
                                                     f64(nrm), f64(pts), f64(comp), C.byref(K)), lib)
    k = K.value
    # K x 3 column-major views of the written rows, the layout layerSolve takes
    return ContactSet(nrm[:3 * k].reshape(3, k).T, pts[:3 * k].reshape(3, k).T, ids[:k], comp[:k])
