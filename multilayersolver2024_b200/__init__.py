"""B200-native multi-layer XPBD step (drop-in for xpbdLayer3D.layerSolve).

The compute path is the native library ``libmlxpbd.so`` (CUDA kernels for
sm_100a behind the C ABI of include/mlxpbd.h); this package holds the host-side
mirror of the reference's ``Mesh3D`` / ``xpbdLayer3D`` interface around it.
"""
from . import _lib
from ._lib import MLX_ENERGY_NEOHOOKEAN, MLX_ENERGY_STVK_VOIGT, MLX_FP32, MLX_FP64, MlxError, load
from .mesh3d import Mesh3D, to_lame
from .xpbd_layer3d import (ContactSet, LayerSet, Solver, StepCache, XpbdLayer3D, contact_velocity_update,
                           find_boundary_vertices, mesh_desc)

__all__ = ["Mesh3D", "XpbdLayer3D", "Solver", "StepCache", "ContactSet", "LayerSet", "to_lame", "load",
           "MlxError", "MLX_FP32", "MLX_FP64", "MLX_ENERGY_STVK_VOIGT", "MLX_ENERGY_NEOHOOKEAN",
           "contact_velocity_update", "find_boundary_vertices", "mesh_desc"]
