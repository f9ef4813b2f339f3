"""ctypes binding of the C ABI declared in include/mlxpbd.h.

The structs below are field-for-field copies of the header's; arrays are passed
as numpy buffers that must stay alive for the duration of the call.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libmlxpbd.so"

MLX_OK = 0
MLX_ERR_ARGUMENT = 1
MLX_ERR_UNSUPPORTED = 2
MLX_ERR_NO_DEVICE = 4
MLX_NOALLOC_MAX_TETS = 524288
MLX_ENERGY_NEOHOOKEAN = 1
MLX_ENERGY_STVK_VOIGT = 2
MLX_FP32 = 0
MLX_FP64 = 1
MLX_OBSTACLE_PLANE = 1
MLX_OBSTACLE_SPHERE = 2
MLX_OBSTACLE_BOX = 3
MLX_MAX_OBSTACLES = 32
MLX_ERR_LIMIT = 6

_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class MeshDesc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_int32), ("num_tets", C.c_int32), ("t", _i32p),
        ("mass", _f64p), ("DmInv", _f64p), ("volume", _f64p),
        ("element_color", _i32p), ("num_colors", C.c_int32),
        ("pinned_dofs", _i32p), ("num_pinned_dofs", C.c_int32),
        ("energy_type", C.c_int32),
        ("alpha", _f64p), ("beta", _f64p), ("mu", _f64p), ("lambda_", _f64p), ("alpha1", _f64p),
        ("precision", C.c_int32), ("device", C.c_int32),
    ]


class LayerDesc(C.Structure):
    _fields_ = [
        ("num_layers", C.c_int32), ("num_columns", C.c_int32),
        ("layers_map", _i32p), ("iterations", _i32p),
        ("is_elastic_element", _u8p), ("is_rigid_element", _u8p),
        ("rigid_body_sets", _i32p), ("vertex_rigid_body", _i32p),
        ("is_boundary_vertex", _u8p), ("is_rigid_vertex", _u8p),
        ("num_rigids", _i32p),
    ]


class SolveParams(C.Structure):
    _fields_ = [
        ("h", C.c_double), ("boundary_compliance", C.c_double), ("contact_resistance", C.c_double),
        ("run_until", C.c_double), ("give_up_threshold", C.c_double),
        ("gravity_compliance", C.c_double), ("gravity", C.c_double),
        ("stop_at_improvement_percent", C.c_double),
        ("compute_residuals", C.c_int32), ("hanging_stop", C.c_int32),
        ("give_up_enabled", C.c_int32), ("last_layer_give_up_enabled", C.c_int32),
        ("use_gravity_constraints", C.c_int32), ("use_rigid_contacts", C.c_int32),
        ("contact_coloring", C.c_int32),
    ]


class Contacts(C.Structure):
    _fields_ = [
        ("num_contacts", C.c_int32), ("normals", _f64p), ("point_colliders", _f64p),
        ("vertex_ids", _i32p), ("compliance", _f64p),
    ]


class SolveInputs(C.Structure):
    _fields_ = [
        ("xi", _f64p), ("lambdai", _f64p), ("oldp", _f64p), ("old_oldp", _f64p), ("f", _f64p),
        ("residualv", _f64p), ("pinnedx", _f64p), ("residual_in", _f64p),
        ("residual_in_len", C.c_int32), ("sum_non_monitored_time", C.c_double),
    ]


class SolveOutputs(C.Structure):
    _fields_ = [
        ("xi", _f64p), ("lambdai", _f64p), ("residual", _f64p), ("residual_capacity", C.c_int32),
        ("residual_len", C.c_int32), ("run_until", C.c_double),
        ("sum_non_monitored_time", C.c_double), ("total_iterations", C.c_int32),
    ]


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"], "array must be contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def f32(a):
    return ptr(a, C.c_float)


def f64(a):
    return ptr(a, C.c_double)


def i32(a):
    return ptr(a, C.c_int32)


def u8(a):
    return ptr(a, C.c_uint8)


class mlx_obstacle(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("normal", C.c_double * 3),
        ("center", C.c_double * 3),
        ("radius", C.c_double),
        ("rotation", C.c_double * 9),
        ("scale", C.c_double * 3),
        ("compliance", C.c_double),
    ]


SIGNATURES = {
    "mlx_last_error": ([], C.c_char_p),
    "mlx_abi_version": ([], C.c_int),
    "mlx_device_count": ([], C.c_int),
    "mlx_create": ([C.POINTER(MeshDesc), C.POINTER(C.c_void_p)], C.c_int),
    "mlx_destroy": ([C.c_void_p], C.c_int),
    "mlx_layer_solve": ([C.c_void_p, C.POINTER(LayerDesc), C.POINTER(SolveParams), C.POINTER(Contacts),
                         C.POINTER(SolveInputs), C.POINTER(SolveOutputs)], C.c_int),
    "mlx_sim_init": ([C.c_void_p, C.POINTER(LayerDesc), C.POINTER(SolveParams), _f64p, _f64p, C.c_double],
                     C.c_int),
    "mlx_sim_add_velocity": ([C.c_void_p, _i32p, _f64p, C.c_int32], C.c_int),
    "mlx_sim_step": ([C.c_void_p, C.c_int32, C.c_int32, _f64p], C.c_int),
    "mlx_sim_get_state": ([C.c_void_p, _f64p, _f64p], C.c_int),
    "mlx_sim_sweep_timing": ([C.c_void_p, C.c_int32], C.c_int),
    "mlx_sim_sweep_stats": ([C.c_void_p, _f64p, _f64p, C.POINTER(C.c_longlong), C.c_int32], C.c_int),
    "mlx_sim_launches_per_step": ([C.c_void_p], C.c_longlong),
    "mlx_last_call_launches": ([C.c_void_p], C.c_longlong),
    "mlx_launch_path": ([C.c_void_p, C.c_char_p, C.c_int32], C.c_int),
    "mlx_sim_autotune": ([C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "mlx_find_contacts": ([C.c_void_p, C.c_void_p, C.c_int32, _f64p, C.c_int32, _i32p, _f64p, _f64p, _f64p, _i32p],
                          C.c_int),
    "mlx_sim_set_obstacles": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_double], C.c_int),
    "mlx_sim_contact_count": ([C.c_void_p, _i32p], C.c_int),
    "mlx_sim_monitor": ([C.c_void_p, _f64p, C.c_int32, _i32p, _i32p, _f64p, _i32p], C.c_int),
    "mlx_sim_warm_start": ([C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_double, _f32p, _f32p, _f32p, _f32p,
                            _f32p, _i32p],
                           C.c_int),
    "mlx_sim_warm_start_fetch": ([C.c_void_p, _f32p, _f32p, C.c_int32, _i32p, _i32p], C.c_int),
    "mlx_sim_multiplier_warm_start": ([C.c_void_p, C.c_int32, C.c_double, C.c_double], C.c_int),
    "mlx_layer_pcg": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "mlx_pcg_solve": ([C.c_void_p, C.c_double, _f64p, C.c_int32, _f64p, _f64p], C.c_int),
    "mlx_wait_probe": ([C.c_int32, C.c_int32, C.c_int64, C.POINTER(C.c_int32)], C.c_int),
    "mlx_build_layers": ([C.c_void_p, _f64p, _f64p, C.c_double, C.c_int32, _i32p, _f64p, _f64p, C.c_int32, _u8p,
                          _i32p, _i32p, _u8p, _u8p, _u8p, _i32p], C.c_int),
    "mlx_mlp_create": ([C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                        C.POINTER(C.c_void_p)], C.c_int),
    "mlx_mlp_destroy": ([C.c_void_p], C.c_int),
    "mlx_mlp_num_params": ([C.c_void_p], C.c_longlong),
    "mlx_mlp_set_params": ([C.c_void_p, _f32p, C.c_longlong], C.c_int),
    "mlx_mlp_get_params": ([C.c_void_p, _f32p, C.c_longlong], C.c_int),
    "mlx_mlp_forward": ([C.c_void_p, _f32p, C.c_int32, _f32p], C.c_int),
    "mlx_mlp_loss_grad": ([C.c_void_p, _f32p, _f32p, C.c_int32, _f32p, _f32p], C.c_int),
    "mlx_mlp_train": ([C.c_void_p, _f32p, _f32p, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _f32p],
                      C.c_int),
    "mlx_stvk_residual_noalloc": ([C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p], C.c_int),
    "mlx_greedy_coloring": ([_i32p, C.c_int32, C.c_int32, _i32p, _i32p], C.c_int),
    "mlx_strain_rate_norms": ([_i32p, C.c_int32, _f64p, _f64p, _f64p, C.c_double, _f64p], C.c_int),
    "mlx_union_find_layers": ([_i32p, C.c_int32, _f64p, C.c_int32, _u8p, _i32p, C.c_int32, _i32p, _i32p],
                              C.c_int),
    "mlx_find_boundary_vertices": ([_i32p, C.c_int32, C.c_int32, _i32p, C.c_int32, _u8p, _u8p, _u8p, _i32p],
                                   C.c_int),
    "mlx_any_nan": ([C.c_int64, _f64p], C.c_int32),
    "mlx_integrate_begin": ([C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, _f64p, _f64p, _f64p, _i32p,
                             C.c_int32, _f64p, _f64p], C.c_int),
    "mlx_integrate_end": ([C.c_int32, C.c_double, _f64p, _f64p, _f64p], C.c_int),
    "mlx_contact_velocity_update": ([C.c_int32, _f64p, _i32p, C.c_int32, C.c_int64, _f64p, C.c_double, C.c_double,
                                     C.c_double, _f64p], C.c_int),
}

_lib = None


class MlxError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def load(path: Path | None = None):
    """Load libmlxpbd.so; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m multilayersolver2024_b200.build` "
                          "(the package has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def check(fn_name, rc, lib=None):
    if rc != MLX_OK:
        lib = lib or load()
        raise MlxError(fn_name, rc, lib.mlx_last_error().decode(errors="replace"))
