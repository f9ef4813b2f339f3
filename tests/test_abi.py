"""The C ABI library loads and exports every entry point include/*.h declares
(no compute call: this runs without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(mlx_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["mlx_create", "mlx_destroy", "mlx_layer_solve", "mlx_last_error", "mlx_greedy_coloring",
                 "mlx_union_find_layers", "mlx_strain_rate_norms", "mlx_find_boundary_vertices", "mlx_sim_step"]:
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.mlx_abi_version() == 1


def test_create_without_device_fails_cleanly(lib):
    """On a host without a B200 the solver refuses with a status, never a crash."""
    if lib.mlx_device_count() > 0:
        pytest.skip("a device is present")
    from multilayersolver2024_b200 import _lib
    from multilayersolver2024_b200.mesh3d import Mesh3D
    from multilayersolver2024_b200 import scenes
    from multilayersolver2024_b200.xpbd_layer3d import mesh_desc
    sc = scenes.config1()
    d, keep = mesh_desc(sc.mesh)
    h = C.c_void_p()
    rc = lib.mlx_create(C.byref(d), C.byref(h))
    assert rc == _lib.MLX_ERR_NO_DEVICE and not h.value
    assert b"device" in lib.mlx_last_error()
