"""The native per-step vector arithmetic of xpbdLayer3D.integrate
(mlx_any_nan, mlx_integrate_begin, mlx_integrate_end; no GPU) against the
reference's element-wise expressions (xpbdLayer3D.m:629, 638-643, 662-664,
737) restated in numpy: the same doubles, on a mesh below and above the
size at which the library splits the pass over threads."""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib
from multilayersolver2024_b200._lib import f64, i32


def _reference(h, g, drag, cf, mass, v, unpinned):
    f = np.zeros(mass.size)
    f[2::3] = f[2::3] + mass[2::3] * g
    f = f + cf
    resv = v.copy()
    u = unpinned - 1
    resv[u] = resv[u] + h * f[u] / mass[u]
    return f, (1 - drag) * resv


@pytest.mark.parametrize("n", [81, 400_000])
@pytest.mark.parametrize("vector_force", [False, True])
def test_begin_and_end_equal_the_reference_expressions(lib, n, vector_force):
    rng = np.random.default_rng(n + vector_force)
    n3 = 3 * n
    mass = np.repeat(rng.uniform(0.1, 2.0, n), 3)
    v = rng.normal(0, 1, n3)
    pinned = np.sort(rng.choice(n3, n3 // 10, replace=False)).astype(np.int32) + 1
    unpinned = np.setdiff1d(np.arange(1, n3 + 1), pinned).astype(np.int32)
    h, g, drag = 1.0 / 60.0, -9.81, 0.01
    cf = rng.normal(0, 1, n3) if vector_force else 0.25
    f_ref, r_ref = _reference(h, g, drag, cf, mass, v, unpinned)
    f, r = np.empty(n3), np.empty(n3)
    rc = lib.mlx_integrate_begin(n3, h, g, drag, 0.0 if vector_force else cf,
                                 f64(cf) if vector_force else None, f64(mass), f64(v), i32(pinned), pinned.size,
                                 f64(f), f64(r))
    assert rc == _lib.MLX_OK
    np.testing.assert_array_equal(f, f_ref)
    np.testing.assert_array_equal(r, r_ref)
    xi, oldp = rng.normal(0, 1, n3), rng.normal(0, 1, n3)
    out = np.empty(n3)
    assert lib.mlx_integrate_end(n3, h, f64(xi), f64(oldp), f64(out)) == _lib.MLX_OK
    np.testing.assert_array_equal(out, (xi - oldp) / h)


@pytest.mark.parametrize("n", [10, 1_000_000])
def test_any_nan(lib, n):
    x = np.random.default_rng(0).normal(0, 1, n)
    assert lib.mlx_any_nan(n, f64(x)) == 0
    for at in (0, n // 2, n - 1):
        y = x.copy()
        y[at] = np.nan
        assert lib.mlx_any_nan(n, f64(y)) == 1
    assert lib.mlx_any_nan(0, None) == 0


def test_argument_errors(lib):
    n3 = 9
    a = np.ones(n3)
    bad = np.array([0], np.int32)
    assert lib.mlx_integrate_begin(n3, 0.01, -9.8, 0.0, 0.0, None, f64(a), f64(a), i32(bad), 1,
                                   f64(np.empty(n3)), f64(np.empty(n3))) == _lib.MLX_ERR_ARGUMENT
    assert b"out of range" in lib.mlx_last_error()
    assert lib.mlx_integrate_begin(8, 0.01, -9.8, 0.0, 0.0, None, f64(a), f64(a), None, 0,
                                   f64(np.empty(n3)), f64(np.empty(n3))) == _lib.MLX_ERR_ARGUMENT
    assert lib.mlx_integrate_begin(n3, 0.01, -9.8, 0.0, 0.0, None, None, f64(a), None, 0,
                                   f64(np.empty(n3)), f64(np.empty(n3))) == _lib.MLX_ERR_ARGUMENT
    assert lib.mlx_integrate_end(n3, 0.01, None, f64(a), f64(np.empty(n3))) == _lib.MLX_ERR_ARGUMENT
    assert lib.mlx_any_nan(3, None) == -_lib.MLX_ERR_ARGUMENT
