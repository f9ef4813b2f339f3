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


def _cvu_reference(normals, ids, v, h, gravity, dim, restitution):
    """contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603) restated in
    numpy: gather, threshold, normal response, last write wins."""
    K = normals.shape[0]
    e = np.full(K, restitution)
    rows = ids.astype(np.int64) - 1
    vn = v.reshape(-1, dim)[rows]
    e[np.linalg.norm(vn, axis=1) <= 2 * gravity * h] = 0
    vt = np.sum(normals * vn, axis=1)
    dv = normals * (-vn + np.minimum(-e * vt, 0)[:, None])
    out = v.copy()
    for k in range(K):  # explicit contact order: a repeated vertex keeps its last contact
        out.reshape(-1, dim)[rows[k]] = vn[k] + dv[k]
    return out


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("gravity", [-9.81, 9.81])
def test_contact_velocity_update_equals_the_reference_expressions(lib, dim, gravity):
    rng = np.random.default_rng(dim)
    nv, K = 500, 700  # more contacts than vertices: repeated vertices
    v = rng.normal(0, 0.5, dim * nv)
    ids = rng.integers(1, nv + 1, K).astype(np.int32)
    n = rng.normal(0, 1, (K, dim))
    n /= np.linalg.norm(n, axis=1)[:, None]
    h, e = 1.0 / 60.0, 1e-2
    ref = _cvu_reference(n, ids, v, h, gravity, dim, e)
    nf = np.asfortranarray(n)
    out = np.empty_like(v)
    assert lib.mlx_contact_velocity_update(K, f64(nf), i32(ids), dim, v.size, f64(v), h, gravity, e,
                                           f64(out)) == _lib.MLX_OK
    np.testing.assert_array_equal(out, ref)
    w = v.copy()  # in place
    assert lib.mlx_contact_velocity_update(K, f64(nf), i32(ids), dim, w.size, f64(w), h, gravity, e,
                                           f64(w)) == _lib.MLX_OK
    np.testing.assert_array_equal(w, ref)
    from multilayersolver2024_b200.xpbd_layer3d import contact_velocity_update
    np.testing.assert_array_equal(contact_velocity_update(n, ids, v, h, gravity, dim, e), ref)


def test_contact_velocity_update_matches_the_oracle(lib, oracle):
    rng = np.random.default_rng(5)
    nv, K = 300, 400
    v = rng.normal(0, 0.5, 3 * nv)
    ids = rng.integers(1, nv + 1, K).astype(np.int32)
    n = rng.normal(0, 1, (K, 3))
    n /= np.linalg.norm(n, axis=1)[:, None]
    from multilayersolver2024_b200.xpbd_layer3d import contact_velocity_update
    got = contact_velocity_update(n, ids, v, 1 / 120, -9.81, 3, 1e-2)
    ref = oracle.contact_velocity_update(n, ids, v.copy(), 1 / 120, -9.81, 1e-2)
    np.testing.assert_array_equal(got, ref)


def test_contact_velocity_update_errors(lib):
    v = np.zeros(9)
    n = np.asfortranarray(np.ones((1, 3)))
    assert lib.mlx_contact_velocity_update(1, f64(n), i32(np.array([4], np.int32)), 3, 9, f64(v), 0.01, -9.8, 0.0,
                                           f64(v)) == _lib.MLX_ERR_ARGUMENT
    assert lib.mlx_contact_velocity_update(1, f64(n), i32(np.array([1], np.int32)), 4, 9, f64(v), 0.01, -9.8, 0.0,
                                           f64(v)) == _lib.MLX_ERR_ARGUMENT
    assert lib.mlx_contact_velocity_update(0, None, None, 3, 9, f64(v), 0.01, -9.8, 0.0, f64(v)) == _lib.MLX_OK
