"""mlx_stvk_residual_noalloc: the residual for callers that cannot allocate.

Callers such as a MATLAB mexcuda function working on gpuArray memory, or a
fixed-rate loop that must not stall on cudaMalloc, own every device buffer;
this entry point reads their device arrays and writes one device double,
keeping its reduction scratch in a fixed array inside the library.  Its value
must equal the residual the regular entry point (mlx_layer_solve with
compute_residuals) reports for the same state, call after call, and the
calls must leave the device's free memory and torch's allocator unchanged.
This file is collected last so a failure here comes after every other test
has run.
"""
import ctypes as C

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib

from helpers import Case, block_mesh

pytestmark = pytest.mark.gpu


def _device(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _state(dims, seed):
    """One StVK layerSolve with residuals on: the mesh, the solve's final
    positions and multipliers, and the residual it reported."""
    m = block_mesh(dims=dims, seed=seed, alpha1=0.01)
    case = Case(m, [0], [1], seed=seed + 1)
    case.integ.computeResiduals = True
    case.integ.hangingStop = -1
    xi, _, residuals, _, lam, _ = case.product(_lib.MLX_FP64)
    assert residuals.size == 2 and residuals[-1] > 0
    return m, case, xi, lam, residuals[-1]


class _Call:
    """Device copies of one state and a call of the entry point on them."""

    def __init__(self, torch, lib, m, case, xi, lam, t=None):
        self.torch, self.lib, self.m, self.h = torch, lib, m, case.h
        t = np.asfortranarray(m.t) if t is None else t
        self.d = [_device(torch, xi, np.float64), _device(torch, np.asarray(t).ravel(order="F"), np.int32),
                  _device(torch, m.DmInv, np.float64), _device(torch, m.perElementXPBDalphaMatrix, np.float64),
                  _device(torch, np.asfortranarray(lam).ravel(order="F"), np.float64),
                  _device(torch, m.elV, np.float64)]
        self.out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()

    def __call__(self, num_tets=None):
        self.out.fill_(-1.0)
        rc = self.lib.mlx_stvk_residual_noalloc(self.m.N, self.m.T if num_tets is None else num_tets,
                                                *[a.data_ptr() for a in self.d], self.h, self.out.data_ptr(),
                                                self.stream)
        assert rc == _lib.MLX_OK, self.lib.mlx_last_error()
        self.torch.cuda.synchronize()
        return self.out.item()


def test_noalloc_residual_matches_layer_solve_twice(gpu, lib):
    torch = pytest.importorskip("torch")
    m, case, xi, lam, expected = _state((6, 3, 3), 21)
    call = _Call(torch, lib, m, case, xi, lam)
    for _ in range(2):
        np.testing.assert_allclose(call(), expected, rtol=1e-9)


def test_noalloc_allocates_nothing(gpu, lib):
    """Free device memory and torch's allocator are the same before and after
    two calls (after one set-up call: the first call in a context looks the
    scratch array up)."""
    torch = pytest.importorskip("torch")
    m, case, xi, lam, expected = _state((6, 3, 3), 31)
    call = _Call(torch, lib, m, case, xi, lam)
    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0, res0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    values = [call(), call()]
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == res0
    assert free1 >= free0, f"free device memory fell by {free0 - free1} bytes"
    np.testing.assert_allclose(values, [expected, expected], rtol=1e-9)


def test_noalloc_many_blocks(gpu, lib):
    """A mesh of thousands of tets spans many partial sums (> 40 blocks)."""
    torch = pytest.importorskip("torch")
    m, case, xi, lam, expected = _state((24, 10, 8), 41)
    assert m.T > 40 * 256
    call = _Call(torch, lib, m, case, xi, lam)
    for _ in range(2):
        np.testing.assert_allclose(call(), expected, rtol=1e-9)


def test_noalloc_empty_mesh_gives_zero(gpu, lib):
    torch = pytest.importorskip("torch")
    m, case, xi, lam, _ = _state((2, 1, 1), 51)
    call = _Call(torch, lib, m, case, xi, lam)
    assert call(num_tets=0) == 0.0


def test_noalloc_bad_index_gives_nan_and_context_stays_usable(gpu, lib):
    """A vertex index beyond the mesh is not read (the kernel checks every
    index against num_vertices before loading): the residual is NaN, and the
    next call on valid data gives the regular value."""
    torch = pytest.importorskip("torch")
    m, case, xi, lam, expected = _state((6, 3, 3), 61)
    t = np.asfortranarray(m.t).copy()
    t[5, 2] = m.N + 1000
    bad = _Call(torch, lib, m, case, xi, lam, t=t)
    assert np.isnan(bad())
    good = _Call(torch, lib, m, case, xi, lam)
    np.testing.assert_allclose(good(), expected, rtol=1e-9)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu, lib):
    rc = lib.mlx_stvk_residual_noalloc(10, _lib.MLX_NOALLOC_MAX_TETS + 1, None, None, None, None, None, None,
                                       0.01, None, None)
    assert rc == _lib.MLX_ERR_ARGUMENT
    assert b"at most" in lib.mlx_last_error()
