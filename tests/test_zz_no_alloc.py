"""mlx_stvk_residual_noalloc: the residual for callers that cannot allocate.

Callers such as a MATLAB mexcuda function working on gpuArray memory, or a
fixed-rate loop that must not stall on cudaMalloc, own every device buffer;
this entry point reads their device arrays and writes one device double,
keeping its reduction scratch in a fixed array inside the library.  Its value
must equal the residual the regular entry point (mlx_layer_solve with
compute_residuals) reports for the same state, call after call.  This file is
collected last so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib

from helpers import Case, block_mesh

pytestmark = pytest.mark.gpu


def _device(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def test_noalloc_residual_matches_layer_solve_twice(gpu, lib):
    torch = pytest.importorskip("torch")
    m = block_mesh(dims=(6, 3, 3), seed=21, alpha1=0.01)
    case = Case(m, [0], [1], seed=22)
    case.integ.computeResiduals = True
    case.integ.hangingStop = -1
    xi, _, residuals, _, lam, _ = case.product(_lib.MLX_FP64)
    expected = residuals[-1]
    assert residuals.size == 2 and expected > 0

    d_x = _device(torch, xi, np.float64)
    d_t = _device(torch, np.asfortranarray(m.t).ravel(order="F"), np.int32)
    d_G = _device(torch, m.DmInv, np.float64)
    d_a = _device(torch, m.perElementXPBDalphaMatrix, np.float64)
    d_l = _device(torch, np.asfortranarray(lam).ravel(order="F"), np.float64)
    d_v = _device(torch, m.elV, np.float64)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for _ in range(2):
        out.fill_(-1.0)
        rc = lib.mlx_stvk_residual_noalloc(m.N, m.T, d_x.data_ptr(), d_t.data_ptr(), d_G.data_ptr(),
                                           d_a.data_ptr(), d_l.data_ptr(), d_v.data_ptr(), case.h,
                                           out.data_ptr(), stream)
        assert rc == _lib.MLX_OK, lib.mlx_last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.item(), expected, rtol=1e-9)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu, lib):
    rc = lib.mlx_stvk_residual_noalloc(10, _lib.MLX_NOALLOC_MAX_TETS + 1, None, None, None, None, None, None,
                                       0.01, None, None)
    assert rc == _lib.MLX_ERR_ARGUMENT
    assert b"at most" in lib.mlx_last_error()
