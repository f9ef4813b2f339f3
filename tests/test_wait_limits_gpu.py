"""The bounded device waits give up and report it (no GPU fault, no hang):
the grid barrier's wait of the persistent layer kernel and the tensor-core
GEMM's mbarrier wait, each run on a condition nothing satisfies with a
20 ms limit; the call returns within a second, reports the timeout, and the
context then runs a layer solve that matches the oracle."""
import ctypes as C
import time

import pytest

from multilayersolver2024_b200 import _lib

from helpers import Case, block_mesh, rel_pos_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", [0, 1])
def test_wait_runs_out_with_a_status(gpu, lib, kind):
    flag = C.c_int32(-1)
    t0 = time.perf_counter()
    rc = lib.mlx_wait_probe(0, kind, 20_000_000, C.byref(flag))
    dt = time.perf_counter() - t0
    assert rc == 0, lib.mlx_last_error()
    assert flag.value == 1
    assert 0.015 <= dt < 1.0
    m = block_mesh(dims=(4, 2, 2), seed=3)
    case = Case(m, [50, 0], [2, 3], seed=4)
    assert rel_pos_err(case.product(_lib.MLX_FP64)[0], case.oracle()[0], m) <= 1e-9
