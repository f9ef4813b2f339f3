"""Config 5 (the learned warm start's workload: Neo-Hookean block, three
layers -- coarse clusters, mid clusters, fine) at reduced size against the
oracle integrate: FP64 <= 1e-9 and FP32 <= 1e-4 of the bounding-box diagonal
over 5 steps; the full-size scene steps stay finite."""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes

from test_step_gpu import _oracle_run, _resident_run

pytestmark = pytest.mark.gpu


def _small():
    return scenes.config5(seed=12, nx=12, ny=6, nz=6, coarse=4, mid=2)


@pytest.mark.parametrize("precision,tol", [(_lib.MLX_FP64, 1e-9), (_lib.MLX_FP32, 1e-4)])
def test_small_block_matches_oracle(gpu, oracle, precision, tol):
    steps = 5
    ref = _oracle_run(_small(), steps, oracle, threads=8)
    got, _ = _resident_run(_small(), steps, precision)
    d = _small().mesh.bbox_diagonal()
    err = max(np.abs(a - b).max() / d for a, b in zip(got, ref))
    assert err <= tol, err


def test_full_scene_steps(gpu):
    sc = scenes.config5()
    assert sc.mesh.T == 393_216
    got, sim = _resident_run(sc, 3, _lib.MLX_FP32)
    assert all(np.all(np.isfinite(p)) for p in got)
    assert np.abs(got[-1] - sc.mesh.p).max() > 0
