"""buildLayers + findBoundaryVertices on the device (mlx_build_layers)
against the reference's compiled mex (golden sets and body counts) and
against the host builder (strain-rate measures, stable sort, union-find,
boundary masks): every output bit-identical, for strain-rate and given
orders, several layer percentages (0 and 100 included) and pinned tets; and
integrate with strain-rate layers built on the device equals integrate with
the host builder."""
from pathlib import Path

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, merge_meshes
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, Solver, StepCache, XpbdLayer3D, build_layers_device,
                                                    find_boundary_vertices, strain_rate_norms, union_find_layers)

from helpers import block_mesh

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"


@pytest.mark.parametrize("tag", ["beam", "block"])
def test_golden_sets_from_the_reference_mex(gpu, tag):
    L = np.load(GOLD / "layers.npz")
    m = Mesh3D.from_arrays(L[f"{tag}_V"], L[f"{tag}_T"], 1e4, 2e4)
    s = Solver(m, precision=_lib.MLX_FP64, material="lame")
    ls = build_layers_device(s, m, L[f"{tag}_p"], L[f"{tag}_oldp"], float(L[f"{tag}_h"]), L[f"{tag}_layers"],
                             L[f"{tag}_forced"].astype(np.uint8), dminv=L[f"{tag}_DmInv"])
    np.testing.assert_array_equal(ls.rigidBodySetsPerLayer, L[f"{tag}_sets"])
    np.testing.assert_array_equal(ls.numRigids, L[f"{tag}_numRigids"])
    s.close()


def _scene(seed):
    parts = [block_mesh(dims=d, energy=_lib.MLX_ENERGY_STVK_VOIGT, seed=seed + k)
             for k, d in enumerate([(8, 3, 3), (5, 4, 2), (6, 2, 2)])]
    return merge_meshes(parts)


def _host(m, p, oldp, h, layers, forced, order=None):
    if order is None:
        order = np.argsort(strain_rate_norms(m, p, oldp, h), kind="stable").astype(np.int32) + 1
    sets, nr = union_find_layers(m, order, layers, forced)
    return find_boundary_vertices(m, sets, nr)


@pytest.mark.parametrize("layers", [[0.0], [0.0, 50.0], [10.0, 35.0, 70.0, 100.0]])
@pytest.mark.parametrize("ordering", ["strain_rate", "given"])
def test_matches_host_builder(gpu, layers, ordering):
    rng = np.random.default_rng(len(layers))
    m = _scene(3)
    s = Solver(m, precision=_lib.MLX_FP32, material="lame")
    forced = np.zeros(m.T, np.uint8)
    forced[m.pinnedTets - 1] = 1
    for trial in range(3):
        oldp = m.p + rng.normal(0, 1e-3, m.p.size)
        p = oldp + rng.normal(0, 2e-3, m.p.size)
        order = rng.permutation(m.T).astype(np.int32) + 1 if ordering == "given" else None
        got = build_layers_device(s, m, p, oldp, 0.01, layers, forced, order)
        ref = _host(m, p, oldp, 0.01, layers, forced, order)
        for name in ("rigidBodySetsPerLayer", "numRigids", "isElasticElement", "isBoundaryVertex", "isRigidVertex",
                     "vertexRigidBody"):
            np.testing.assert_array_equal(getattr(got, name), getattr(ref, name), err_msg=f"{name} trial {trial}")
        assert got.numRigids.max() > 0 or max(layers) == 0
    s.close()


def test_integrate_with_device_layers_equals_host_layers(gpu):
    def run(builder):
        m = block_mesh(dims=(8, 3, 3), energy=_lib.MLX_ENERGY_STVK_VOIGT, seed=5)
        m.v[2::3] = -1.0 * (m.p[0::3] / m.p[0::3].max())
        it = XpbdLayer3D()
        it.setLayers([60, 30, 0])
        it.iterations = [2, 2, 4]
        it.precision = _lib.MLX_FP64
        it.layerBuilder = builder
        cache = StepCache()
        out = []
        for frame in range(1, 5):
            it.integrate(m, 1.0 / 60.0, ContactSet(), cache, frame)
            out.append((m.p.copy(), cache.layers.copy()))
        return out
    a, b = run("device"), run("host")
    for k, ((pa, la), (pb, lb)) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(la, lb, err_msg=f"layers step {k}")
        np.testing.assert_array_equal(pa, pb, err_msg=f"positions step {k}")
