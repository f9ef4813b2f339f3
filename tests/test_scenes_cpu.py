"""Scene builders without a GPU: the replicated cantilever (copies of the
8x2x2 cantilever in one mesh) has the layout Mesh3D.mergeMesh gives its parts
(3d/@Mesh3D/Mesh3D.m:300-338): vertices and tets concatenated with offsets,
every copy's colours, masses and rest shapes equal to the solo cantilever's,
and every copy's x = 0 face pinned."""
import numpy as np

from multilayersolver2024_b200 import scenes
from multilayersolver2024_b200.mesh3d import merge_meshes


def test_replicated_cantilever_layout():
    k, per_row = 8, 4
    rep = scenes.config1_replicated(k, per_row=per_row)
    one = scenes.config1()
    m, s = rep.mesh, one.mesh
    assert (m.N, m.T) == (k * s.N, k * s.T)
    assert (rep.h, rep.layers, rep.iterations) == (one.h, one.layers, one.iterations)
    assert rep.custom_sets.shape == (m.T, 1) and not rep.custom_sets.any()
    np.testing.assert_array_equal(m.elementColor, np.tile(s.elementColor, k))
    assert m.numColors == s.numColors
    np.testing.assert_array_equal(m.t, np.concatenate([s.t + c * s.N for c in range(k)]))
    np.testing.assert_allclose(m.mass, np.tile(s.mass, k), rtol=1e-12)
    np.testing.assert_allclose(m.DmInv, np.tile(s.DmInv, (k, 1)), rtol=1e-9, atol=1e-12)
    np.testing.assert_array_equal(m.pinnedInds, np.concatenate([s.pinnedInds + c * s.N for c in range(k)]))
    # copies on the y-z grid, 0.4 m apart
    P, P1 = m.p.reshape(k, s.N, 3), s.p.reshape(s.N, 3)
    for c in range(k):
        shift = np.broadcast_to([0.0, 0.4 * (c % per_row), 0.4 * (c // per_row)], P1.shape)
        np.testing.assert_allclose(P[c] - P1, shift, atol=1e-12)
    np.testing.assert_array_equal(m.part_vertex_offsets, s.N * np.arange(k + 1))
    np.testing.assert_array_equal(m.part_tet_offsets, s.T * np.arange(k + 1))


def test_replicated_cantilever_equals_merge_meshes():
    """The direct construction equals merge_meshes over the translated copies."""
    k, per_row = 3, 2
    rep = scenes.config1_replicated(k, per_row=per_row)
    parts = []
    for c in range(k):
        part = scenes.config1().mesh
        V = part.p.reshape(-1, 3) + np.array([0.0, 0.4 * (c % per_row), 0.4 * (c // per_row)])
        parts.append(type(part).from_arrays(V, part.t, part.mu, part.lam, rho=part.rho, alpha1=part.alpha1,
                                            energy_type=part.energy_type))
        parts[-1].pin(part.pinnedInds)
    ref = merge_meshes(parts)
    np.testing.assert_array_equal(rep.mesh.t, ref.t)
    np.testing.assert_array_equal(rep.mesh.elementColor, ref.elementColor)
    np.testing.assert_array_equal(rep.mesh.pinnedDOFs, ref.pinnedDOFs)
    np.testing.assert_allclose(rep.mesh.p, ref.p, atol=1e-12)
    np.testing.assert_allclose(rep.mesh.mass, ref.mass, rtol=1e-12)
