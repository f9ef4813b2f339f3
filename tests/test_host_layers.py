"""Host-side logic of the product (CPU): colouring, layer builder, boundary
masks and mesh precompute, against the oracle and the reference's mex."""
from pathlib import Path

import numpy as np
import pytest

from multilayersolver2024_b200 import scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, greedy_coloring, material_blocks, rest_state, to_lame
from multilayersolver2024_b200.xpbd_layer3d import (XpbdLayer3D, find_boundary_vertices, strain_rate_norms,
                                                    union_find_layers)

GOLD = Path(__file__).resolve().parent / "golden"


def _valid_coloring(t, col):
    seen = {}
    for e, c in enumerate(col):
        for v in t[e]:
            assert (int(v), int(c)) not in seen, "two tets of one colour share a vertex"
            seen[(int(v), int(c))] = e


@pytest.mark.parametrize("dims", [(8, 2, 2), (5, 4, 3), (12, 12, 2)])
def test_coloring_matches_first_fit(oracle, dims):
    V, T, _ = scenes.generate_beam(*dims)
    col, nc = greedy_coloring(T, V.shape[0])
    ocol, onc = oracle.greedy_coloring(T, V.shape[0])
    assert np.array_equal(col, ocol) and nc == onc
    _valid_coloring(T, col)


def test_coloring_beyond_64_colours(oracle):
    """A fan of tets around one vertex needs more colours than one bitset word."""
    n = 150
    T = np.stack([np.zeros(n), np.arange(1, n + 1), np.arange(n + 1, 2 * n + 1), np.arange(2 * n + 1, 3 * n + 1)],
                 1).astype(np.int32) + 1
    col, nc = greedy_coloring(T, 3 * n + 1)
    ocol, onc = oracle.greedy_coloring(T, 3 * n + 1)
    assert nc == n == onc and np.array_equal(col, ocol)


@pytest.mark.parametrize("tag", ["beam", "block"])
def test_product_layer_builder_matches_reference_mex(tag):
    L = np.load(GOLD / "layers.npz")
    V, T = L[f"{tag}_V"], L[f"{tag}_T"]
    m = Mesh3D.from_arrays(V, T, 1e4, 2e4)
    n = strain_rate_norms(m, L[f"{tag}_p"], L[f"{tag}_oldp"], float(L[f"{tag}_h"]))
    np.testing.assert_allclose(n, L[f"{tag}_norms"], rtol=1e-12, atol=1e-12 * np.abs(L[f"{tag}_norms"]).max())
    assert np.array_equal(np.argsort(n, kind="stable") + 1, L[f"{tag}_order"])
    sets, nr = union_find_layers(m, L[f"{tag}_order"], L[f"{tag}_layers"], L[f"{tag}_forced"])
    assert np.array_equal(sets, L[f"{tag}_sets"]) and np.array_equal(nr, L[f"{tag}_numRigids"])


def test_boundary_masks_match_oracle(oracle):
    L = np.load(GOLD / "layers.npz")
    V, T, sets = L["block_V"], L["block_T"], L["block_sets"]
    m = Mesh3D.from_arrays(V, T, 1e4, 2e4)
    ls = find_boundary_vertices(m, sets, L["block_numRigids"])
    bnd, ela, rig, vb = oracle.find_boundary_vertices(T, V.shape[0], sets)
    assert np.array_equal(ls.isBoundaryVertex, bnd) and np.array_equal(ls.isElasticElement, ela)
    assert np.array_equal(ls.isRigidVertex, rig) and np.array_equal(ls.vertexRigidBody, vb)
    # a boundary vertex is rigid and touches an elastic tet
    assert np.all(ls.isRigidVertex[ls.isBoundaryVertex.astype(bool)])


def test_mesh_precompute_matches_oracle(oracle):
    import ctypes as C
    lib = oracle.load()
    V, T, _ = scenes.generate_beam(3, 2, 2, 0.1)
    rng = np.random.default_rng(2)
    nt = T.shape[0]
    E = rng.uniform(1e4, 1e6, nt)
    mu, lam = to_lame(0.3, E)
    a1 = rng.uniform(0, 0.02, nt)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=a1)
    G, vol = np.zeros(9 * nt), np.zeros(nt)
    lib.orc_rest_state(oracle.f64(np.ascontiguousarray(m.p)), oracle.i32(np.asfortranarray(T)), nt,
                       oracle.f64(G), oracle.f64(vol))
    np.testing.assert_allclose(m.DmInv.ravel(), G, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(m.elV, vol, rtol=1e-13)
    al, ai, be = np.zeros(36 * nt), np.zeros(36 * nt), np.zeros(36 * nt)
    lib.orc_update_materials(oracle.f64(mu), oracle.f64(lam), oracle.f64(a1), nt, oracle.f64(al), oracle.f64(ai),
                             oracle.f64(be))
    np.testing.assert_allclose(m.perElementXPBDalphaMatrix.ravel(), al, rtol=1e-12, atol=1e-22)
    np.testing.assert_array_equal(m.perElementXPBDalphaInvMatrix.ravel(), ai)
    np.testing.assert_array_equal(m.perElementXPBDbeta.ravel(), be)
    mass = np.zeros(3 * m.N)
    lib.orc_compute_mass(oracle.i32(np.asfortranarray(T)), nt, m.N, oracle.f64(m.elV),
                         oracle.f64(np.full(nt, 1000.0)), oracle.f64(mass))
    np.testing.assert_array_equal(m.mass, mass)


def test_generated_beam_is_positively_oriented_and_sized():
    V, T, cube = scenes.generate_beam(64, 16, 16, 0.1)
    assert V.shape[0] == 18785 and T.shape[0] == 98304
    _, vol = rest_state(V.reshape(-1), T)
    assert np.all(vol > 0)
    np.testing.assert_allclose(vol.sum(), 6.4 * 1.6 * 1.6, rtol=1e-12)


def test_set_layers_mirrors_unique():
    integ = XpbdLayer3D()
    integ.setLayers([80, 60, 40, 0])
    assert integ.sortedLayers == [0, 40, 60, 80] and integ.layersMap == [4, 3, 2, 1]
    integ.setLayers([50, 0])
    assert integ.layersMap == [2, 1]


def test_config2_clusters_do_not_share_vertices():
    s = scenes.config2()
    m = s.mesh
    sets = s.custom_sets[:, 1]
    owner = np.zeros(m.N + 1, np.int32)
    for k in range(4):
        v = m.t[:, k]
        rig = sets > 0
        prev = owner[v[rig]]
        assert np.all((prev == 0) | (prev == sets[rig]))
        owner[v[rig]] = sets[rig]
    assert sets.max() == 32
    assert not np.any(sets[m.pinnedTets - 1])
