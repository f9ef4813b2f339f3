"""Mesh files (TetGen .node/.ele, Medit .mesh) and the TimingData CSV
format (CPU only).  The reference's own assets are read when the reference
tree is present (skipped otherwise)."""
import os
from pathlib import Path

import numpy as np
import pytest

from multilayersolver2024_b200 import scenes
from multilayersolver2024_b200.meshio import (load_mesh, load_poly, orient_tets, read_ele, read_mesh, read_node,
                                              write_ele, write_node)
from multilayersolver2024_b200.simulate import TimingData, matlab_d, write_td_csv

REF = Path(os.environ["MLX_REFERENCE_TREE"]) if os.environ.get("MLX_REFERENCE_TREE") else None


@pytest.mark.parametrize("first", [0, 1])
def test_node_ele_round_trip(tmp_path, first):
    V, T, _ = scenes.generate_beam(3, 2, 2, 0.1)
    write_node(tmp_path / "b.node", V, first)
    write_ele(tmp_path / "b.ele", T, first)
    V2, A, B, f = read_node(tmp_path / "b.node")
    T2, TA = read_ele(tmp_path / "b.ele", f)
    assert f == first and B is None and A.shape == (len(V), 0) and TA.shape == (len(T), 0)
    np.testing.assert_array_equal(V2, V)
    np.testing.assert_array_equal(T2, T)
    m = load_poly(tmp_path / "b", 1e4, 2e4, scale=(2.0, 1.0, 1.0))
    assert m.N == len(V) and m.T == len(T)
    np.testing.assert_allclose(m.p.reshape(-1, 3)[:, 0], 2.0 * V[:, 0])


def test_node_attributes_markers_comments(tmp_path):
    (tmp_path / "c.node").write_text("# points\n4 3 1 1\n1 0 0 0 7 1\n2 1 0 0 7 0\n\n3 0 1 0 7 1  # c\n4 0 0 1 7 0\n")
    (tmp_path / "c.ele").write_text("1 4 1\n1 1 2 3 4 5\n")
    V, A, B, f = read_node(tmp_path / "c.node")
    T, TA = read_ele(tmp_path / "c.ele", f)
    assert f == 1
    np.testing.assert_array_equal(A[:, 0], [7, 7, 7, 7])
    np.testing.assert_array_equal(B, [1, 0, 1, 0])
    np.testing.assert_array_equal(T, [[1, 2, 3, 4]])
    np.testing.assert_array_equal(TA[:, 0], [5])


def test_medit_mesh_and_orientation(tmp_path):
    (tmp_path / "t.mesh").write_text(
        "MeshVersionFormatted 1\nDimension 3\nVertices\n4\n0 0 0 0\n1 0 0 0\n0 1 0 0\n0 0 1 0\n"
        "Triangles\n1\n1 2 3 0\nTetrahedra\n1\n1 3 2 4 2\nEnd\n")
    V, T, TL, F = read_mesh(tmp_path / "t.mesh")
    np.testing.assert_array_equal(T, [[1, 3, 2, 4]])  # negatively oriented as written
    np.testing.assert_array_equal(TL, [2])
    np.testing.assert_array_equal(F, [[1, 2, 3]])
    np.testing.assert_array_equal(orient_tets(V, T), [[1, 3, 4, 2]])
    m = load_mesh(tmp_path / "t.mesh", [1e3, 1e4, 1e5], [2e3, 2e4, 2e5])
    assert m.elV[0] > 0 and m.mu[0] == 1e3  # label 2 is the smallest label: first table entry


@pytest.mark.skipif(REF is None or not (REF / "3d/data/cube.node").exists(),
                    reason="MLX_REFERENCE_TREE is not set to the reference tree")
def test_reference_assets():
    cube = load_poly(REF / "3d/data/cube", 1e4, 2e4)
    assert (cube.N, cube.T) == (8, 6) and np.all(cube.elV > 0)
    np.testing.assert_allclose(cube.elV.sum(), 1.0)
    arma = load_poly(REF / "3d/data/arma_6", 1e4, 2e4)
    assert arma.N == 259 and np.all(arma.elV > 0)
    caps = load_mesh(REF / "3d/data/capsuleCoarse.mesh", 1e4, 2e4)
    assert caps.N == 475 and np.all(caps.elV > 0)


def test_timing_csv_format(tmp_path):
    td = TimingData()
    for k in range(3):
        td.contactCount = 10 * k
        td.countParticles = td.countTotalParticles = 81
        td.countTris = td.countTotalTris = 192
        td.stepSum = 0.01 * (k + 1)
        td.residual, td.residualPreSolve = 0.5, 2.0
        td.lastContact, td.lastSimulate = 1e-4, 2.5e-3
        td.integrateForces = 2e-3
        td.logData()
    assert td.log.shape == (11, 3) and td.logCounts.shape == (10, 3)
    (path,) = write_td_csv([td], str(tmp_path / "run_"), ["gpu"])
    lines = path.read_text().splitlines()
    assert lines[0].split(",")[:3] == ["contactCount", "countParticles", "countElements"]
    assert lines[0].split(",")[-1] == "connected components" and len(lines[0].split(",")) == 21
    assert lines[2].split(",")[:3] == ["10", "81", "192"]
    assert lines[2].split(",")[7] == "2.000000e-02"
    assert matlab_d(3.0) == "3" and matlab_d(0.5) == "5.000000e-01" and matlab_d(float("nan")) == "NaN"
