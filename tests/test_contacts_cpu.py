"""Known answers for the oracle's contact finders and the rotation helper
(CPU only)."""
import numpy as np

from multilayersolver2024_b200.contacts import (PlaneContactFinder3D, PlatformContactDetector, SphereContactFinder,
                                                rotation_matrix_degrees)


def test_rotation_matrix_degrees():
    R = rotation_matrix_degrees([0, 0, 90])
    np.testing.assert_allclose(R, [[0, -1, 0], [1, 0, 0], [0, 0, 1]], atol=1e-15)
    R = rotation_matrix_degrees([30, -20, 75])
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
    assert np.isclose(np.linalg.det(R), 1.0)
    # 'XYZ': R = Rx Ry Rz
    Rx = rotation_matrix_degrees([30, 0, 0])
    Ry = rotation_matrix_degrees([0, -20, 0])
    Rz = rotation_matrix_degrees([0, 0, 75])
    np.testing.assert_allclose(R, Rx @ Ry @ Rz, atol=1e-15)


def test_platform_finder_known_answers(oracle):
    # unit box (scale 2, half extents 1) at the origin, axis aligned
    p = np.array([0.0, 0.0, 0.9,      # nearest the +z face: n = +z, phi = -0.1
                  -0.8, 0.1, 0.0,     # nearest the -x face: n = -x, phi = -0.2
                  0.0, 0.0, 1.5,      # outside
                  0.5, 0.5, 0.5])     # tie between all axes: the first (x) wins, phi = -0.5
    n, q, ids, a = oracle.find_contacts_platform(p, np.eye(3), [2.0, 2.0, 2.0], [0.0, 0.0, 0.0], 3e-5)
    np.testing.assert_array_equal(ids, [1, 2, 4])
    np.testing.assert_allclose(n, [[0, 0, 1], [-1, 0, 0], [1, 0, 0]])
    np.testing.assert_allclose(q, [[0, 0, 1.0], [-1.0, 0.1, 0], [1.0, 0.5, 0.5]], atol=1e-15)
    np.testing.assert_array_equal(a, [3e-5] * 3)


def test_finder_loop_concatenates_in_order(oracle):
    p = np.array([0.0, 0.0, -0.1, 0.0, 0.0, 0.05, 2.0, 0.0, 0.2])
    finders = [SphereContactFinder(0.5, [0, 0, 0]), PlaneContactFinder3D([0, 0, 2.0], [0, 0, 0], 1e-6),
               PlatformContactDetector([0, 0, 0], [1, 1, 1], [2, 0, 0], 2e-6)]
    cs = oracle.find_contacts(finders, p)
    # sphere: vertices 1, 2; plane (raw normal length 2 -> D = 0): vertex 1; box: vertex 3
    np.testing.assert_array_equal(cs.vertex_ids, [1, 2, 1, 3])
    np.testing.assert_array_equal(cs.compliance, [1e-4, 1e-4, 1e-6, 2e-6])
    np.testing.assert_allclose(cs.normals[2], [0, 0, 1])
