"""The oracle pinned against the reference itself (CPU only).

Golden fixtures in tests/golden come from the reference's own code: its
symbolic Green-strain expressions (3d/constraints/StVKconstraintGrad3D.m,
evaluated by tests/golden/make_golden.py) and its layer-builder mex files
compiled unchanged (3d/mex/mexEdiffNorm3D.cpp, 2d/mex/mexUnionFindByVertice.cpp).
"""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


def test_stvk_constraint_grad_matches_reference_expressions(oracle):
    g = np.load(GOLD / "stvk_grad.npz")
    worst = 0.0
    for i in range(g["x"].shape[0]):
        grad, C = oracle.stvk_constraint_grad(g["DmInv"][i].T.reshape(-1), g["x"][i])
        worst = max(worst, np.abs(grad - g["gradC"][i]).max() / np.abs(g["gradC"][i]).max(),
                    np.abs(C - g["C"][i]).max() / np.abs(g["C"][i]).max())
    assert worst <= 1e-14


@pytest.mark.parametrize("tag", ["beam", "block"])
def test_layer_builder_matches_reference_mex(oracle, tag):
    L = np.load(GOLD / "layers.npz")
    N = L[f"{tag}_V"].shape[0]
    n = oracle.strain_rate_norms(L[f"{tag}_T"], L[f"{tag}_DmInv"], L[f"{tag}_p"], L[f"{tag}_oldp"],
                                 float(L[f"{tag}_h"]))
    np.testing.assert_allclose(n, L[f"{tag}_norms"], rtol=1e-12, atol=1e-12 * np.abs(L[f"{tag}_norms"]).max())
    assert np.array_equal(np.argsort(n, kind="stable") + 1, L[f"{tag}_order"])
    sets, nr = oracle.union_find_layers(L[f"{tag}_order"], L[f"{tag}_layers"], L[f"{tag}_forced"],
                                        L[f"{tag}_T"], N)
    assert np.array_equal(sets, L[f"{tag}_sets"])
    assert np.array_equal(nr, L[f"{tag}_numRigids"])


def test_union_find_live_reference_mex(oracle):
    """Random orders, layer sets and forced-elastic masks against the compiled
    reference mex (needs oracle/_ref, built where the reference is mounted)."""
    if not oracle.ref_available("mexUnionFindByVertice"):
        pytest.skip("oracle/_ref not built (reference tree not mounted)")
    from multilayersolver2024_b200 import scenes
    uf = oracle.RefMex("mexUnionFindByVertice")
    rng = np.random.default_rng(3)
    for dims in [(4, 3, 2), (7, 2, 3)]:
        V, T, _ = scenes.generate_beam(*dims)
        N, nt = V.shape[0], T.shape[0]
        for _ in range(5):
            order = (rng.permutation(nt) + 1).astype(np.int32)
            forced = rng.random(nt) < 0.15
            layers = np.sort(rng.choice(np.arange(0, 101, 5), 3, replace=False)).astype(float)
            layers[0] = 0.0
            ref_sets, ref_nr = uf(2, order.astype(float), layers[None, :], forced, np.asfortranarray(T), float(N))
            sets, nr = oracle.union_find_layers(order, layers, forced, T, N)
            assert np.array_equal(sets, ref_sets.astype(np.int32))
            assert np.array_equal(nr, ref_nr.ravel().astype(np.int32))


def test_exp_rodrigues_is_a_rotation(oracle):
    import ctypes as C
    lib = oracle.load()
    rng = np.random.default_rng(0)
    for w in list(rng.normal(0, 3, (20, 3))) + [np.zeros(3)]:
        R = np.zeros(9)
        lib.orc_exp_rodrigues(oracle.f64(np.ascontiguousarray(w)), 0.01, oracle.f64(R))
        R = R.reshape(3, 3, order="F")
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
        assert abs(np.linalg.det(R) - 1) < 1e-14


def _rest_tet():
    x = np.array([0, 0, 0, 0.1, 0, 0, 0, 0.1, 0, 0, 0, 0.1], float)
    Dm = np.stack([x[3:6] - x[:3], x[6:9] - x[:3], x[9:12] - x[:3]], 1)
    return x, np.linalg.inv(Dm)


def test_stvk_rest_state_is_a_fixed_point(oracle):
    """x = rest => C = 0, dlambda = 0, dx = 0 (matStvkVoigtConstraint3D)."""
    from multilayersolver2024_b200.mesh3d import material_blocks, to_lame
    x, G = _rest_tet()
    mu, lam = to_lame(0.3, 1e5)
    a, _, b = material_blocks(np.array([mu]), np.array([lam]), np.array([0.01]))
    h = 0.01
    dx, dl, C = np.zeros(12), np.zeros(6), np.zeros(6)
    oracle.load().orc_stvk_voigt_project(
        oracle.f64(x), oracle.f64(x.copy()), oracle.f64(np.ascontiguousarray(G.T.reshape(-1))),
        oracle.f64(np.ascontiguousarray(a[0] / h ** 2)), oracle.f64(np.zeros(6)), oracle.f64(np.full(12, 2.0)),
        1e-3 / 6, oracle.f64(np.ascontiguousarray(b[0] * h ** 2)), h, oracle.f64(dx), oracle.f64(dl), oracle.f64(C))
    assert np.abs(C).max() < 1e-15 and np.abs(dl).max() < 1e-15 and np.abs(dx).max() < 1e-15


def test_stvk_one_tet_stretch_known_answer(oracle):
    """A 10% stretch along x of a right tet: E11 = ((1.1)^2 - 1)/2 = 0.105,
    other strains 0; C = vol * E."""
    x, G = _rest_tet()
    xs = x.copy()
    xs[0::3] *= 1.1
    grad, C = oracle.stvk_constraint_grad(G.T.reshape(-1), xs)
    np.testing.assert_allclose(C, [0.105, 0, 0, 0, 0, 0], atol=1e-15)


def test_nh_gradients_match_finite_differences(oracle):
    """The 3D Neo-Hookean pair (no 3D reference exists): C_D = sqrt(||F||^2 +
    J^2 - 4J), C_H = J - 1; the update uses their finite-difference gradients
    and solves the coupled 2x2 block; at rest both vanish and nothing moves."""
    lib = oracle.load()
    rng = np.random.default_rng(1)
    x0, G = _rest_tet()
    Gc = np.ascontiguousarray(G.T.reshape(-1))
    mu, lm, vol, h = 3e4, 5e4, 1e-3 / 6, 0.01
    minv = rng.uniform(0.5, 2.0, 4).repeat(3)

    def CC(xx):
        dx, dl, C, aT = np.zeros(12), np.zeros(2), np.zeros(2), np.zeros(2)
        lib.orc_nh_project(oracle.f64(np.ascontiguousarray(xx)), oracle.f64(Gc), mu, lm, vol, h,
                           oracle.f64(np.zeros(2)), oracle.f64(np.ascontiguousarray(minv)), oracle.f64(dx),
                           oracle.f64(dl), oracle.f64(C), oracle.f64(aT))
        return C, dx, dl, aT

    C, dx, dl, aT = CC(x0)
    assert np.abs(C).max() < 1e-7 and np.abs(dx).max() < 1e-15
    x = x0 + rng.normal(0, 0.01, 12)
    C, dx, dl, aT = CC(x)
    Ds = np.stack([x[3:6] - x[:3], x[6:9] - x[:3], x[9:12] - x[:3]], 1)
    F = Ds @ G
    J = np.linalg.det(F)
    assert abs(C[0] - np.sqrt((F * F).sum() + J * J - 4 * J)) < 1e-12
    assert abs(C[1] - (J - 1)) < 1e-14
    np.testing.assert_allclose(aT, [1 / (vol * mu * h * h), 1 / (vol * (lm - mu) * h * h)], rtol=1e-14)
    eps = 1e-7
    gD = np.zeros(12)
    gH = np.zeros(12)
    for i in range(12):
        e = np.zeros(12)
        e[i] = eps
        gD[i] = (CC(x + e)[0][0] - CC(x - e)[0][0]) / (2 * eps)
        gH[i] = (CC(x + e)[0][1] - CC(x - e)[0][1]) / (2 * eps)
    A = np.array([[gD @ (minv * gD) + aT[0], gD @ (minv * gH)], [gD @ (minv * gH), gH @ (minv * gH) + aT[1]]])
    np.testing.assert_allclose(dl, np.linalg.solve(A, -C), rtol=1e-6)
    np.testing.assert_allclose(dx, minv * (gD * dl[0] + gH * dl[1]), rtol=1e-5, atol=1e-13)


def test_nh_energy_is_stable_neo_hookean():
    """mu/2 B + (lambda-mu)/2 (J-1)^2 equals the stable Neo-Hookean energy
    mu/2 (I_C - 3) + lambda/2 (J - 1 - mu/lambda)^2 up to a constant."""
    rng = np.random.default_rng(4)
    mu, lm = 2.0, 7.0
    for _ in range(20):
        F = np.eye(3) + rng.normal(0, 0.4, (3, 3))
        J = np.linalg.det(F)
        Ic = (F * F).sum()
        split = mu / 2 * (Ic + J * J - 4 * J) + (lm - mu) / 2 * (J - 1) ** 2
        snh = mu / 2 * (Ic - 3) + lm / 2 * (J - 1 - mu / lm) ** 2
        assert abs(split - snh + mu * mu / (2 * lm)) < 1e-12
        assert Ic + J * J - 4 * J >= -1e-12


LAYER_SOLVE_CASES = ["single_damped", "three_layers_contacts_monitor", "two_layers_elastic_contacts",
                     "run_until_hanging_stop"]


def reference_case(name):
    import sys
    sys.path.insert(0, str(GOLD))
    from make_golden import build_case
    case = build_case(name)
    gold = np.load(GOLD / "layer_solve.npz")
    np.testing.assert_array_equal(case.xi, gold[f"{name}_input_xi"])  # same inputs as when generated
    return case, gold


@pytest.mark.parametrize("name", LAYER_SOLVE_CASES)
def test_oracle_layer_solve_matches_reference_execution(oracle, name):
    """xpbdLayer3D.layerSolve executed from the reference's MATLAB source
    (tests/golden/mlite.py) vs the oracle restatement: positions, residual
    array (incl. the K x K contact term) and runUntil."""
    case, gold = reference_case(name)
    xi, _, res, run_until, _, _ = case.oracle()
    d = case.mesh.bbox_diagonal()
    assert np.abs(xi - gold[f"{name}_xi"]).max() / d <= 1e-12
    np.testing.assert_allclose(res, gold[f"{name}_residual"], rtol=1e-10, atol=1e-15)
    assert run_until == pytest.approx(float(gold[f"{name}_run_until"]), rel=1e-10)
