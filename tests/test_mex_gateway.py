"""The MATLAB gateway mexLayerSolve3D (same 50 arguments and 4 results as
xpbdLayer3D.layerSolve), driven through the headless mx runtime."""
import os
from pathlib import Path

import numpy as np
import pytest

from multilayersolver2024_b200 import _lib

from helpers import Case, block_mesh, plane_contacts, rel_pos_err, sphere_contacts

GATEWAY = Path(__file__).resolve().parents[1] / "multilayersolver2024_b200" / "mex" / "libmexLayerSolve3D.so"


def _gateway():
    from oracle.oracle import MexLib
    if not GATEWAY.exists():
        pytest.fail(f"{GATEWAY} was not built")
    return MexLib(GATEWAY)


def layer_solve_args(case):
    """The argument list of xpbdLayer3D.layerSolve (xpbdLayer3D.m:44-93) with
    MATLAB classes: logical masks, int32 ids where the reference has them."""
    m, ls, it = case.mesh, case.ls, case.integ
    c = case.contacts
    K = c.vertex_ids.size
    return [
        ls.isElasticElement.astype(bool), ls.isRigidElement.astype(bool), ls.rigidBodySetsPerLayer,
        ls.vertexRigidBody, ls.isBoundaryVertex.astype(bool), ls.isRigidVertex.astype(bool),
        case.xi, np.asfortranarray(case.lam), 0.0, case.h, ls.numRigids.astype(float), np.array([[0.0]]),
        it.boundaryCompliance, it.contactResistance, c.compliance.reshape(-1, 1) if K else np.zeros((0, 1)),
        np.array([it.iterations], float), np.array([it.layers], float), it.runUntilResSmallerThan,
        np.array(bool(it.computeResiduals)), float(it.hangingStop), np.array(bool(it.giveUpEnabled)),
        it.giveUpThreshold, np.array(bool(it.LastLayerGiveUpEnabled)), np.array(bool(it.useGravityConstraints)),
        case.oldp, case.oldOldp, c.normals if K else np.zeros((0, 3)), c.points if K else np.zeros((0, 3)),
        c.vertex_ids.astype(float).reshape(-1, 1) if K else np.zeros((0, 1)), m.mass, np.asfortranarray(m.t),
        m.unpinnedDOFs.astype(float), m.pinnedDOFs.astype(float), m.DmInv.reshape(-1),
        m.perElementXPBDalphaMatrix.reshape(-1), m.perElementXPBDalphaInvMatrix.reshape(-1),
        m.elementColor.astype(float), m.elementDOFs, float(m.numColors), case.f,
        np.array(it.layersMap, float), it.gravityCompliance, it.Gravity, case.resv,
        m.perElementXPBDbeta.reshape(-1), m.elV, np.array(True), np.array(bool(it.useRigidContacts)),
        it.StopAtImprovementPercent, case.pinnedx,
    ]


def test_gateway_checks_its_argument_count():
    g = _gateway()
    with pytest.raises(RuntimeError, match="50 inputs"):
        g(4, np.zeros(3))


@pytest.mark.gpu
def test_gateway_matches_oracle(gpu, monkeypatch):
    monkeypatch.setenv("MLXPBD_PRECISION", "fp64")
    m = block_mesh(dims=(6, 3, 3), seed=31, alpha1=0.01)
    case = Case(m, [50, 0], [3, 6], seed=32)
    case.integ.boundaryCompliance = 0.0
    case.integ.computeResiduals = True
    case.integ.hangingStop = 100
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet
    case.contacts = ContactSet.concat([plane_contacts(case.xi, [0, 0, 1.0], [0, 0, 0.004]),
                                       sphere_contacts(case.xi, 0.12, [0.3, 0.15, 0.0])])
    args = layer_solve_args(case)
    assert len(args) == 50
    g = _gateway()
    xi, snm, res, run_until = g(4, *args)
    ref = case.oracle()
    assert rel_pos_err(xi.ravel(), ref[0], m) <= 1e-9
    np.testing.assert_allclose(res.ravel(), ref[2], rtol=1e-9, atol=1e-14)
    assert float(run_until.ravel()[0]) == pytest.approx(ref[3])
    # a second call reuses the cached solver
    xi2, _, _, _ = g(4, *args)
    assert rel_pos_err(xi2.ravel(), ref[0], m) <= 1e-9
