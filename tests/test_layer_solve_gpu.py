"""Parity of the CUDA layerSolve (through the C ABI) with the CPU oracle.

Every case feeds identical inputs to both sides.  Tolerances:
  FP64 product vs FP64 oracle: max |dx| <= 1e-9 of the bounding-box diagonal
    (same algorithm, different summation order in reductions);
  FP32 product vs FP64 oracle, one layerSolve call: <= 2e-5 of the diagonal.
"""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib
from multilayersolver2024_b200.xpbd_layer3d import ContactSet, Solver

from helpers import Case, block_mesh, plane_contacts, rel_pos_err, sphere_contacts

pytestmark = pytest.mark.gpu

TOL64 = 1e-9
TOL32 = 2e-5


def _contacts(case):
    # the sphere overlaps the ground contacts, so some vertices carry two
    # contacts (the elastic scatter's last-write-wins rule is exercised)
    p = case.xi
    return ContactSet.concat([plane_contacts(p, [0, 0, 1.0], [0, 0, 0.004]),
                              sphere_contacts(p, 0.12, [0.45, 0.15, 0.0])])


def _compare(case, prec=_lib.MLX_FP64, material="blocks", tol=TOL64):
    got = case.product(prec, material)
    ref = case.oracle(material)
    err = rel_pos_err(got[0], ref[0], case.mesh)
    assert err <= tol, f"position error {err:.3e} > {tol:.1e}"
    return got, ref


@pytest.mark.parametrize("energy", [_lib.MLX_ENERGY_STVK_VOIGT, _lib.MLX_ENERGY_NEOHOOKEAN])
def test_single_layer_fp64(gpu, energy):
    m = block_mesh(energy=energy, alpha1=0.01 if energy == _lib.MLX_ENERGY_STVK_VOIGT else 0.0)
    case = Case(m, [0], [12], seed=1)
    got, ref = _compare(case)
    lam_err = np.abs(got[4] - ref[4]).max() / max(np.abs(ref[4]).max(), 1e-30)
    assert lam_err <= 1e-8
    assert got[5] == ref[5] == 12


@pytest.mark.parametrize("energy", [_lib.MLX_ENERGY_STVK_VOIGT, _lib.MLX_ENERGY_NEOHOOKEAN])
@pytest.mark.parametrize("rigid_contacts", [True, False])
def test_multilayer_bodies_contacts_fp64(gpu, energy, rigid_contacts):
    m = block_mesh(dims=(8, 3, 3), energy=energy, seed=2)
    case = Case(m, [50, 25, 0], [2, 3, 6], seed=3)
    case.integ.boundaryCompliance = 0.0
    case.integ.useRigidContacts = rigid_contacts
    case.integ.contactResistance = 0.9
    case.contacts = _contacts(case)
    assert case.contacts.vertex_ids.size > 0
    assert case.ls.numRigids.max() > 0 and case.ls.isBoundaryVertex.any()
    _compare(case)


def test_residual_monitor_and_stop_rules_fp64(gpu):
    """computeResiduals + StopAtImprovementPercent + runUntil + hangingStop +
    give-up: identical residual arrays, iteration counts and runUntil."""
    m = block_mesh(dims=(6, 3, 3), seed=4)
    case = Case(m, [60, 30, 0], [3, 3, 4], seed=5)
    integ = case.integ
    integ.computeResiduals = True
    integ.StopAtImprovementPercent = 60
    integ.runUntilResSmallerThan = 0.0
    integ.hangingStop = 40
    integ.giveUpEnabled = True
    case.contacts = _contacts(case)
    got, ref = _compare(case)
    assert got[5] == ref[5], (got[5], ref[5])
    assert got[2].size == ref[2].size
    np.testing.assert_allclose(got[2], ref[2], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(got[3], ref[3], rtol=1e-9)


@pytest.mark.parametrize("spread", ["three_values", "all_distinct"])
def test_contact_residual_term_with_mixed_compliances_fp64(gpu, spread):
    """The residual's contact term meets every contact's compliance (the
    reference's K x 1 x K expansion, xpbdLayer3D.m:581-583).  With up to 32
    distinct compliances the device takes each once, times its count; with
    more it runs the K x K loop.  Both give the oracle's residual array."""
    m = block_mesh(dims=(8, 4, 4), seed=4)  # 49 contacts
    case = Case(m, [60, 0], [3, 6], seed=5)
    integ = case.integ
    integ.computeResiduals = True
    integ.runUntilResSmallerThan = 0.0
    integ.hangingStop = 30
    integ.contactResistance = 0.9
    c = _contacts(case)
    K = c.vertex_ids.size
    assert K > 32
    rng = np.random.default_rng(11)
    if spread == "three_values":
        c.compliance = rng.choice(np.array([1e-4, 5e-5, 2e-4]), K)
    else:
        c.compliance = rng.uniform(5e-5, 2e-4, K)
    case.contacts = c
    got, ref = _compare(case)
    assert got[5] == ref[5], (got[5], ref[5])
    np.testing.assert_allclose(got[2], ref[2], rtol=1e-9, atol=1e-14)


def test_lame_material_form_matches_blocks_fp64(gpu):
    m = block_mesh(alpha1=0.02, seed=6)
    case = Case(m, [40, 0], [3, 6], seed=7)
    a = case.product(_lib.MLX_FP64, "lame")
    b = case.oracle("blocks")
    assert rel_pos_err(a[0], b[0], m) <= 1e-9


@pytest.mark.parametrize("energy", [_lib.MLX_ENERGY_STVK_VOIGT, _lib.MLX_ENERGY_NEOHOOKEAN])
def test_multilayer_fp32_within_tolerance(gpu, energy):
    m = block_mesh(dims=(8, 3, 3), energy=energy, seed=8)
    case = Case(m, [50, 0], [3, 8], seed=9)
    case.integ.boundaryCompliance = 0.0
    case.contacts = _contacts(case)
    _compare(case, prec=_lib.MLX_FP32, material="lame", tol=TOL32)


def test_solver_reuse_across_calls(gpu):
    """Cached layer descriptions are refreshed when the layer masks change."""
    m = block_mesh(seed=10)
    s = Solver(m, precision=_lib.MLX_FP64)
    c1 = Case(m, [50, 0], [2, 4], seed=11)
    c2 = Case(m, [50, 0], [2, 4], seed=12)
    for c in (c1, c2, c1):
        got = c.product(solver=s)
        ref = c.oracle()
        assert rel_pos_err(got[0], ref[0], m) <= TOL64


def test_errors_are_reported(gpu, lib):
    import ctypes as C
    from multilayersolver2024_b200.xpbd_layer3d import mesh_desc
    m = block_mesh(seed=13)
    bad = m.elementColor.copy()
    bad[:] = 1
    d, keep = mesh_desc(m, 1, 0)
    keep["c"] = np.ascontiguousarray(bad, np.int32)
    d.element_color = _lib.i32(keep["c"])
    h = C.c_void_p()
    rc = lib.mlx_create(C.byref(d), C.byref(h))
    assert rc == _lib.MLX_ERR_ARGUMENT
    assert b"colouring" in lib.mlx_last_error()
    case = Case(m, [0], [3], seed=14)
    case.integ.runUntilResSmallerThan = 1e-3
    case.integ.computeResiduals = False
    solver = Solver(m, precision=_lib.MLX_FP64)  # keep a reference for the duration of the call
    rc, _ = case.run(lib.mlx_layer_solve, solver.handle)
    assert rc == _lib.MLX_ERR_ARGUMENT and b"compute_residuals" in lib.mlx_last_error()
    solver.close()


@pytest.mark.parametrize("name", ["single_damped", "three_layers_contacts_monitor", "two_layers_elastic_contacts",
                                  "run_until_hanging_stop"])
def test_fp64_matches_reference_execution(gpu, name):
    """The CUDA layerSolve (FP64) against results of the reference's own
    MATLAB source executed by tests/golden/mlite.py."""
    from test_oracle_pins import reference_case
    case, gold = reference_case(name)
    xi, _, res, run_until, _, _ = case.product(_lib.MLX_FP64)
    assert rel_pos_err(xi, gold[f"{name}_xi"], case.mesh) <= TOL64
    np.testing.assert_allclose(res, gold[f"{name}_residual"], rtol=1e-9, atol=1e-14)
    assert run_until == pytest.approx(float(gold[f"{name}_run_until"]), rel=1e-9)


LAUNCH_PATHS = {
    # name: (MLXPBD_CLUSTER, MLXPBD_CLUSTER_SIZE, MLXPBD_PERSISTENT, MLXPBD_PDL)
    "default": ("", "", "", ""),
    "cluster_auto": ("1", "", "0", "1"),
    "cluster_16": ("1", "16", "0", "1"),
    "cluster_4": ("1", "4", "0", "1"),
    "colour_launches_pdl": ("0", "", "0", "1"),
    "colour_launches": ("0", "", "0", "0"),
    "persistent_grid": ("0", "", "1", "1"),
}


def _set_path(monkeypatch, name):
    for var, val in zip(("MLXPBD_CLUSTER", "MLXPBD_CLUSTER_SIZE", "MLXPBD_PERSISTENT", "MLXPBD_PDL"),
                        LAUNCH_PATHS[name]):
        if val:
            monkeypatch.setenv(var, val)
        else:
            monkeypatch.delenv(var, raising=False)


@pytest.mark.parametrize("path", list(LAUNCH_PATHS))
def test_launch_paths_agree(gpu, monkeypatch, path):
    """Fixed iteration counts run as one thread-block cluster per layer with
    the vertex records in distributed shared memory (MLXPBD_CLUSTER=1; forced
    to 16 and 4 CTAs so that small meshes exercise remote records), as one launch per
    colour with or without programmatic dependent launches, or as one
    cooperative launch per layer; all match the oracle, bodies, glue and
    contacts included."""
    _set_path(monkeypatch, path)
    m = block_mesh(dims=(8, 3, 3), energy=_lib.MLX_ENERGY_NEOHOOKEAN, seed=41)
    case = Case(m, [50, 25, 0], [2, 3, 5], seed=42)
    case.integ.boundaryCompliance = 0.0
    case.contacts = _contacts(case)
    _compare(case)


@pytest.mark.parametrize("path", ["cluster_16", "cluster_4"])
@pytest.mark.parametrize("prec,tol", [(_lib.MLX_FP64, TOL64), (_lib.MLX_FP32, TOL32)])
@pytest.mark.parametrize("rigid_contacts", [True, False])
def test_cluster_path_stvk_damped(gpu, monkeypatch, path, prec, tol, rigid_contacts):
    """The cluster kernel on the damped StVK constraint (old positions read
    from global memory), rigid and elastic contacts and pinning, both storage
    precisions."""
    _set_path(monkeypatch, path)
    m = block_mesh(dims=(8, 3, 3), energy=_lib.MLX_ENERGY_STVK_VOIGT, alpha1=0.01, seed=43)
    case = Case(m, [50, 25, 0], [2, 3, 5], seed=44)
    case.integ.boundaryCompliance = 1e-7
    case.integ.useRigidContacts = rigid_contacts
    case.integ.contactResistance = 0.9
    case.contacts = _contacts(case)
    _compare(case, prec=prec, tol=tol)
