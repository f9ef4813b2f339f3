"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

Loads oracle/liboracle.so (the FP64 C++ restatement of the reference path, see
oracle.cpp) and, when built, the reference's own mex files compiled unchanged
against the headless mx runtime (oracle/_ref/*.so).  Only tests, the smoke
check and bench.py's CPU-baseline leg import this module; the product never
does.  ``integrate`` below is an independent restatement of
xpbdLayer3D.integrate (3d/integrator/xpbdLayer3D.m:621-745) built on the
oracle's C functions.  The marshalling to the oracle's C entry points (the
argument structs of include/mlxpbd.h, contact lists, layer sets, parameters)
is this module's own, so a layout error in the product's marshalling cannot
hide in both sides of a comparison; the integrator settings and meshes it
receives are plain data (attributes are read, no product code is called).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF = HERE / "_ref"

_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    sig = {
        "orc_last_error": ([], C.c_char_p),
        "orc_set_threads": ([C.c_int], None),
        "orc_max_threads": ([], C.c_int),
        "orc_stvk_constraint_grad": ([_f64p, _f64p, _f64p, _f64p], None),
        "orc_stvk_voigt_project": ([_f64p, _f64p, _f64p, _f64p, _f64p, _f64p, C.c_double, _f64p, C.c_double,
                                    _f64p, _f64p, _f64p], None),
        "orc_nh_project": ([_f64p, _f64p, C.c_double, C.c_double, C.c_double, C.c_double, _f64p, _f64p, _f64p,
                            _f64p, _f64p, _f64p], None),
        "orc_exp_rodrigues": ([_f64p, C.c_double, _f64p], None),
        "orc_greedy_coloring": ([_i32p, C.c_int32, C.c_int32, _i32p], C.c_int),
        "orc_rest_state": ([_f64p, _i32p, C.c_int32, _f64p, _f64p], None),
        "orc_update_materials": ([_f64p, _f64p, _f64p, C.c_int32, _f64p, _f64p, _f64p], None),
        "orc_compute_mass": ([_i32p, C.c_int32, C.c_int32, _f64p, _f64p, _f64p], None),
        "orc_strain_rate_norms": ([_i32p, C.c_int32, _f64p, _f64p, _f64p, C.c_double, _f64p], None),
        "orc_union_find_layers": ([_i32p, C.c_int32, _f64p, C.c_int32, _u8p, _i32p, C.c_int32, _i32p, _i32p],
                                  C.c_int),
        "orc_find_boundary_vertices": ([_i32p, C.c_int32, C.c_int32, _i32p, C.c_int32, _u8p, _u8p, _u8p, _i32p],
                                       None),
        "orc_layer_solve": ([C.POINTER(MeshDesc), C.POINTER(LayerDesc), C.POINTER(SolveParams),
                             C.POINTER(Contacts), C.POINTER(SolveInputs), C.POINTER(SolveOutputs)], C.c_int),
        "orc_contact_velocity_update": ([_f64p, _i32p, C.c_int32, _f64p, C.c_double, C.c_double, C.c_double],
                                        None),
        "orc_find_contacts_plane": ([_f64p, C.c_int32, _f64p, _f64p, C.c_double, _i32p, _f64p, _f64p, _f64p],
                                    C.c_int),
        "orc_find_contacts_sphere": ([_f64p, C.c_int32, C.c_double, _f64p, _i32p, _f64p, _f64p, _f64p], C.c_int),
        "orc_find_contacts_platform": ([_f64p, C.c_int32, _f64p, _f64p, _f64p, C.c_double, _i32p, _f64p, _f64p,
                                        _f64p], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _p(a, t):
    if a is None:
        return C.cast(None, C.POINTER(t))
    return a.ctypes.data_as(C.POINTER(t))


# ---- the argument structs of include/mlxpbd.h (layout of the C header) ----
class MeshDesc(C.Structure):
    _fields_ = [("num_vertices", C.c_int32), ("num_tets", C.c_int32), ("t", _i32p), ("mass", _f64p),
                ("DmInv", _f64p), ("volume", _f64p), ("element_color", _i32p), ("num_colors", C.c_int32),
                ("pinned_dofs", _i32p), ("num_pinned_dofs", C.c_int32), ("energy_type", C.c_int32),
                ("alpha", _f64p), ("beta", _f64p), ("mu", _f64p), ("lambda_", _f64p), ("alpha1", _f64p),
                ("precision", C.c_int32), ("device", C.c_int32)]


class LayerDesc(C.Structure):
    _fields_ = [("num_layers", C.c_int32), ("num_columns", C.c_int32), ("layers_map", _i32p),
                ("iterations", _i32p), ("is_elastic_element", _u8p), ("is_rigid_element", _u8p),
                ("rigid_body_sets", _i32p), ("vertex_rigid_body", _i32p), ("is_boundary_vertex", _u8p),
                ("is_rigid_vertex", _u8p), ("num_rigids", _i32p)]


class SolveParams(C.Structure):
    _fields_ = [("h", C.c_double), ("boundary_compliance", C.c_double), ("contact_resistance", C.c_double),
                ("run_until", C.c_double), ("give_up_threshold", C.c_double), ("gravity_compliance", C.c_double),
                ("gravity", C.c_double), ("stop_at_improvement_percent", C.c_double),
                ("compute_residuals", C.c_int32), ("hanging_stop", C.c_int32), ("give_up_enabled", C.c_int32),
                ("last_layer_give_up_enabled", C.c_int32), ("use_gravity_constraints", C.c_int32),
                ("use_rigid_contacts", C.c_int32), ("contact_coloring", C.c_int32)]


class Contacts(C.Structure):
    _fields_ = [("num_contacts", C.c_int32), ("normals", _f64p), ("point_colliders", _f64p),
                ("vertex_ids", _i32p), ("compliance", _f64p)]


class SolveInputs(C.Structure):
    _fields_ = [("xi", _f64p), ("lambdai", _f64p), ("oldp", _f64p), ("old_oldp", _f64p), ("f", _f64p),
                ("residualv", _f64p), ("pinnedx", _f64p), ("residual_in", _f64p), ("residual_in_len", C.c_int32),
                ("sum_non_monitored_time", C.c_double)]


class SolveOutputs(C.Structure):
    _fields_ = [("xi", _f64p), ("lambdai", _f64p), ("residual", _f64p), ("residual_capacity", C.c_int32),
                ("residual_len", C.c_int32), ("run_until", C.c_double), ("sum_non_monitored_time", C.c_double),
                ("total_iterations", C.c_int32)]


ENERGY_NEOHOOKEAN = 1  # mlx_mesh_desc.energy_type of the stable Neo-Hookean pair (include/mlxpbd.h)
OBSTACLE_PLANE, OBSTACLE_SPHERE, OBSTACLE_BOX = 1, 2, 3  # MLX_OBSTACLE_* of include/mlxpbd.h


class ContactList:
    """One contact list in simulate3D's format: normals and point colliders
    (K x 3), 1-based vertex ids, compliances."""

    def __init__(self, normals=None, points=None, vertex_ids=None, compliance=None):
        self.normals = np.zeros((0, 3)) if normals is None else np.asarray(normals, float).reshape(-1, 3)
        self.points = np.zeros((0, 3)) if points is None else np.asarray(points, float).reshape(-1, 3)
        self.vertex_ids = np.zeros(0, np.int32) if vertex_ids is None else np.asarray(vertex_ids, np.int32).ravel()
        self.compliance = np.zeros(0) if compliance is None else np.asarray(compliance, float).ravel()

    @staticmethod
    def concat(lists):
        lists = [c for c in lists if c.vertex_ids.size]
        if not lists:
            return ContactList()
        return ContactList(np.concatenate([c.normals for c in lists]), np.concatenate([c.points for c in lists]),
                           np.concatenate([c.vertex_ids for c in lists]),
                           np.concatenate([c.compliance for c in lists]))


def _mesh_desc(mesh, material, keep):
    """mlx_mesh_desc of a mesh (FP64 oracle: precision and device unused)."""
    def k(a, dt):
        keep.append(np.ascontiguousarray(a, dt) if dt is not None else a)
        return keep[-1]
    d = MeshDesc()
    d.num_vertices, d.num_tets = int(mesh.N), int(mesh.T)
    d.t = i32(k(np.asfortranarray(mesh.t, np.int32), None))
    d.mass = f64(k(mesh.mass, np.float64))
    d.DmInv = f64(k(mesh.DmInv, np.float64))
    d.volume = f64(k(mesh.elV, np.float64))
    d.element_color = i32(k(mesh.elementColor, np.int32))
    d.num_colors = int(mesh.numColors)
    d.pinned_dofs = i32(k(mesh.pinnedDOFs, np.int32))
    d.num_pinned_dofs = int(np.asarray(mesh.pinnedDOFs).size)
    d.energy_type = int(mesh.energy_type)
    if int(mesh.energy_type) != ENERGY_NEOHOOKEAN and material == "blocks":
        d.alpha = f64(k(mesh.perElementXPBDalphaMatrix, np.float64))
        d.beta = f64(k(mesh.perElementXPBDbeta, np.float64))
    else:
        d.mu = f64(k(mesh.mu, np.float64))
        d.lambda_ = f64(k(mesh.lam, np.float64))
        d.alpha1 = f64(k(mesh.alpha1, np.float64))
    d.precision, d.device = 1, 0
    return d


def _layer_desc(sets, num_rigids, is_rigid_element, is_elastic, is_boundary, is_rigid_vertex, vertex_body,
                layersMap, iterations, keep):
    arrs = [np.asfortranarray(sets, np.int32), np.ascontiguousarray(num_rigids, np.int32),
            np.asfortranarray(is_rigid_element, np.uint8), np.asfortranarray(is_elastic, np.uint8),
            np.asfortranarray(is_boundary, np.uint8), np.asfortranarray(is_rigid_vertex, np.uint8),
            np.asfortranarray(vertex_body, np.int32), np.ascontiguousarray(layersMap, np.int32),
            np.ascontiguousarray(iterations, np.int32)]
    keep.extend(arrs)
    s_, nr, rig, ela, bnd, rv, vb, lm, it = arrs
    d = LayerDesc()
    d.num_layers, d.num_columns = lm.size, s_.shape[1]
    d.layers_map, d.iterations = i32(lm), i32(it)
    d.is_elastic_element, d.is_rigid_element = u8(ela), u8(rig)
    d.rigid_body_sets, d.vertex_rigid_body = i32(s_), i32(vb)
    d.is_boundary_vertex, d.is_rigid_vertex = u8(bnd), u8(rv)
    d.num_rigids = i32(nr)
    return d


def _contacts(c, keep):
    out = Contacts()
    K = int(c.vertex_ids.size)
    out.num_contacts = K
    if K:
        arrs = [np.asfortranarray(c.normals.reshape(K, 3), float), np.asfortranarray(c.points.reshape(K, 3), float),
                np.ascontiguousarray(c.vertex_ids, np.int32), np.ascontiguousarray(c.compliance, float)]
        keep.extend(arrs)
        out.normals, out.point_colliders, out.vertex_ids, out.compliance = (f64(arrs[0]), f64(arrs[1]),
                                                                              i32(arrs[2]), f64(arrs[3]))
    return out


def params(integ, h):
    """mlx_solve_params from an integrator's properties (xpbdLayer3D.m:5-40)."""
    P = SolveParams()
    P.h = h
    P.boundary_compliance = integ.boundaryCompliance
    P.contact_resistance = integ.contactResistance
    P.run_until = integ.runUntilResSmallerThan
    P.give_up_threshold = integ.giveUpThreshold
    P.gravity_compliance = integ.gravityCompliance
    P.gravity = integ.Gravity
    P.stop_at_improvement_percent = integ.StopAtImprovementPercent
    P.compute_residuals = int(bool(integ.computeResiduals))
    P.hanging_stop = int(integ.hangingStop)
    P.give_up_enabled = int(bool(integ.giveUpEnabled))
    P.last_layer_give_up_enabled = int(bool(integ.LastLayerGiveUpEnabled))
    P.use_gravity_constraints = int(bool(integ.useGravityConstraints))
    P.use_rigid_contacts = int(bool(integ.useRigidContacts))
    P.contact_coloring = int(bool(getattr(integ, "contactColoring", False)))
    return P


def f64(a):
    return _p(a, C.c_double)


def i32(a):
    return _p(a, C.c_int32)


def u8(a):
    return _p(a, C.c_uint8)


# ---- single-function wrappers ------------------------------------------------
def stvk_constraint_grad(DmInv9, x12):
    lib = load()
    g = np.zeros(72)
    c = np.zeros(6)
    lib.orc_stvk_constraint_grad(f64(np.ascontiguousarray(DmInv9, float)), f64(np.ascontiguousarray(x12, float)),
                                 f64(g), f64(c))
    return g.reshape(12, 6).T.copy(), c  # gradC 6 x 12


def greedy_coloring(t, N):
    lib = load()
    tf = np.asfortranarray(t, dtype=np.int32)
    col = np.zeros(tf.shape[0], np.int32)
    nc = lib.orc_greedy_coloring(i32(tf), tf.shape[0], N, i32(col))
    return col, nc


def strain_rate_norms(t, DmInv, p, oldp, h):
    lib = load()
    tf = np.asfortranarray(t, dtype=np.int32)
    out = np.zeros(tf.shape[0])
    lib.orc_strain_rate_norms(i32(tf), tf.shape[0], f64(np.ascontiguousarray(DmInv)), f64(np.ascontiguousarray(p)),
                              f64(np.ascontiguousarray(oldp)), h, f64(out))
    return out


def union_find_layers(order, sorted_layers, forced, t, N):
    lib = load()
    tf = np.asfortranarray(t, dtype=np.int32)
    T = tf.shape[0]
    sl = np.ascontiguousarray(sorted_layers, float)
    sets = np.zeros((T, sl.size), np.int32, order="F")
    nr = np.zeros(sl.size, np.int32)
    lib.orc_union_find_layers(i32(np.ascontiguousarray(order, np.int32)), T, f64(sl), sl.size,
                              u8(np.ascontiguousarray(forced, np.uint8)), i32(tf), N, i32(sets), i32(nr))
    return sets, nr


def find_boundary_vertices(t, N, sets):
    lib = load()
    tf = np.asfortranarray(t, dtype=np.int32)
    sets = np.asfortranarray(sets, dtype=np.int32)
    T, L = sets.shape
    bnd = np.zeros((N, L), np.uint8, order="F")
    ela = np.zeros((T, L), np.uint8, order="F")
    rig = np.zeros((N, L), np.uint8, order="F")
    vb = np.zeros((N, L), np.int32, order="F")
    lib.orc_find_boundary_vertices(i32(tf), T, N, i32(sets), L, u8(bnd), u8(ela), u8(rig), i32(vb))
    return bnd, ela, rig, vb


def find_contacts_plane(p, normal, position, compliance=1e-4):
    lib = load()
    N = p.size // 3
    ids = np.zeros(N, np.int32); n = np.zeros(3 * N); q = np.zeros(3 * N); a = np.zeros(N)
    K = lib.orc_find_contacts_plane(f64(np.ascontiguousarray(p)), N, f64(np.asarray(normal, float)),
                                    f64(np.asarray(position, float)), compliance, i32(ids), f64(n), f64(q), f64(a))
    return (n[:3 * K].reshape(3, K).T.copy(), q[:3 * K].reshape(3, K).T.copy(), ids[:K].copy(), a[:K].copy())


def find_contacts_sphere(p, radius, center):
    lib = load()
    N = p.size // 3
    ids = np.zeros(N, np.int32); n = np.zeros(3 * N); q = np.zeros(3 * N); a = np.zeros(N)
    K = lib.orc_find_contacts_sphere(f64(np.ascontiguousarray(p)), N, radius, f64(np.asarray(center, float)),
                                     i32(ids), f64(n), f64(q), f64(a))
    return (n[:3 * K].reshape(3, K).T.copy(), q[:3 * K].reshape(3, K).T.copy(), ids[:K].copy(), a[:K].copy())


def find_contacts_platform(p, rotation, scale, center, compliance=1e-4):
    lib = load()
    N = p.size // 3
    ids = np.zeros(N, np.int32); n = np.zeros(3 * N); q = np.zeros(3 * N); a = np.zeros(N)
    K = lib.orc_find_contacts_platform(f64(np.ascontiguousarray(p)), N,
                                       f64(np.ascontiguousarray(np.asarray(rotation, float).reshape(9))),
                                       f64(np.asarray(scale, float)), f64(np.asarray(center, float)), compliance,
                                       i32(ids), f64(n), f64(q), f64(a))
    return (n[:3 * K].reshape(3, K).T.copy(), q[:3 * K].reshape(3, K).T.copy(), ids[:K].copy(), a[:K].copy())


def find_contacts(finders, p):
    """simulate3D's finder loop (3d/simulate3D.m:156-171) on the oracle's
    finders: the lists concatenated in finder order.  A finder is given by
    its kind (the MLX_OBSTACLE_* numbers of include/mlxpbd.h) and data."""
    lists = []
    for f in finders:
        if f.kind == OBSTACLE_SPHERE:
            r = find_contacts_sphere(p, f.radius, f.center)
        elif f.kind == OBSTACLE_BOX:
            r = find_contacts_platform(p, f.rotation, f.scale, f.center, f.compliance)
        elif f.kind == OBSTACLE_PLANE:
            r = find_contacts_plane(p, f.normal, f.center, f.compliance)
        else:
            raise ValueError(f"unknown finder kind {f.kind}")
        lists.append(ContactList(*r))
    return ContactList.concat(lists)


def layer_solve(mesh, ls, layersMap, iterations, P, contacts, xi, lambdai, oldp, oldOldp, f, resv, pinnedx,
                residual_in, sum_non_monitored_time=0.0, material="blocks", want_lambda=False):
    """orc_layer_solve (xpbdLayer3D.layerSolve restated) on numpy arrays.  `ls`
    carries the layer masks (rigidBodySetsPerLayer, numRigids,
    isRigidElement, isElasticElement, isBoundaryVertex, isRigidVertex,
    vertexRigidBody), `P` is a SolveParams, `contacts` a ContactList.
    Returns (xi, sumNonMonitoredTime, residualArray, runUntil, lambdai or
    None, total_iterations)."""
    lib = load()
    keep = []
    md = _mesh_desc(mesh, material, keep)
    ld = _layer_desc(ls.rigidBodySetsPerLayer, ls.numRigids, ls.isRigidElement, ls.isElasticElement,
                     ls.isBoundaryVertex, ls.isRigidVertex, ls.vertexRigidBody, layersMap, iterations, keep)
    ct = _contacts(contacts, keep)
    arr = lambda a: keep.append(np.ascontiguousarray(a, np.float64)) or keep[-1]
    xi_, oldp_, oo_, f_, rv_ = arr(xi), arr(oldp), arr(oldOldp), arr(f), arr(resv)
    px_ = arr(pinnedx if pinnedx is not None else np.zeros(0))
    rin = arr(residual_in)
    lam_ = None if lambdai is None else np.asfortranarray(lambdai, np.float64)
    inp = SolveInputs()
    inp.xi, inp.lambdai, inp.oldp, inp.old_oldp, inp.f = f64(xi_), f64(lam_), f64(oldp_), f64(oo_), f64(f_)
    inp.residualv, inp.pinnedx, inp.residual_in = f64(rv_), f64(px_), f64(rin)
    inp.residual_in_len = rin.size
    inp.sum_non_monitored_time = sum_non_monitored_time
    if not P.compute_residuals:
        cap = rin.size + 1
    else:
        cap = rin.size + 1 + max(0, P.hanging_stop) + int(np.sum(iterations)) + 100000
    out_xi = np.empty(xi_.size)
    if want_lambda and lam_ is None:
        raise ValueError("want_lambda needs lambdai")
    out_lam = np.zeros(lam_.shape, order="F") if want_lambda else None
    out_res = np.zeros(cap)
    out = SolveOutputs()
    out.xi, out.lambdai, out.residual, out.residual_capacity = f64(out_xi), f64(out_lam), f64(out_res), cap
    rc = lib.orc_layer_solve(C.byref(md), C.byref(ld), C.byref(P), C.byref(ct), C.byref(inp), C.byref(out))
    if rc != 0:
        raise RuntimeError(f"orc_layer_solve failed ({rc}): {lib.orc_last_error().decode()}")
    return (out_xi, out.sum_non_monitored_time, out_res[:out.residual_len].copy(), out.run_until, out_lam,
            out.total_iterations)


def contact_velocity_update(normals, vids, v, h, gravity, e):
    lib = load()
    v = np.ascontiguousarray(v, float).copy()
    K = int(np.asarray(vids).size)
    if K:
        nf = np.asfortranarray(np.asarray(normals, float).reshape(K, 3))
        lib.orc_contact_velocity_update(f64(nf), i32(np.ascontiguousarray(vids, np.int32)), K, f64(v), h, gravity, e)
    return v


def integrate(integ, mesh, h, contacts, cache, frame, material="blocks"):
    """Independent restatement of xpbdLayer3D.integrate (xpbdLayer3D.m:621-745)
    on the oracle's functions.  ``integ`` provides the integrator properties,
    ``cache`` has oldp/oldOldp; ``mesh.p``/``mesh.v`` are advanced in place.
    Returns the residual array and total iterations."""
    if cache.oldp is None or np.any(np.isnan(cache.oldp)) or frame == 1:
        cache.oldp = mesh.p.copy()
        integ.pinnedx = mesh.p[mesh.pinnedDOFs - 1].copy()
    N, T = mesh.N, mesh.T
    f = np.zeros(3 * N)
    f[2::3] += mesh.mass[2::3] * integ.Gravity
    f = f + integ.CustomForce
    if integ.customRigidSets is not None:
        sets = np.asfortranarray(integ.customRigidSets, dtype=np.int32)
        nr = np.array([sets[:, c].max(initial=0) for c in range(sets.shape[1])], np.int32)
    else:
        norms = strain_rate_norms(mesh.t, mesh.DmInv, mesh.p, cache.oldp, h)
        order = (np.argsort(norms, kind="stable") + 1).astype(np.int32)
        forced = np.zeros(T, np.uint8)
        forced[mesh.pinnedTets - 1] = 1
        sets, nr = union_find_layers(order, integ.sortedLayers, forced, mesh.t, N)
    bnd, ela, rig, vb = find_boundary_vertices(mesh.t, N, sets)

    class _Layers:  # buildLayers + findBoundaryVertices output (xpbdLayer3D.m:646-652)
        rigidBodySetsPerLayer, numRigids = sets, nr
        isRigidElement = np.asfortranarray((sets != 0).astype(np.uint8))
        isElasticElement, isBoundaryVertex, isRigidVertex, vertexRigidBody = ela, bnd, rig, vb
    cache.oldOldp = cache.oldp
    cache.oldp = mesh.p.copy()
    xi = mesh.p.copy()
    resv = mesh.v.copy()
    up = mesh.unpinnedDOFs - 1
    resv[up] += h * f[up] / mesh.mass[up]
    resv = (1 - integ.airDrag) * resv
    lam = np.zeros((T, 6), order="F")
    cl = ContactList(contacts.normals, contacts.points, contacts.vertex_ids, contacts.compliance)
    xi, snm, resArr, runUntil, _, iters = layer_solve(mesh, _Layers, integ.layersMap, integ.iterations,
                                                      params(integ, h), cl, xi, lam, cache.oldp,
                                                      cache.oldOldp, f, resv, integ.pinnedx, np.array([0.0]),
                                                      0.0, material)
    integ.runUntilResSmallerThan = runUntil
    mesh.v = (xi - cache.oldp) / h
    mesh.p = xi
    mesh.v = contact_velocity_update(contacts.normals, contacts.vertex_ids, mesh.v, h, integ.Gravity, 1e-2)
    return resArr, iters


# ---- the reference's own mex files (compiled unchanged, oracle/_ref) --------
class MexLib:
    """Calls the mexFunction of a library built against the headless mx
    runtime (multilayersolver2024_b200/mex), passing numpy arrays as mxArrays
    (bool -> logical, int32 -> int32, anything else -> double)."""

    def __init__(self, path):
        path = Path(path)
        if not path.exists():
            raise FileNotFoundError(path)
        lib = C.CDLL(str(path))
        vp = C.c_void_p
        lib.mxCreateDoubleMatrix.argtypes = [C.c_size_t, C.c_size_t, C.c_int]
        lib.mxCreateDoubleMatrix.restype = vp
        lib.mxCreateLogicalMatrix.argtypes = [C.c_size_t, C.c_size_t]
        lib.mxCreateLogicalMatrix.restype = vp
        lib.mxCreateNumericMatrix.argtypes = [C.c_size_t, C.c_size_t, C.c_int, C.c_int]
        lib.mxCreateNumericMatrix.restype = vp
        lib.mxGetData.argtypes = [vp]
        lib.mxGetData.restype = vp
        lib.mxGetM.argtypes = [vp]
        lib.mxGetM.restype = C.c_size_t
        lib.mxGetN.argtypes = [vp]
        lib.mxGetN.restype = C.c_size_t
        lib.mxDestroyArray.argtypes = [vp]
        lib.mxshim_call_mex.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp), C.c_char_p, C.c_size_t]
        lib.mxshim_call_mex.restype = C.c_int
        self.lib = lib

    def _make(self, a):
        a = np.asarray(a)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        m, n = a.shape
        if a.dtype == np.bool_:
            h = self.lib.mxCreateLogicalMatrix(m, n)
            buf = np.asfortranarray(a).view(np.uint8)
        elif a.dtype == np.int32:
            h = self.lib.mxCreateNumericMatrix(m, n, 12, 0)
            buf = np.asfortranarray(a)
        else:
            h = self.lib.mxCreateDoubleMatrix(m, n, 0)
            buf = np.asfortranarray(a, dtype=np.float64)
        if buf.size:
            C.memmove(self.lib.mxGetData(h), buf.ctypes.data, buf.nbytes)
        return h

    def __call__(self, nlhs, *args):
        vp = C.c_void_p
        prhs = (vp * len(args))(*[self._make(a) for a in args])
        plhs = (vp * nlhs)()
        err = C.create_string_buffer(1024)
        rc = self.lib.mxshim_call_mex(nlhs, plhs, len(args), prhs, err, 1024)
        for h in prhs:
            self.lib.mxDestroyArray(h)
        if rc:
            raise RuntimeError(err.value.decode())
        outs = []
        for h in plhs:
            m, n = self.lib.mxGetM(h), self.lib.mxGetN(h)
            out = np.zeros((m, n), order="F")
            if out.size:
                C.memmove(out.ctypes.data, self.lib.mxGetData(h), out.nbytes)
            self.lib.mxDestroyArray(h)
            outs.append(out)
        return outs


class RefMex(MexLib):
    """A reference mex file compiled unchanged into oracle/_ref."""

    def __init__(self, name):
        super().__init__(REF / f"{name}.so")


def ref_available(name="mexUnionFindByVertice"):
    return (REF / f"{name}.so").exists()
