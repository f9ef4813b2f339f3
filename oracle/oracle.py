"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle.

Loads oracle/liboracle.so (the FP64 C++ restatement of the reference path, see
oracle.cpp) and, when built, the reference's own mex files compiled unchanged
against the headless mx runtime (oracle/_ref/*.so).  Only tests, the smoke
check and bench.py's CPU-baseline leg import this module; the product never
does.  ``integrate`` below is an independent restatement of
xpbdLayer3D.integrate (3d/integrator/xpbdLayer3D.m:621-745) built on the
oracle's C functions.
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
    from multilayersolver2024_b200._lib import (Contacts, LayerDesc, MeshDesc, SolveInputs, SolveOutputs,
                                                SolveParams)
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
    return a.ctypes.data_as(C.POINTER(t))


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
    finders: the lists concatenated in finder order."""
    from multilayersolver2024_b200 import _lib
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet
    sets = []
    for f in finders:
        if f.kind == _lib.MLX_OBSTACLE_PLANE:
            r = find_contacts_plane(p, f.normal, f.center, f.compliance)
        elif f.kind == _lib.MLX_OBSTACLE_SPHERE:
            r = find_contacts_sphere(p, f.radius, f.center)
        else:
            r = find_contacts_platform(p, f.rotation, f.scale, f.center, f.compliance)
        sets.append(ContactSet(*r))
    return ContactSet.concat(sets)


def layer_solve(mesh, ls, layersMap, iterations, params, contacts, xi, lambdai, oldp, oldOldp, f, resv, pinnedx,
                residual_in, sum_non_monitored_time=0.0, material="blocks", want_lambda=False):
    """orc_layer_solve with the same marshalling as the product call."""
    from multilayersolver2024_b200.xpbd_layer3d import call_layer_solve, mesh_desc, pack_layer_desc
    lib = load()
    md, keep = mesh_desc(mesh, 1, 0, material)
    ld, keep2 = pack_layer_desc(ls, layersMap, iterations)
    rc, res = call_layer_solve(lib.orc_layer_solve, C.byref(md), ld, params, contacts, xi, lambdai, oldp,
                               oldOldp, f, resv, pinnedx, residual_in, sum_non_monitored_time, want_lambda)
    if rc != 0:
        raise RuntimeError(f"orc_layer_solve failed ({rc}): {lib.orc_last_error().decode()}")
    return res


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
    from multilayersolver2024_b200.xpbd_layer3d import LayerSet, make_params, pack_contacts
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
    ls = LayerSet(sets, nr, np.asfortranarray((sets != 0).astype(np.uint8)), ela, bnd, rig, vb)
    cache.oldOldp = cache.oldp
    cache.oldp = mesh.p.copy()
    xi = mesh.p.copy()
    resv = mesh.v.copy()
    up = mesh.unpinnedDOFs - 1
    resv[up] += h * f[up] / mesh.mass[up]
    resv = (1 - integ.airDrag) * resv
    lam = np.zeros((T, 6), order="F")
    cts, keep = pack_contacts(contacts.normals, contacts.points, contacts.vertex_ids, contacts.compliance)
    xi, snm, resArr, runUntil, _, iters = layer_solve(mesh, ls, integ.layersMap, integ.iterations,
                                                      make_params(integ, h), cts, xi, lam, cache.oldp,
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
