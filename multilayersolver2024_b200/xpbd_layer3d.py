"""Host-side mirror of the reference integrator ``xpbdLayer3D``.

Same property names and defaults (3d/integrator/xpbdLayer3D.m:5-40,
2d/integrator/Integrator.m:17-27), same ``setLayers`` / ``buildLayers`` /
``integrate`` flow (xpbdLayer3D.m:595-745), and a static ``layerSolve`` with
the reference's argument order (xpbdLayer3D.m:44-93).  ``layerSolve`` runs on
the GPU through the C ABI (include/mlxpbd.h); there is no CPU fallback: if the
native library or the device is missing the call raises.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (Contacts, LayerDesc, MeshDesc, SolveInputs, SolveOutputs, SolveParams, check, f64, i32,
                   load, u8)
from .mesh3d import Mesh3D


def _F(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


@dataclass
class LayerSet:
    """buildLayers + findBoundaryVertices output (xpbdLayer3D.m:646-652)."""

    rigidBodySetsPerLayer: np.ndarray   # (T, Ls) int32, Fortran order
    numRigids: np.ndarray               # (Ls,) int32
    isRigidElement: np.ndarray          # (T, Ls) uint8
    isElasticElement: np.ndarray        # (T, Ls) uint8
    isBoundaryVertex: np.ndarray        # (N, Ls) uint8
    isRigidVertex: np.ndarray           # (N, Ls) uint8
    vertexRigidBody: np.ndarray         # (N, Ls) int32


def find_boundary_vertices(mesh: Mesh3D, sets: np.ndarray, num_rigids) -> LayerSet:
    """xpbdLayer2D.findBoundaryVertices through the native helper."""
    lib = load()
    sets = _F(sets, np.int32)
    T, L = sets.shape
    N = mesh.N
    bnd = np.zeros((N, L), np.uint8, order="F")
    ela = np.zeros((T, L), np.uint8, order="F")
    rig = np.zeros((N, L), np.uint8, order="F")
    vb = np.zeros((N, L), np.int32, order="F")
    check("mlx_find_boundary_vertices",
          lib.mlx_find_boundary_vertices(i32(mesh.t), T, N, i32(sets), L, u8(bnd), u8(ela), u8(rig), i32(vb)))
    return LayerSet(sets, np.asarray(num_rigids, np.int32), _F(sets != 0, np.uint8), ela, bnd, rig, vb)


def build_layers_device(solver, mesh: Mesh3D, p, oldp, h, sorted_layers, forced, order=None, dminv=None) -> LayerSet:
    """buildLayers + findBoundaryVertices on the device (``mlx_build_layers``):
    strain-rate order of p / oldp (with the mesh's DmInv, or `dminv`), or the
    given 1-based `order`; the same bits as the host builder."""
    lib = solver._lib
    sl = np.ascontiguousarray(sorted_layers, np.float64)
    L, T, N = sl.size, mesh.T, mesh.N
    fe = np.ascontiguousarray(forced, np.uint8)
    sets = np.zeros((T, L), np.int32, order="F")
    nr = np.zeros(L, np.int32)
    ela = np.zeros((T, L), np.uint8, order="F")
    bnd = np.zeros((N, L), np.uint8, order="F")
    rig = np.zeros((N, L), np.uint8, order="F")
    vb = np.zeros((N, L), np.int32, order="F")
    if order is None:
        pp, op = np.ascontiguousarray(p, np.float64), np.ascontiguousarray(oldp, np.float64)
        if dminv is not None:
            dm = np.ascontiguousarray(dminv, np.float64)
        else:
            # kept on the mesh: the library copies DmInv to the device once per host pointer
            if getattr(mesh, "_dminv_c", None) is None or mesh._dminv_c.base is not None:
                mesh._dminv_c = np.ascontiguousarray(mesh.DmInv, np.float64).copy()
            dm = mesh._dminv_c
        check("mlx_build_layers", lib.mlx_build_layers(solver.handle, f64(pp), f64(op), float(h), 0, None, f64(dm),
                                                       f64(sl), L, u8(fe), i32(sets), i32(nr), u8(ela), u8(bnd),
                                                       u8(rig), i32(vb)), lib)
    else:
        o = np.ascontiguousarray(order, np.int32)
        check("mlx_build_layers", lib.mlx_build_layers(solver.handle, None, None, float(h), 1, i32(o), None,
                                                       f64(sl), L, u8(fe), i32(sets), i32(nr), u8(ela), u8(bnd),
                                                       u8(rig), i32(vb)), lib)
    return LayerSet(sets, nr, _F(sets != 0, np.uint8), ela, bnd, rig, vb)


def strain_rate_norms(mesh: Mesh3D, p, oldp, h) -> np.ndarray:
    lib = load()
    out = np.zeros(mesh.T)
    check("mlx_strain_rate_norms",
          lib.mlx_strain_rate_norms(i32(mesh.t), mesh.T, f64(mesh.DmInv), f64(np.ascontiguousarray(p)),
                                    f64(np.ascontiguousarray(oldp)), float(h), f64(out)))
    return out


def union_find_layers(mesh: Mesh3D, order, sorted_layers, forced_elastic):
    lib = load()
    order = np.ascontiguousarray(order, dtype=np.int32)
    sl = np.ascontiguousarray(sorted_layers, dtype=np.float64)
    fe = np.ascontiguousarray(forced_elastic, dtype=np.uint8)
    sets = np.zeros((mesh.T, sl.size), np.int32, order="F")
    nr = np.zeros(sl.size, np.int32)
    check("mlx_union_find_layers",
          lib.mlx_union_find_layers(i32(order), mesh.T, f64(sl), sl.size, u8(fe), i32(mesh.t), mesh.N,
                                    i32(sets), i32(nr)))
    return sets, nr


def mesh_desc(mesh: Mesh3D, precision=_lib.MLX_FP32, device=0, material="blocks"):
    """The mlx_mesh_desc of a mesh; returns (desc, arrays to keep alive)."""
    keep = {}

    def k(name, a):
        keep[name] = a
        return a

    d = MeshDesc()
    d.num_vertices = mesh.N
    d.num_tets = mesh.T
    d.t = i32(k("t", _F(mesh.t, np.int32)))
    d.mass = f64(k("mass", np.ascontiguousarray(mesh.mass)))
    d.DmInv = f64(k("DmInv", np.ascontiguousarray(mesh.DmInv)))
    d.volume = f64(k("vol", np.ascontiguousarray(mesh.elV)))
    d.element_color = i32(k("color", np.ascontiguousarray(mesh.elementColor, np.int32)))
    d.num_colors = mesh.numColors
    d.pinned_dofs = i32(k("pin", np.ascontiguousarray(mesh.pinnedDOFs, np.int32)))
    d.num_pinned_dofs = int(mesh.pinnedDOFs.size)
    d.energy_type = mesh.energy_type
    if mesh.energy_type == _lib.MLX_ENERGY_STVK_VOIGT and material == "blocks":
        d.alpha = f64(k("alpha", np.ascontiguousarray(mesh.perElementXPBDalphaMatrix)))
        d.beta = f64(k("beta", np.ascontiguousarray(mesh.perElementXPBDbeta)))
    else:
        d.mu = f64(k("mu", np.ascontiguousarray(mesh.mu)))
        d.lambda_ = f64(k("lam", np.ascontiguousarray(mesh.lam)))
        d.alpha1 = f64(k("a1", np.ascontiguousarray(mesh.alpha1)))
    d.precision = precision
    d.device = device
    return d, keep


class Solver:
    """A device-resident copy of one mesh (``mlx_create``)."""

    def __init__(self, mesh: Mesh3D, precision=_lib.MLX_FP32, device=0, material="blocks"):
        lib = load()
        self._lib = lib
        self.mesh = mesh
        self.precision = precision
        d, keep = mesh_desc(mesh, precision, device, material)
        h = C.c_void_p()
        check("mlx_create", lib.mlx_create(C.byref(d), C.byref(h)), lib)
        self.handle = h

    def layer_pcg(self, pcg_iterations=50, every=35):
        """The PCG in the layer solve (``mlx_layer_pcg``): Newton-PCG
        corrections of the last layer, ``pcg_iterations`` PCG iterations each,
        before its Gauss-Seidel and after every ``every`` iterations;
        pcg_iterations = 0 turns them off.  The defaults are the fastest
        setting to residual 1e-4 on a 393 k-tet Neo-Hookean block that stays
        as close to the plain solve as 50 or 100 iterations every 50 sweeps
        (fewer PCG iterations per correction move the converged positions
        further from it)."""
        check("mlx_layer_pcg", self._lib.mlx_layer_pcg(self.handle, int(pcg_iterations), int(every)), self._lib)

    @property
    def launch_path(self) -> str:
        """How fixed-iteration layers are launched (``mlx_launch_path``)."""
        buf = C.create_string_buffer(256)
        self._lib.mlx_launch_path(self.handle, buf, 256)
        return buf.value.decode()

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.mlx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ResidentSim:
    """Device-resident stepping of one mesh (``mlx_sim_*``): the integrate step
    of xpbdLayer3D with a fixed layer description and the state kept on the GPU."""

    def __init__(self, solver: Solver, integ: "XpbdLayer3D", ls: LayerSet, h: float, p0=None, v0=None):
        self.solver = solver
        self._lib = solver._lib
        mesh = solver.mesh
        self._ld, self._keep = pack_layer_desc(ls, integ.layersMap, integ.iterations)
        P = make_params(integ, h)
        p0 = np.ascontiguousarray(mesh.p if p0 is None else p0, np.float64)
        v0 = np.ascontiguousarray(mesh.v if v0 is None else v0, np.float64)
        check("mlx_sim_init", self._lib.mlx_sim_init(solver.handle, C.byref(self._ld), C.byref(P), f64(p0), f64(v0),
                                                      float(integ.airDrag)), self._lib)

    def add_velocity(self, dofs, dv):
        d = np.ascontiguousarray(dofs, np.int32)
        v = np.ascontiguousarray(dv, np.float64)
        check("mlx_sim_add_velocity", self._lib.mlx_sim_add_velocity(self.solver.handle, i32(d), f64(v), d.size),
              self._lib)

    def step(self, n=1, graph=True, timed=False):
        ms = C.c_double(0.0)
        check("mlx_sim_step", self._lib.mlx_sim_step(self.solver.handle, int(n), int(bool(graph)),
                                                      C.byref(ms) if timed else None), self._lib)
        return ms.value if timed else None

    def state(self):
        N = self.solver.mesh.N
        p, v = np.zeros(3 * N), np.zeros(3 * N)
        check("mlx_sim_get_state", self._lib.mlx_sim_get_state(self.solver.handle, f64(p), f64(v)), self._lib)
        return p, v

    def sweep_timing(self, on=True):
        check("mlx_sim_sweep_timing", self._lib.mlx_sim_sweep_timing(self.solver.handle, int(bool(on))), self._lib)

    def sweep_stats(self, reset=True):
        ms, b, n = C.c_double(), C.c_double(), C.c_longlong()
        check("mlx_sim_sweep_stats", self._lib.mlx_sim_sweep_stats(self.solver.handle, C.byref(ms), C.byref(b),
                                                                    C.byref(n), int(bool(reset))), self._lib)
        return ms.value, b.value, n.value

    @property
    def launches_per_step(self):
        return int(self._lib.mlx_sim_launches_per_step(self.solver.handle))

    def set_obstacles(self, finders, restitution=1e-2):
        """Contacts with analytic obstacles detected on the device every step
        (``mlx_sim_set_obstacles``); restitution as contactVelocityUpdate's e."""
        from .contacts import pack_finders
        arr, n = pack_finders(finders)
        self._obstacles = arr
        check("mlx_sim_set_obstacles", self._lib.mlx_sim_set_obstacles(self.solver.handle, C.cast(arr, C.c_void_p), n,
                                                                        float(restitution)), self._lib)

    def monitor(self, capacity=16384):
        """Residual monitor of the last step (``mlx_sim_monitor``): the
        residual array, total projectGS iterations, runUntilResSmallerThan
        and a status (0 ok)."""
        ra = np.zeros(capacity)
        n, it, st = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        ru = C.c_double(0)
        check("mlx_sim_monitor", self._lib.mlx_sim_monitor(self.solver.handle, f64(ra), capacity, C.byref(n),
                                                            C.byref(it), C.byref(ru), C.byref(st)), self._lib)
        return ra[:min(n.value, capacity)].copy(), it.value, ru.value, st.value

    def warm_start(self, record=False, mode=0, net=None, feature_norm=None, output_norm=None, corrections=None,
                   fallback_residual=1e-3):
        """Learned warm start (``mlx_sim_warm_start``): mode 0 off, 1 the
        perceptron ``net`` with feature / output normalisation ((mean, std)
        pairs of 44 and 8 values), 2 fixed ``corrections`` (clusters x 8).
        Clusters whose predicted rigid-fit residual exceeds
        ``fallback_residual`` (m; <= 0: never) keep the plain start.
        ``record`` keeps every step's features and targets.  Returns the
        number of clusters."""
        from ._lib import f32
        fm, fs = (None, None) if feature_norm is None else (np.ascontiguousarray(feature_norm[0], np.float32),
                                                          np.ascontiguousarray(feature_norm[1], np.float32))
        om, osd = (None, None) if output_norm is None else (np.ascontiguousarray(output_norm[0], np.float32),
                                                           np.ascontiguousarray(output_norm[1], np.float32))
        corr = None if corrections is None else np.ascontiguousarray(corrections, np.float32)
        self._ws_keep = (net, fm, fs, om, osd, corr)
        nb = C.c_int32(0)
        check("mlx_sim_warm_start", self._lib.mlx_sim_warm_start(
            self.solver.handle, int(bool(record)), int(mode), net.handle if net is not None else None,
            float(fallback_residual), f32(fm), f32(fs), f32(om), f32(osd), f32(corr), C.byref(nb)), self._lib)
        self._ws_nb = nb.value
        return nb.value

    def multiplier_warm_start(self, on=True, scale=1.0, extrapolation=0.0):
        """Multiplier warm start (``mlx_sim_multiplier_warm_start``): the
        last layer of each step starts from scale * lambda_{n-1} +
        extrapolation * (lambda_{n-1} - lambda_{n-2}) with the matching
        position shift."""
        check("mlx_sim_multiplier_warm_start", self._lib.mlx_sim_multiplier_warm_start(
            self.solver.handle, int(bool(on)), float(scale), float(extrapolation)), self._lib)

    def warm_start_records(self):
        """Features (clusters x 44) and targets (clusters x 8) of the last step."""
        return self._ws_fetch()[:2]

    def warm_start_fallbacks(self):
        """Clusters that kept the plain start in the last step (gated)."""
        return self._ws_fetch()[2]

    def _ws_fetch(self):
        from ._lib import f32
        nb = self._ws_nb
        feat = np.zeros((nb, 44), np.float32)
        tgt = np.zeros((nb, 8), np.float32)
        n, fb = C.c_int32(0), C.c_int32(0)
        check("mlx_sim_warm_start_fetch", self._lib.mlx_sim_warm_start_fetch(self.solver.handle, f32(feat), f32(tgt),
                                                                              nb, C.byref(n), C.byref(fb)), self._lib)
        return feat, tgt, fb.value

    def contact_count(self):
        """Contact vertices of the last step."""
        n = C.c_int32(0)
        check("mlx_sim_contact_count", self._lib.mlx_sim_contact_count(self.solver.handle, C.byref(n)), self._lib)
        return n.value

    def autotune(self, reps=10):
        """Per-colour tile autotuner (``mlx_sim_autotune``); returns one
        step's device time in ms before and after tuning."""
        b, a = C.c_double(), C.c_double()
        check("mlx_sim_autotune", self._lib.mlx_sim_autotune(self.solver.handle, int(reps), C.byref(b), C.byref(a)),
              self._lib)
        return b.value, a.value


def pack_layer_desc(ls: LayerSet, layersMap, iterations):
    keep = [ls]
    lm = np.ascontiguousarray(layersMap, np.int32)
    it = np.ascontiguousarray(iterations, np.int32)
    keep += [lm, it]
    d = LayerDesc()
    d.num_layers = lm.size
    d.num_columns = ls.rigidBodySetsPerLayer.shape[1]
    d.layers_map = i32(lm)
    d.iterations = i32(it)
    d.is_elastic_element = u8(ls.isElasticElement)
    d.is_rigid_element = u8(ls.isRigidElement)
    d.rigid_body_sets = i32(ls.rigidBodySetsPerLayer)
    d.vertex_rigid_body = i32(ls.vertexRigidBody)
    d.is_boundary_vertex = u8(ls.isBoundaryVertex)
    d.is_rigid_vertex = u8(ls.isRigidVertex)
    nr = np.ascontiguousarray(ls.numRigids, np.int32)
    keep.append(nr)
    d.num_rigids = i32(nr)
    return d, keep


def pack_contacts(normals, points, vertex_ids, compliance):
    c = Contacts()
    K = 0 if vertex_ids is None else int(np.asarray(vertex_ids).size)
    keep = []
    c.num_contacts = K
    if K:
        n = _F(np.asarray(normals).reshape(K, 3), np.float64)
        p = _F(np.asarray(points).reshape(K, 3), np.float64)
        v = np.ascontiguousarray(vertex_ids, np.int32).ravel()
        a = np.ascontiguousarray(compliance, np.float64).ravel()
        keep = [n, p, v, a]
        c.normals, c.point_colliders, c.vertex_ids, c.compliance = f64(n), f64(p), i32(v), f64(a)
    return c, keep


def make_params(integ: "XpbdLayer3D", h: float) -> SolveParams:
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


def call_layer_solve(fn, solver_or_desc, layer_desc, params, contacts, xi, lambdai, oldp, oldOldp, f,
                     residualv, pinnedx, residual_in, sum_non_monitored_time=0.0, want_lambda=False,
                     residual_capacity=None):
    """Marshal one layerSolve call for ``fn`` (mlx_layer_solve or the same
    signature); returns (xi, sumNonMonitoredTime, residualArray, runUntil,
    lambdai or None, total_iterations)."""
    N3 = xi.size
    keep = []
    arr = lambda a, dt=np.float64: keep.append(np.ascontiguousarray(a, dt)) or keep[-1]
    xi_ = arr(xi)
    lam_ = None if lambdai is None else _F(lambdai, np.float64)  # None: zeros
    keep.append(lam_)
    oldp_ = arr(oldp); oo_ = arr(oldOldp); f_ = arr(f); rv_ = arr(residualv)
    px_ = arr(pinnedx if pinnedx is not None else np.zeros(0)); rin = arr(residual_in)
    inp = SolveInputs()
    inp.xi, inp.lambdai, inp.oldp, inp.old_oldp, inp.f = f64(xi_), f64(lam_), f64(oldp_), f64(oo_), f64(f_)
    inp.residualv, inp.pinnedx, inp.residual_in = f64(rv_), f64(px_), f64(rin)
    inp.residual_in_len = rin.size
    inp.sum_non_monitored_time = sum_non_monitored_time
    if residual_capacity:
        cap = residual_capacity
    elif not params.compute_residuals:
        cap = rin.size + 1  # the residual array comes back as it went in
    else:
        cap = (rin.size + 1 + max(0, params.hanging_stop if params.hanging_stop >= 0 else 0) +
               sum(int(layer_desc.iterations[i]) for i in range(layer_desc.num_layers)) + 100000)
    out_xi = np.empty(N3)  # every value is written
    if want_lambda and lam_ is None:
        raise ValueError("want_lambda needs lambdai")
    out_lam = np.zeros(lam_.shape, order="F") if want_lambda else None
    out_res = np.zeros(cap)
    out = SolveOutputs()
    out.xi = f64(out_xi)
    out.lambdai = f64(out_lam)
    out.residual = f64(out_res)
    out.residual_capacity = cap
    rc = fn(solver_or_desc, C.byref(layer_desc), C.byref(params), C.byref(contacts), C.byref(inp), C.byref(out))
    return rc, (out_xi, out.sum_non_monitored_time, out_res[:out.residual_len].copy(), out.run_until,
                out_lam, out.total_iterations)


@dataclass
class StepCache:
    """The per-mesh cache fields integrate touches (3d/tools/solve/setupCache.m:41-42)."""

    oldp: np.ndarray = None
    oldOldp: np.ndarray = None
    residualArray: np.ndarray = None
    layers: np.ndarray = None


@dataclass
class ContactSet:
    normals: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    points: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    vertex_ids: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    compliance: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @staticmethod
    def concat(sets):
        sets = [s for s in sets if s is not None and s.vertex_ids.size]
        if not sets:
            return ContactSet()
        return ContactSet(np.concatenate([s.normals for s in sets]), np.concatenate([s.points for s in sets]),
                          np.concatenate([s.vertex_ids for s in sets]).astype(np.int32),
                          np.concatenate([s.compliance for s in sets]))


def _any_nan(lib, x) -> bool:
    """any(isnan(x)) (xpbdLayer3D.m:629) in one native pass."""
    x = np.ascontiguousarray(x, np.float64)
    r = lib.mlx_any_nan(x.size, f64(x))
    if r < 0:
        check("mlx_any_nan", -r, lib)
    return bool(r)


def contact_velocity_update(normals, vertex_ids, v, h, gravity, dim=3, restitution=1e-5):
    """xpbdLayer2D.contactVelocityUpdate (2d/integrator/xpbdLayer2D.m:577-603)
    in one native pass (``mlx_contact_velocity_update``); returns a new array
    (`v` itself without contacts)."""
    K = normals.shape[0]
    if K == 0:
        return v
    lib = load()
    n = np.asfortranarray(np.asarray(normals, np.float64).reshape(K, dim))
    ids = np.ascontiguousarray(vertex_ids, np.int32).ravel()[:K]
    vin = np.ascontiguousarray(v, np.float64)
    out = np.empty(vin.size)
    check("mlx_contact_velocity_update", lib.mlx_contact_velocity_update(K, f64(n), i32(ids), dim, vin.size, f64(vin),
                                                                         float(h), float(gravity), float(restitution),
                                                                         f64(out)), lib)
    return out


class XpbdLayer3D:
    """xpbdLayer3D: the multi-layer XPBD integrator."""

    def __init__(self):
        # Integrator base (2d/integrator/Integrator.m:17-27)
        self.Gravity = -9.8
        self.CustomForce = 0.0
        # xpbdLayer3D properties (xpbdLayer3D.m:5-40)
        self.iterations = [10]
        self.layers = [0]
        self.sortedLayers = [0]
        self.layersMap = [1]
        self.boundaryCompliance = 1e-8
        self.computeResiduals = False
        self.energyType = 2
        self.giveUpEnabled = False
        self.LastLayerGiveUpEnabled = False
        self.giveUpThreshold = 0.0
        self.contactResistance = 0.5
        self.gravityCompliance = 0.001
        self.LayerOrderingType = 0
        self.runUntilResSmallerThan = -1.0
        self.hangingStop = 1000
        self.useGravityConstraints = True
        self.runOnGPU = True
        self.airDrag = 0.0
        self.useRigidContacts = True
        self.StopAtImprovementPercent = 0.0
        # where buildLayers runs for strain-rate / random layers: "device"
        # (mlx_build_layers) or "host" (the native host helpers)
        self.layerBuilder = "device"
        # elastic contacts projected inside the colour sweep (mlx_solve_params
        # contact_coloring); False keeps the reference's order
        self.contactColoring = False
        self.pinnedx = None
        # fixed rigid sets per sorted layer column (LayerOrderingType 4, "custom")
        self.customRigidSets = None
        self.rng = np.random.default_rng(0)
        self.precision = _lib.MLX_FP32
        self.device = 0
        self._solvers = {}
        self.last_total_iterations = 0

    def setLayers(self, layers):
        """xpbdLayer3D.setLayers (:595-599): sortedLayers = unique(layers),
        layersMap = its inverse index (1-based)."""
        self.layers = list(layers)
        s, ic = np.unique(np.asarray(layers, dtype=np.float64), return_inverse=True)
        self.sortedLayers = s.tolist()
        self.layersMap = (ic + 1).astype(np.int32).tolist()

    def solver(self, mesh: Mesh3D) -> Solver:
        key = id(mesh)
        s = self._solvers.get(key)
        if s is None or s.mesh is not mesh:
            s = Solver(mesh, precision=self.precision, device=self.device)
            self._solvers[key] = s
        return s

    @property
    def customRigidSets(self):
        """Fixed rigid sets per sorted layer column (T x Ls), or None.  Stored
        as a read-only copy when assigned -- the value semantics of the
        reference's MATLAB property: changing them means assigning them."""
        return self._custom_sets

    @customRigidSets.setter
    def customRigidSets(self, sets):
        if sets is None:
            self._custom_sets = None
        else:
            a = np.array(sets, dtype=np.int32, order="F", copy=True)
            a.flags.writeable = False
            self._custom_sets = a
        self._custom_counts = None

    def buildLayers(self, mesh: Mesh3D, cache: StepCache, h: float):
        """xpbdLayer3D.buildLayers (:601-619)."""
        if self.customRigidSets is not None:
            sets = self.customRigidSets
            if self._custom_counts is None:
                self._custom_counts = np.asarray([int(sets[:, c].max(initial=0)) for c in range(sets.shape[1])],
                                                 np.int32)
            return sets, self._custom_counts
        if self.LayerOrderingType == 1:
            order = self.rng.permutation(mesh.T) + 1
        else:
            norms = strain_rate_norms(mesh, mesh.p, cache.oldp, h)
            order = np.argsort(norms, kind="stable") + 1
        forced = np.zeros(mesh.T, np.uint8)
        forced[mesh.pinnedTets - 1] = 1
        return union_find_layers(mesh, order, self.sortedLayers, forced)

    @staticmethod
    def layerSolve(isElasticElement, isRigidElement, rigidBodySetsPerLayer, vertexRigidBody, isBoundaryVertex,
                   isRigidVertex, xi, lambdai, sumNonMonitoredTime, h, numRigids, residualArray,
                   boundaryCompliance, contactResistance, contactCompliance, iterations, layers,
                   runUntilResSmallerThan, computeResiduals, hangingStop, giveUpEnabled, giveUpThreshold,
                   LastLayerGiveUpEnabled, useGravityConstraints, oldp, oldOldp, contactNormals, pointColliders,
                   contactVertexID, mass, T, unpinnedDOFs, pinnedDOFs, DmInv, perElementXPBDalphaMatrix,
                   perElementXPBDalphaInvMatrix, elementColor, elementDOFs, numColors, f, layersMap,
                   gravityCompliance, gravity, residualv, perElementXPBDBeta, volume, runOnGPU, useRigidContacts,
                   StopAtImprovementPercent, pinnedx, *, solver: Solver):
        """xpbdLayer3D.layerSolve (xpbdLayer3D.m:44-232) on the GPU.  Argument
        order and meaning as the reference; the mesh arrays must be those the
        ``solver`` was created from.  Returns (xi, sumNonMonitoredTime,
        residualArray, runUntilResSmallerThan)."""
        ls = LayerSet(_F(rigidBodySetsPerLayer, np.int32), np.asarray(numRigids, np.int32),
                      _F(isRigidElement, np.uint8), _F(isElasticElement, np.uint8), _F(isBoundaryVertex, np.uint8),
                      _F(isRigidVertex, np.uint8), _F(vertexRigidBody, np.int32))
        ld, keep = pack_layer_desc(ls, layersMap, iterations)
        P = SolveParams()
        P.h, P.boundary_compliance, P.contact_resistance = h, boundaryCompliance, contactResistance
        P.run_until, P.give_up_threshold = runUntilResSmallerThan, giveUpThreshold
        P.gravity_compliance, P.gravity = gravityCompliance, gravity
        P.stop_at_improvement_percent = StopAtImprovementPercent
        P.compute_residuals, P.hanging_stop = int(bool(computeResiduals)), int(hangingStop)
        P.give_up_enabled, P.last_layer_give_up_enabled = int(bool(giveUpEnabled)), int(bool(LastLayerGiveUpEnabled))
        P.use_gravity_constraints, P.use_rigid_contacts = int(bool(useGravityConstraints)), int(bool(useRigidContacts))
        cts, keep2 = pack_contacts(contactNormals, pointColliders, contactVertexID,
                                   np.asarray(contactCompliance).ravel())
        lib = load()
        rc, res = call_layer_solve(lib.mlx_layer_solve, solver.handle, ld, P, cts, xi, lambdai, oldp, oldOldp, f,
                                   residualv, pinnedx, residualArray, sumNonMonitoredTime)
        check("mlx_layer_solve", rc, lib)
        return res[0], res[1], res[2], res[3]

    def _boundary_vertices(self, mesh, sets, num_rigids):
        """findBoundaryVertices of this step's sets.  Fixed custom sets give
        the same result every step, so it is kept while they and the mesh
        stay the same."""
        if self.customRigidSets is None:
            return find_boundary_vertices(mesh, sets, num_rigids)
        c = getattr(self, "_fbv", None)
        if c is not None and c[0] is mesh and c[1] is sets:  # the stored sets are read-only
            return c[2]
        ls = find_boundary_vertices(mesh, sets, num_rigids)
        self._fbv = (mesh, sets, ls)
        return ls

    def _layer_desc(self, ls):
        """pack_layer_desc of this step, kept while the layer set object, the
        layers map and the iteration counts stay the same."""
        key = (tuple(np.ravel(self.layersMap).tolist()), tuple(np.ravel(self.iterations).tolist()))
        c = getattr(self, "_ld", None)
        if c is not None and c[0] is ls and c[1] == key:
            return c[2], c[3]
        ld, keep = pack_layer_desc(ls, self.layersMap, self.iterations)
        self._ld = (ls, key, ld, keep)
        return ld, keep

    def integrate(self, mesh: Mesh3D, h: float, contacts: ContactSet, cache: StepCache, frame: int):
        """xpbdLayer3D.integrate (xpbdLayer3D.m:621-745)."""
        assert len(self.layers) and len(self.iterations)
        assert self.boundaryCompliance < 1e-5
        sumNonMonitoredTime = 0.0
        lib = load()
        if cache.oldp is None or frame == 1 or _any_nan(lib, cache.oldp):
            cache.oldp = mesh.p.copy()
            self.pinnedx = mesh.p[mesh.pinnedDOFs - 1].copy()
        tic = time.perf_counter()
        # forces and residual velocity (xpbdLayer3D.m:638-643, 662-664) in one
        # native pass; the pinned DOFs get no h f / m term
        n3 = 3 * mesh.N
        # the residual velocity only feeds layerSolve (which copies it), so
        # one buffer serves every step: no fresh pages to fault in
        resv = getattr(self, "_resv_buf", None)
        if resv is None or resv.size != n3:
            resv = self._resv_buf = np.empty(n3)
        f = np.empty(n3)
        cf = self.CustomForce
        cfv = None if np.ndim(cf) == 0 else np.ascontiguousarray(np.broadcast_to(cf, (n3,)), np.float64)
        pins = np.ascontiguousarray(mesh.pinnedDOFs, np.int32)
        check("mlx_integrate_begin", lib.mlx_integrate_begin(
            n3, float(h), float(self.Gravity), float(self.airDrag), float(cf) if cfv is None else 0.0, f64(cfv),
            f64(np.ascontiguousarray(mesh.mass, np.float64)), f64(np.ascontiguousarray(mesh.v, np.float64)),
            i32(pins), pins.size, f64(f), f64(resv)), lib)
        mesh.f = f
        if self.customRigidSets is None and self.layerBuilder == "device":
            # buildLayers and findBoundaryVertices in one device call
            forced = np.zeros(mesh.T, np.uint8)
            forced[mesh.pinnedTets - 1] = 1
            order = self.rng.permutation(mesh.T).astype(np.int32) + 1 if self.LayerOrderingType == 1 else None
            ls = build_layers_device(self.solver(mesh), mesh, mesh.p, cache.oldp, h, self.sortedLayers, forced,
                                     order)
        else:
            sets, numRigids = self.buildLayers(mesh, cache, h)
            ls = self._boundary_vertices(mesh, sets, numRigids)
        cache.layers = ls.isRigidElement
        cache.oldOldp = cache.oldp
        cache.oldp = mesh.p.copy()
        xi = mesh.p  # layerSolve only reads it; mesh.p is replaced by its result
        lambdai = None  # zeros(T, 6) (xpbdLayer3D.m:666): the library zeroes them on the device
        residualArray = np.array([0.0])
        ld, keep = self._layer_desc(ls)
        cts, keep2 = pack_contacts(contacts.normals, contacts.points, contacts.vertex_ids, contacts.compliance)
        rc, res = call_layer_solve(lib.mlx_layer_solve, self.solver(mesh).handle, ld, make_params(self, h), cts,
                                   xi, lambdai, cache.oldp, cache.oldOldp, f, resv, self.pinnedx, residualArray,
                                   sumNonMonitoredTime)
        check("mlx_layer_solve", rc, lib)
        xi, sumNonMonitoredTime, residualArray, self.runUntilResSmallerThan = res[0], res[1], res[2], res[3]
        self.last_total_iterations = res[5]
        cache.residualArray = residualArray[1:]
        v = np.empty(n3)
        check("mlx_integrate_end", lib.mlx_integrate_end(n3, float(h), f64(xi), f64(cache.oldp), f64(v)), lib)
        mesh.v = v
        mesh.p = xi
        mesh.v = contact_velocity_update(contacts.normals, contacts.vertex_ids, mesh.v, h, self.Gravity, 3, 1e-2)
        integrate_forces = time.perf_counter() - tic - sumNonMonitoredTime
        return {"integrateForces": integrate_forces, "residual": float(residualArray[-1]),
                "residualPreSolve": float(residualArray[0]), "iterations": res[5]}
