"""Shared builders for the parity tests: one layerSolve input set, run through
the product (C ABI on the GPU) and the oracle with identical arguments."""
from __future__ import annotations

import numpy as np

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.mesh3d import Mesh3D, to_lame
from multilayersolver2024_b200.xpbd_layer3d import (ContactSet, Solver, XpbdLayer3D, call_layer_solve,
                                                    find_boundary_vertices, make_params, pack_contacts,
                                                    pack_layer_desc, union_find_layers)


def block_mesh(dims=(6, 3, 3), energy=_lib.MLX_ENERGY_STVK_VOIGT, seed=0, alpha1=0.0, edge=0.1, pin_x0=True):
    rng = np.random.default_rng(seed)
    V, T, _ = scenes.generate_beam(*dims, edge=edge)
    nt = T.shape[0]
    E = np.exp(rng.uniform(np.log(2e4), np.log(2e5), nt))
    mu, lam = to_lame(rng.uniform(0.25, 0.4, nt), E)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=alpha1, energy_type=energy)
    if pin_x0:
        m.pin(np.nonzero(np.isclose(V[:, 0], 0.0))[0] + 1)
    return m


def plane_contacts(p, normal, point, compliance=1e-4):
    from oracle import oracle as O  # the finder restatement of the oracle builds the inputs
    n, q, ids, a = O.find_contacts_plane(p, normal, point, compliance)
    return ContactSet(n, q, ids, a)


def sphere_contacts(p, radius, center):
    from oracle import oracle as O
    n, q, ids, a = O.find_contacts_sphere(p, radius, center)
    return ContactSet(n, q, ids, a)


class Case:
    """One layerSolve call: mesh, layers, params, contacts and step vectors."""

    def __init__(self, mesh, layers, iterations, seed=0, contacts=None, order=None, integ=None, h=0.01,
                 perturb=0.004, vel=0.3):
        rng = np.random.default_rng(seed)
        self.mesh = mesh
        self.integ = integ or XpbdLayer3D()
        self.integ.setLayers(layers)
        self.integ.iterations = list(iterations)
        self.h = h
        N, T = mesh.N, mesh.T
        self.xi = mesh.p + rng.normal(0, perturb, 3 * N)
        self.xi[mesh.pinnedDOFs - 1] = mesh.p[mesh.pinnedDOFs - 1]
        self.oldp = mesh.p + rng.normal(0, perturb, 3 * N)
        self.oldOldp = self.oldp.copy()
        self.resv = rng.normal(0, vel, 3 * N)
        self.resv[mesh.pinnedDOFs - 1] = 0
        self.f = np.zeros(3 * N)
        self.pinnedx = mesh.p[mesh.pinnedDOFs - 1].copy()
        self.lam = np.asfortranarray(rng.normal(0, 1e-6, (T, 6)))
        if order is None:
            order = rng.permutation(T) + 1
        forced = np.zeros(T, np.uint8)
        forced[mesh.pinnedTets - 1] = 1
        sets, nr = union_find_layers(mesh, order, self.integ.sortedLayers, forced)
        self.ls = find_boundary_vertices(mesh, sets, nr)
        self.contacts = contacts or ContactSet()

    def run(self, fn, handle, want_lambda=True):
        ld, k1 = pack_layer_desc(self.ls, self.integ.layersMap, self.integ.iterations)
        c = self.contacts
        cts, k2 = pack_contacts(c.normals, c.points, c.vertex_ids, c.compliance)
        rc, res = call_layer_solve(fn, handle, ld, make_params(self.integ, self.h), cts, self.xi, self.lam,
                                   self.oldp, self.oldOldp, self.f, self.resv, self.pinnedx, np.array([0.0]), 0.0,
                                   want_lambda)
        return rc, res

    def product(self, precision=_lib.MLX_FP64, material="blocks", solver=None):
        lib = _lib.load()
        s = solver or Solver(self.mesh, precision=precision, material=material)
        rc, res = self.run(lib.mlx_layer_solve, s.handle)
        _lib.check("mlx_layer_solve", rc, lib)
        return res

    def oracle(self, material="blocks", want_lambda=True):
        """The same call on the CPU oracle, marshalled by the oracle's own code."""
        from oracle import oracle as O
        c = self.contacts
        return O.layer_solve(self.mesh, self.ls, self.integ.layersMap, self.integ.iterations,
                             O.params(self.integ, self.h), O.ContactList(c.normals, c.points, c.vertex_ids, c.compliance),
                             self.xi, self.lam, self.oldp, self.oldOldp, self.f, self.resv, self.pinnedx,
                             np.array([0.0]), 0.0, material, want_lambda)


def rel_pos_err(a, b, mesh):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / mesh.bbox_diagonal())
