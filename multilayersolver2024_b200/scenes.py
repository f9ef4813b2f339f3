"""Synthetic scenes of the benchmark configurations (seeded, no datasets).

``generate_beam`` follows the reference's cube-grid generator
(3d/tools/meshReaders/generateBeam.m:1-41): vertices on a unit grid, six tets
per cube with the same corner pattern.  Two deliberate differences, both
required by the solver: the long axis is x (so the x = 0 face can be pinned),
and a tet whose corner order gives det(Dm) < 0 has its last two corners
swapped, because the reference's pattern leaves half the tets inverted and its
mass/volume precompute assumes positive volumes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .mesh3d import Mesh3D, merge_meshes, to_lame


def generate_beam(nx: int, ny: int, nz: int, edge: float = 1.0, origin=(0.0, 0.0, 0.0)):
    """Cube grid of nx*ny*nz cubes, 6 tets per cube.  Returns V (N, 3) and
    1-based T (6*nx*ny*nz, 4) plus the (ix, iy, iz) cube of every tet."""
    ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # vertex id = iz*(ny+1)*(nx+1) + iy*(nx+1) + ix (x fastest)
    V = np.zeros(((nx + 1) * (ny + 1) * (nz + 1), 3))
    vid = lambda a, b, c: c * (ny + 1) * (nx + 1) + b * (nx + 1) + a
    V[vid(ix, iy, iz).ravel()] = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1) * edge
    V += np.asarray(origin, dtype=np.float64)
    cx, cy, cz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    # cubes in generateBeam's loop order: z outer, then y, then x
    order = np.lexsort((cx.ravel(), cy.ravel(), cz.ravel()))
    cx, cy, cz = cx.ravel()[order], cy.ravel()[order], cz.ravel()[order]
    v1 = vid(cx, cy, cz); v2 = vid(cx + 1, cy, cz); v3 = vid(cx, cy + 1, cz); v4 = vid(cx + 1, cy + 1, cz)
    v5 = vid(cx, cy, cz + 1); v6 = vid(cx + 1, cy, cz + 1); v7 = vid(cx, cy + 1, cz + 1)
    v8 = vid(cx + 1, cy + 1, cz + 1)
    pattern = [(v1, v2, v3, v6), (v2, v3, v4, v6), (v3, v5, v6, v7), (v3, v6, v7, v8), (v1, v3, v5, v6),
               (v3, v4, v6, v8)]
    T = np.stack([np.stack(p, 1) for p in pattern], 1).reshape(-1, 4)
    cube = np.repeat(np.stack([cx, cy, cz], 1), 6, axis=0)
    D = np.stack([V[T[:, k]] - V[T[:, 0]] for k in (1, 2, 3)], axis=2)
    neg = np.linalg.det(D) < 0
    T[neg, 2], T[neg, 3] = T[neg, 3].copy(), T[neg, 2].copy()
    return V, (T + 1).astype(np.int32), cube


def cluster_rigid_sets(cube: np.ndarray, dims, cluster: int, forced_elastic: np.ndarray) -> np.ndarray:
    """Fixed rigid clusters of cluster^3 cubes for a coarse layer.  A cube on
    an internal cluster seam (index % cluster == cluster-1, not on the outer
    face) stays elastic, so neighbouring clusters never share a vertex and
    each cluster is exactly one body; forced-elastic (pinned) tets stay
    elastic as buildLayers does (xpbdLayer3D.m:614-615).  Body ids are
    numbered 1.. by their first tet, as mexUnionFindByVertice's copyLayer."""
    dims = np.asarray(dims)
    seam = np.zeros(cube.shape[0], dtype=bool)
    for a in range(3):
        seam |= (cube[:, a] % cluster == cluster - 1) & (cube[:, a] != dims[a] - 1)
    key = (cube[:, 0] // cluster) + (dims[0] // cluster + 1) * (
        (cube[:, 1] // cluster) + (dims[1] // cluster + 1) * (cube[:, 2] // cluster))
    rigid = ~seam & ~forced_elastic
    sets = np.zeros(cube.shape[0], dtype=np.int32)
    label = {}
    for e in np.nonzero(rigid)[0]:
        k = int(key[e])
        if k not in label:
            label[k] = len(label) + 1
        sets[e] = label[k]
    return sets


@dataclass
class Scene:
    name: str
    mesh: Mesh3D
    h: float
    steps: int
    layers: list
    iterations: list
    gravity: float = -9.81
    custom_sets: np.ndarray = None       # (T, Lsorted) fixed rigid sets, or None
    contact_finders: list = field(default_factory=list)
    impulse: tuple = None                # (dofs 1-based, dv) applied before step 1
    settings: dict = field(default_factory=dict)


def config1(energy=_lib.MLX_ENERGY_STVK_VOIGT) -> Scene:
    """Plain single-layer XPBD cantilever: 8x2x2 cubes of 0.1 m (81 vertices,
    192 tets), E = 1e5, nu = 0.3, rho = 1000, x = 0 face pinned, dt = 0.01,
    20 iterations, layers [0], 200 steps, undamped (alpha1 = 0)."""
    V, T, cube = generate_beam(8, 2, 2, 0.1)
    mu, lam = to_lame(0.3, 1e5)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=energy)
    m.pin(np.nonzero(np.isclose(V[:, 0], 0.0))[0] + 1)
    return Scene("config1_cantilever_8x2x2", m, 0.01, 200, [0], [20])


def config1_replicated(copies: int = 16384, per_row: int = 128, energy=_lib.MLX_ENERGY_STVK_VOIGT) -> Scene:
    """`copies` independent copies of the config-1 cantilever in one mesh, laid
    out as Mesh3D.mergeMesh lays out its parts (vertices and tets
    concatenated, tets offset by the vertices before them, colours overlaid:
    first-fit colouring of disjoint parts gives every part its solo colours).
    Copies sit on a grid in the y-z plane, 0.4 m apart, `per_row` per row;
    every copy's x = 0 face is pinned.  Settings as config1 (one layer [0],
    20 iterations, dt = 0.01, undamped); the rigid sets are given (all zero)
    so a step builds no layers."""
    V1, T1, _ = generate_beam(8, 2, 2, 0.1)
    n1, t1 = V1.shape[0], T1.shape[0]
    k = np.arange(copies)
    off = np.stack([np.zeros(copies), 0.4 * (k % per_row), 0.4 * (k // per_row)], 1)
    V = (V1[None, :, :] + off[:, None, :]).reshape(-1, 3)
    T = (T1[None, :, :].astype(np.int64) + (n1 * k)[:, None, None]).reshape(-1, 4).astype(np.int32)
    mu, lam = to_lame(0.3, 1e5)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=energy)
    m.pin(np.nonzero(np.isclose(V[:, 0], 0.0))[0] + 1)
    m.part_vertex_offsets = n1 * np.arange(copies + 1)
    m.part_tet_offsets = t1 * np.arange(copies + 1)
    sets = np.zeros((m.T, 1), np.int32, order="F")
    return Scene(f"config1_cantilever_8x2x2_x{copies}", m, 0.01, 200, [0], [20], custom_sets=sets)


def config2(seed: int = 2, nx=64, ny=16, nz=16, cluster=8, energy=_lib.MLX_ENERGY_NEOHOOKEAN) -> Scene:
    """Plain multi-layer Neo-Hookean block: 64x16x16 cubes (18,785 vertices,
    98,304 tets), per-tet E log-uniform in [1e4, 1e7], nu uniform in
    [0.25, 0.45], coarse layer of fixed 8^3-cube rigid clusters then the fine
    layer, 5 coarse + 10 fine iterations, dt = 1/60, base (z = 0) pinned,
    seeded random surface impulse at t = 0, 300 steps.  `energy` swaps the
    material model (the StVK Voigt constraint: the same scene for the
    reference's own constraint)."""
    rng = np.random.default_rng(seed)
    V, T, cube = generate_beam(nx, ny, nz, 0.1)
    nt = T.shape[0]
    E = np.exp(rng.uniform(np.log(1e4), np.log(1e7), nt))
    nu = rng.uniform(0.25, 0.45, nt)
    mu, lam = to_lame(nu, E)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=energy)
    m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
    forced = np.zeros(nt, dtype=bool)
    forced[m.pinnedTets - 1] = True
    coarse = cluster_rigid_sets(cube, (nx, ny, nz), cluster, forced)
    sets = np.asfortranarray(np.stack([np.zeros(nt, np.int32), coarse], 1))  # sorted columns: [fine, coarse]
    # impulse: random velocity on a seeded patch of the top surface
    top = np.nonzero(np.isclose(V[:, 2], nz * 0.1))[0]
    c = V[top[rng.integers(len(top))]]
    patch = top[np.linalg.norm(V[top, :2] - c[:2], axis=1) < 0.4]
    dv = rng.normal(0.0, 1.0, (len(patch), 3)) * 0.5 + np.array([0.0, 0.0, -2.0])
    dofs = np.stack([patch * 3 + 1, patch * 3 + 2, patch * 3 + 3], 1).ravel().astype(np.int32)
    return Scene("config2_nh_block_64x16x16", m, 1.0 / 60.0, 300, [50, 0], [5, 10], custom_sets=sets,
                 impulse=(dofs, dv.ravel()))


def config5(seed: int = 5, nx=64, ny=32, nz=32, coarse=8, mid=4) -> Scene:
    """The learned warm start's workload: the config-2 scene class at
    64x32x32 cubes (70,785 vertices, 393,216 tets), per-tet E log-uniform in
    [1e4, 1e7], nu uniform in [0.25, 0.45], Neo-Hookean, base pinned, seeded
    surface impulse; three layers -- coarse^3-cube clusters (5 iterations),
    mid^3-cube clusters (5), fine (10) -- dt = 1/60.  Other seeds give the
    training scenes (other materials and impulses)."""
    rng = np.random.default_rng(seed)
    V, T, cube = generate_beam(nx, ny, nz, 0.1)
    nt = T.shape[0]
    E = np.exp(rng.uniform(np.log(1e4), np.log(1e7), nt))
    nu = rng.uniform(0.25, 0.45, nt)
    mu, lam = to_lame(nu, E)
    m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=_lib.MLX_ENERGY_NEOHOOKEAN)
    m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
    forced = np.zeros(nt, dtype=bool)
    forced[m.pinnedTets - 1] = True
    sc = cluster_rigid_sets(cube, (nx, ny, nz), coarse, forced)
    sm = cluster_rigid_sets(cube, (nx, ny, nz), mid, forced)
    sets = np.asfortranarray(np.stack([np.zeros(nt, np.int32), sm, sc], 1))  # sorted columns: [fine, mid, coarse]
    patch, dv = _surface_impulse(rng, V, nz * 0.1)
    dofs = np.stack([patch * 3 + 1, patch * 3 + 2, patch * 3 + 3], 1).ravel().astype(np.int32)
    return Scene(f"config5_nh_block_{nx}x{ny}x{nz}", m, 1.0 / 60.0, 300, [50, 25, 0], [5, 5, 10], custom_sets=sets,
                 impulse=(dofs, dv.ravel()))


def config5_batch(seed: int = 100, n_scenes: int = 16, nx=32, ny=16, nz=16, coarse=8, mid=4,
                  spacing=1.0) -> Scene:
    """Training batch of the learned warm start: `n_scenes` blocks of the
    config-5 scene class (Neo-Hookean, per-tet E log-uniform in [1e4, 1e7],
    nu uniform in [0.25, 0.45], base pinned, a seeded surface impulse), each
    with its own seed (seed * 1000 + i), laid out along x `spacing` m apart
    and merged into one mesh as Mesh3D.mergeMesh does; the three layers of
    config 5 (coarse^3- and mid^3-cube clusters, then fine)."""
    meshes, cols_c, cols_m, imp_dofs, imp_dv = [], [], [], [], []
    x0, nb_c, nb_m, voff = 0.0, 0, 0, 0
    for i in range(n_scenes):
        rng = np.random.default_rng(seed * 1000 + i)
        V, T, cube = generate_beam(nx, ny, nz, 0.1, origin=(x0, 0.0, 0.0))
        x0 += nx * 0.1 + spacing
        nt = T.shape[0]
        E = np.exp(rng.uniform(np.log(1e4), np.log(1e7), nt))
        mu, lam = to_lame(rng.uniform(0.25, 0.45, nt), E)
        m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=_lib.MLX_ENERGY_NEOHOOKEAN)
        m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
        forced = np.zeros(nt, dtype=bool)
        forced[m.pinnedTets - 1] = True
        sc = cluster_rigid_sets(cube, (nx, ny, nz), coarse, forced)
        sm = cluster_rigid_sets(cube, (nx, ny, nz), mid, forced)
        sc[sc > 0] += nb_c
        sm[sm > 0] += nb_m
        nb_c, nb_m = int(max(nb_c, sc.max(initial=0))), int(max(nb_m, sm.max(initial=0)))
        cols_c.append(sc)
        cols_m.append(sm)
        patch, dv = _surface_impulse(rng, V, nz * 0.1)
        g = patch + voff
        imp_dofs.append(np.stack([g * 3 + 1, g * 3 + 2, g * 3 + 3], 1).ravel())
        imp_dv.append(dv.ravel())
        voff += m.N
        meshes.append(m)
    mesh = merge_meshes(meshes)
    sets = np.asfortranarray(np.stack([np.zeros(mesh.T, np.int32), np.concatenate(cols_m).astype(np.int32),
                                       np.concatenate(cols_c).astype(np.int32)], 1))
    sc = Scene(f"config5_batch_{n_scenes}x{nx}x{ny}x{nz}_seed{seed}", mesh, 1.0 / 60.0, 300, [50, 25, 0], [5, 5, 10],
               custom_sets=sets, impulse=(np.concatenate(imp_dofs).astype(np.int32), np.concatenate(imp_dv)))
    sc.settings["parts"] = meshes
    return sc


def _surface_impulse(rng, V, top_z, radius=0.4):
    """A seeded velocity on a patch of the top surface (0-based vertex ids)."""
    top = np.nonzero(np.isclose(V[:, 2], top_z))[0]
    c = V[top[rng.integers(len(top))]]
    patch = top[np.linalg.norm(V[top, :2] - c[:2], axis=1) < radius]
    dv = rng.normal(0.0, 1.0, (len(patch), 3)) * 0.5 + np.array([0.0, 0.0, -2.0])
    return patch, dv


def batch_block_dims(rng, tmin=2000, tmax=40000):
    """Cube-grid dimensions (nx, ny, nz) with 6*nx*ny*nz close to a tet count
    drawn log-uniformly from [tmin, tmax], random aspect ratios in [1, 3]."""
    target = np.exp(rng.uniform(np.log(tmin), np.log(tmax)))
    rx, ry = rng.uniform(1.0, 3.0, 2)
    n = (target / (6.0 * rx * ry)) ** (1.0 / 3.0)
    return max(int(round(rx * n)), 2), max(int(round(ry * n)), 2), max(int(round(n)), 2)


def config3(seed: int = 3, n_scenes: int = 256, tmin=2000, tmax=40000, cluster=4) -> Scene:
    """Batched Neo-Hookean blocks: `n_scenes` independent cube-grid blocks
    (0.1 m cubes) whose dimensions give 2k-40k tets (log-uniform, seeded),
    per-tet E log-uniform in [1e4, 1e6] Pa, nu = 0.35, base pinned, a seeded
    surface impulse each, merged into one mesh as Mesh3D.mergeMesh does
    (colours overlaid).  Two layers: fixed cluster^3-cube rigid clusters (5
    iterations), then the fine layer (10 iterations); dt = 1/60, 200 steps.
    Every block starts at the origin: the scenes share no vertex and the
    solver has no mesh-to-mesh contact, so they stay independent wherever
    they are, and FP32 positions near the origin keep the precision of a
    single scene (blocks laid side by side reach hundreds of metres, where an
    FP32 ulp is ~6e-5 m against 0.1 m cube edges)."""
    rng = np.random.default_rng(seed)
    meshes, sets, imp_dofs, imp_dv = [], [], [], []
    nbodies, voff = 0, 0
    for _ in range(n_scenes):
        nx, ny, nz = batch_block_dims(rng, tmin, tmax)
        V, T, cube = generate_beam(nx, ny, nz, 0.1)
        nt = T.shape[0]
        E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), nt))
        mu, lam = to_lame(0.35, E)
        m = Mesh3D.from_arrays(V, T, mu, lam, rho=1000.0, alpha1=0.0, energy_type=_lib.MLX_ENERGY_NEOHOOKEAN)
        m.pin(np.nonzero(np.isclose(V[:, 2], 0.0))[0] + 1)
        forced = np.zeros(nt, dtype=bool)
        forced[m.pinnedTets - 1] = True
        coarse = cluster_rigid_sets(cube, (nx, ny, nz), cluster, forced)
        coarse[coarse > 0] += nbodies
        nbodies = int(max(nbodies, coarse.max(initial=0)))
        sets.append(coarse)
        patch, dv = _surface_impulse(rng, V, nz * 0.1)
        g = patch + voff
        imp_dofs.append(np.stack([g * 3 + 1, g * 3 + 2, g * 3 + 3], 1).ravel())
        imp_dv.append(dv.ravel())
        voff += m.N
        meshes.append(m)
    mesh = merge_meshes(meshes)
    coarse = np.concatenate(sets).astype(np.int32)
    custom = np.asfortranarray(np.stack([np.zeros(mesh.T, np.int32), coarse], 1))
    sc = Scene(f"config3_batch_{n_scenes}_nh_blocks", mesh, 1.0 / 60.0, 200, [50, 0], [5, 10], custom_sets=custom,
               impulse=(np.concatenate(imp_dofs).astype(np.int32), np.concatenate(imp_dv)))
    sc.settings["parts"] = meshes
    return sc


def config4(seed: int = 4, n_boxes: int = 32, cubes: int = 12, grid=(8, 4), spacing=2.0, n_spheres: int = 4,
            coarse: int = 4, mid: int = 2, drop=(0.5, 3.0), contact_coloring: bool = True) -> Scene:
    """Contact-heavy drop: `n_boxes` StVK boxes of cubes^3 cubes (0.1 m, 6 tets
    per cube; 32 x 10,368 tets by default), E = 5e5 Pa, nu = 0.3, with seeded
    rotations, over a ground plane z = 0 and `n_spheres` analytic spheres
    (radius in [0.3, 0.6] m, half sunk in the ground under seeded boxes).  A
    box's lowest possible point (its half diagonal below its centre) starts a
    seeded height in `drop` m above what lies under it.  Three layers:
    coarse^3-cube rigid clusters, mid^3-cube rigid clusters, then the fine
    layer; 15 iterations split as the reference's cube drop example splits
    its own (1 and 4 rigid-layer iterations, the rest fine) with its contact
    resistance 0.9 (3d/examples/XPBD/cubeDrop_xpbd.m:27-35) and the finders'
    default contact compliance 1e-4; dt = 1/120, 500 steps.  Boxes sit on a
    grid `spacing` m apart, so they meet the obstacles and not each other.
    Contacts are coloured together with the elastic constraints (the
    configuration's definition: each vertex's contacts join the first colour
    phase whose tets do not touch it); contact_coloring=False keeps the
    reference's order (contacts after all colours, Jacobi, xpbdLayer3D.m:330).
    Returns the merged mesh; `contact_finders` holds the obstacles."""
    from .contacts import PlaneContactFinder3D, SphereContactFinder, rotation_matrix_degrees
    rng = np.random.default_rng(seed)
    half = cubes * 0.1 / 2
    xy = [np.array([(k % grid[0]) * spacing, ((k // grid[0]) % grid[1]) * spacing]) for k in range(n_boxes)]
    finders = [PlaneContactFinder3D([0.0, 0.0, 1.0], [0.0, 0.0, 0.0])]
    base = np.zeros(n_boxes)
    for k in rng.choice(n_boxes, size=min(n_spheres, n_boxes), replace=False):
        r = rng.uniform(0.3, 0.6)
        x, y = xy[k] + rng.uniform(-0.3, 0.3, 2)
        finders.append(SphereContactFinder(r, [x, y, 0.5 * r]))
        base[k] = 1.5 * r
    meshes, sets_c, sets_m = [], [], []
    nb_c = nb_m = 0
    for k in range(n_boxes):
        V, T, cube = generate_beam(cubes, cubes, cubes, 0.1)
        R = rotation_matrix_degrees(rng.uniform(0, 360, 3))
        c = np.array([xy[k][0], xy[k][1], base[k] + rng.uniform(*drop) + half * np.sqrt(3.0)])
        V = (V - half) @ R.T + c
        m = Mesh3D.from_arrays(V, T, *to_lame(0.3, 5e5), rho=1000.0, alpha1=0.0,
                               energy_type=_lib.MLX_ENERGY_STVK_VOIGT)
        none = np.zeros(m.T, dtype=bool)
        sc = cluster_rigid_sets(cube, (cubes, cubes, cubes), coarse, none)
        sm = cluster_rigid_sets(cube, (cubes, cubes, cubes), mid, none)
        sc[sc > 0] += nb_c
        sm[sm > 0] += nb_m
        nb_c = int(max(nb_c, sc.max(initial=0)))
        nb_m = int(max(nb_m, sm.max(initial=0)))
        sets_c.append(sc)
        sets_m.append(sm)
        meshes.append(m)
    mesh = merge_meshes(meshes)
    # sorted columns: [fine (0), mid (25), coarse (50)]
    custom = np.asfortranarray(np.stack([np.zeros(mesh.T, np.int32), np.concatenate(sets_m),
                                         np.concatenate(sets_c)], 1).astype(np.int32))
    sc = Scene(f"config4_drop_{n_boxes}_boxes_{cubes}c", mesh, 1.0 / 120.0, 500, [50, 25, 0], [1, 4, 10],
               gravity=-9.81, custom_sets=custom, contact_finders=finders)
    sc.settings["parts"] = meshes
    sc.settings["contactResistance"] = 0.9
    sc.settings["contactColoring"] = bool(contact_coloring)
    return sc
