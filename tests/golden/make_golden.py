"""Generate the golden fixtures of tests/golden from the reference itself.

Run where the reference tree is mounted and oracle/_ref is built
(``make -C oracle REF=<tree>``), giving the tree by --ref or the environment
variable MLX_REFERENCE_TREE:

    python tests/golden/make_golden.py --ref <reference tree>

Writes
  stvk_grad.npz   C (6) and gradC (6x12) of the reference's symbolic Green-strain
                  constraint, 3d/constraints/StVKconstraintGrad3D.m, evaluated
                  here with numpy by translating the file's own expressions
                  (elementwise MATLAB -> numpy, same operation order);
  layers.npz      per-tet strain-rate norms and rigid-body IDs per layer from the
                  reference's 3d/mex/mexEdiffNorm3D.cpp and
                  2d/mex/mexUnionFindByVertice.cpp, compiled unchanged against
                  the headless mx runtime (oracle/_ref);
  layer_solve.npz inputs and results of xpbdLayer3D.layerSolve
                  (3d/integrator/xpbdLayer3D.m:44-232) on small scenes,
                  produced by executing the reference's own MATLAB functions
                  with the MATLAB-subset interpreter tests/golden/mlite.py
                  (MATLAB itself is not installed).
The reference sources are read, never copied; only computed numbers are kept.
"""
from __future__ import annotations

import argparse
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def _translate(expr: str) -> str:
    expr = re.sub(r"DmInv\((\d),(\d),:\)", lambda m: f"DmInv[{int(m.group(1)) - 1},{int(m.group(2)) - 1}]", expr)
    expr = re.sub(r"x\((\d+),:,:\)", lambda m: f"x[{int(m.group(1)) - 1}]", expr)
    return expr.replace(".*", "*").replace("./", "/").replace(".^", "**")


def _split_top(s: str, sep=";"):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        parts.append(cur)
    return parts


def eval_stvk_symbolic(src: str, DmInv: np.ndarray, x: np.ndarray):
    """Evaluate StVKconstraintGrad3D's expression list.  DmInv (3, 3, n),
    x (12, n).  Returns gradC (6, 12, n) and C (6, n) as the file's reshape
    and pagetranspose define them."""
    env = {"DmInv": DmInv, "x": x, "np": np}
    lists = {}
    for raw in src.splitlines():
        line = raw.strip()
        m = re.match(r"^(t\d+)\s*=\s*(.*);$", line)
        if m:
            env[m.group(1)] = eval(_translate(m.group(2)), env)
            continue
        m = re.match(r"^(mt\d+)\s*=\s*\[(.*)\];$", line)
        if m:
            lists[m.group(1)] = [eval(_translate(e), env) for e in _split_top(m.group(2))]
            continue
        m = re.match(r"^out\s*=\s*\[(.*)\];$", line)
        if m:
            out = []
            for name in _split_top(m.group(1)):
                out += lists[name.strip()]
            n = x.shape[1]
            out = np.stack([np.broadcast_to(o, (n,)) for o in out])  # (78, n)
            grad = out[:72].reshape(6, 12, n)  # reshape(out(1:72),12,6) then pagetranspose
            C = out[72:78]
            return grad, C
    raise ValueError("StVKconstraintGrad3D: no `out = [...]` line found")


def random_tets(rng, n):
    """Well-shaped random tets (rest) and perturbed current positions."""
    base = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.1
    rest = base[None] + rng.normal(0, 0.015, (n, 4, 3))
    Dm = np.stack([rest[:, k] - rest[:, 0] for k in (1, 2, 3)], axis=2)
    DmInv = np.linalg.inv(Dm)  # (n, 3, 3)
    cur = rest + rng.normal(0, 0.01, (n, 4, 3))
    return DmInv, cur.reshape(n, 12)


def make_stvk(ref: Path, out: Path, n=256, seed=11):
    src = (ref / "3d/constraints/StVKconstraintGrad3D.m").read_text()
    rng = np.random.default_rng(seed)
    DmInv, x = random_tets(rng, n)
    grad, C = eval_stvk_symbolic(src, DmInv.transpose(1, 2, 0), x.T)
    np.savez_compressed(out / "stvk_grad.npz", DmInv=DmInv, x=x, gradC=grad.transpose(2, 0, 1), C=C.T,
                        seed=seed)


def make_layers(out: Path, seed=5):
    from multilayersolver2024_b200 import scenes
    from oracle.oracle import RefMex
    uf = RefMex("mexUnionFindByVertice")
    ed = RefMex("mexEdiffNorm3D")
    rng = np.random.default_rng(seed)
    data = {}
    for tag, dims in (("beam", (8, 2, 2)), ("block", (6, 5, 4))):
        V, T, _ = scenes.generate_beam(*dims, edge=0.1)
        N, nt = V.shape[0], T.shape[0]
        p0 = V.reshape(-1)
        p = p0 + rng.normal(0, 0.004, p0.shape)
        oldp = p0 + rng.normal(0, 0.004, p0.shape)
        # F = B*p in computeB3D's layout (9 rows per tet, entry 3(d-1)+(j-1) = F(d,j))
        ids = T - 1
        Dm = np.stack([V[ids[:, k]] - V[ids[:, 0]] for k in (1, 2, 3)], axis=2)
        G = np.linalg.inv(Dm)
        def Bp(q):
            Q = q.reshape(-1, 3)
            Ds = np.stack([Q[ids[:, k]] - Q[ids[:, 0]] for k in (1, 2, 3)], axis=2)
            F = Ds @ G
            return F.reshape(nt, 9).reshape(-1)  # row-major F per tet
        h = 0.01
        norms = ed(1, Bp(p), Bp(oldp), h)[0].ravel()
        order = np.argsort(norms, kind="stable") + 1
        forced = np.zeros(nt, bool)
        forced[rng.choice(nt, nt // 10, replace=False)] = True
        layers = np.array([[0.0, 20.0, 45.0, 70.0]])
        sets, nr = uf(2, order.astype(float), layers, forced, np.asfortranarray(T.astype(np.int32)), float(N))
        data.update({f"{tag}_V": V, f"{tag}_T": T, f"{tag}_p": p, f"{tag}_oldp": oldp, f"{tag}_h": h,
                     f"{tag}_DmInv": G.transpose(0, 2, 1).reshape(nt, 9), f"{tag}_norms": norms,
                     f"{tag}_order": order.astype(np.int32), f"{tag}_forced": forced,
                     f"{tag}_layers": layers.ravel(), f"{tag}_sets": sets.astype(np.int32),
                     f"{tag}_numRigids": nr.ravel().astype(np.int32)})
    np.savez_compressed(out / "layers.npz", **data)


LAYER_SOLVE_CASES = {
    # name: (dims, energy seed, alpha1, layers, iterations, case seed, contacts, settings)
    "single_damped": ((4, 2, 2), 31, 0.01, [0], [3], 32, False, {}),
    "three_layers_contacts_monitor": ((4, 3, 3), 2, 0.0, [50, 25, 0], [2, 3, 4], 3, True,
                                      dict(boundaryCompliance=0.0, contactResistance=0.9, computeResiduals=True,
                                           StopAtImprovementPercent=60, runUntilResSmallerThan=0.0,
                                           hangingStop=40, giveUpEnabled=True)),
    "two_layers_elastic_contacts": ((4, 3, 3), 5, 0.02, [60, 0], [3, 5], 6, True,
                                    dict(boundaryCompliance=1e-8, useRigidContacts=False)),
    "run_until_hanging_stop": ((5, 2, 2), 7, 0.0, [40, 0], [2, 3], 8, False,
                               dict(computeResiduals=True, runUntilResSmallerThan=1e-9, hangingStop=12,
                                    boundaryCompliance=0.0)),
}


def build_case(name):
    """The layerSolve inputs of one named case (deterministic)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import Case, block_mesh, plane_contacts, sphere_contacts
    from multilayersolver2024_b200.xpbd_layer3d import ContactSet
    dims, eseed, a1, layers, iters, cseed, contacts, settings = LAYER_SOLVE_CASES[name]
    m = block_mesh(dims=dims, seed=eseed, alpha1=a1)
    case = Case(m, layers, iters, seed=cseed)
    for k, v in settings.items():
        setattr(case.integ, k, v)
    if contacts:
        case.contacts = ContactSet.concat([plane_contacts(case.xi, [0, 0, 1.0], [0, 0, 0.004]),
                                           sphere_contacts(case.xi, 0.12, [0.25, 0.15, 0.0])])
    return case


def reference_layer_solve_args(case):
    """layerSolve's 50 arguments with the MATLAB classes and page shapes of
    xpbdLayer3D.integrate (xpbdLayer3D.m:684-733)."""
    import mlite
    m, ls, it, c = case.mesh, case.ls, case.integ, case.contacts
    K = c.vertex_ids.size
    col = lambda a: mlite.M(np.asarray(a, dtype=float).reshape(-1, 1))
    sc = lambda v: mlite.M(float(v))
    pages = lambda a, n: np.ascontiguousarray(np.asarray(a).reshape(-1, n, n).transpose(2, 1, 0))
    return [
        ls.isElasticElement.astype(bool), ls.isRigidElement.astype(bool), ls.rigidBodySetsPerLayer,
        ls.vertexRigidBody, ls.isBoundaryVertex.astype(bool), ls.isRigidVertex.astype(bool),
        col(case.xi), np.asfortranarray(case.lam), sc(0.0), sc(case.h), col(ls.numRigids), sc(0.0),
        sc(it.boundaryCompliance), sc(it.contactResistance),
        np.asarray(c.compliance, float).reshape(1, 1, K) if K else np.zeros((1, 1, 0)),
        mlite.M(np.array(it.iterations, float)), mlite.M(np.array(it.layers, float)),
        sc(it.runUntilResSmallerThan), mlite.M(bool(it.computeResiduals)), sc(it.hangingStop),
        mlite.M(bool(it.giveUpEnabled)), sc(it.giveUpThreshold), mlite.M(bool(it.LastLayerGiveUpEnabled)),
        mlite.M(bool(it.useGravityConstraints)), col(case.oldp), col(case.oldOldp),
        mlite.M(np.asarray(c.normals, float).reshape(K, 3)) if K else np.zeros((0, 3)),
        mlite.M(np.asarray(c.points, float).reshape(K, 3)) if K else np.zeros((0, 3)),
        col(c.vertex_ids) if K else np.zeros((0, 1)), col(m.mass), np.asfortranarray(m.t),
        mlite.M(m.unpinnedDOFs.astype(float)), col(m.pinnedDOFs), pages(m.DmInv, 3),
        pages(m.perElementXPBDalphaMatrix, 6), pages(m.perElementXPBDalphaInvMatrix, 6), col(m.elementColor),
        m.elementDOFs, sc(m.numColors), col(case.f), col(it.layersMap), sc(it.gravityCompliance),
        sc(it.Gravity), col(case.resv), pages(m.perElementXPBDbeta, 6), col(m.elV), mlite.M(False),
        mlite.M(bool(it.useRigidContacts)), sc(it.StopAtImprovementPercent), col(case.pinnedx),
    ]


def make_layer_solve(ref: Path, out: Path):
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import mlite
    interp = mlite.Interpreter(ref, mlite.LAYER_SOLVE_TABLE)
    data = {}
    for name in LAYER_SOLVE_CASES:
        case = build_case(name)
        xi, _snm, res, run_until = interp.call("xpbdLayer3D.layerSolve", reference_layer_solve_args(case), nargout=4)
        data[f"{name}_xi"] = np.asarray(xi, float).ravel()
        data[f"{name}_residual"] = np.asarray(res, float).ravel()
        data[f"{name}_run_until"] = float(np.asarray(run_until).ravel()[0])
        data[f"{name}_input_xi"] = case.xi  # lets a test confirm it rebuilt the same inputs
    np.savez_compressed(out / "layer_solve.npz", **data)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MLX_REFERENCE_TREE"))
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference tree by --ref or MLX_REFERENCE_TREE")
    out = Path(__file__).resolve().parent
    make_stvk(Path(a.ref), out)
    make_layers(out)
    make_layer_solve(Path(a.ref), out)
    print("wrote", sorted(p.name for p in out.glob("*.npz")))


if __name__ == "__main__":
    main()
