"""simulate3D's step loop without the drawing (3d/simulate3D.m:156-171 contact
finders, :183-281 integrate, :294-340 counts) and its TimingData record
(2d/TimingData.m:9-70 fields and labels, :77-106 logData), with writeTDcsv's
file format (util/figures/writeTDcsv.m:40-60): one header line of the count
labels then the time labels, one line per frame, every value printed with
MATLAB's ``%d`` (integers as integers, other values as ``%e``).

The contact finders run on the device (``mlx_find_contacts``) and the step
through ``XpbdLayer3D.integrate`` (``mlx_layer_solve``).
"""
from __future__ import annotations

import math
import time
from pathlib import Path

import numpy as np

COUNT_LABELS = ["contactCount", "countParticles", "countElements", "countTotalParticles", "countTotalElements",
                "rigidBodies", "totalDofs", "stepSum", "residual", "residualPreSolve"]
TIME_LABELS = ["Collision Detection", "Simulation Step Total", "Compute Forces and C", "Elastification QuickSolve",
               "Elastification (Bookkeeping)", "Integrate Forces", "Integrate Contact", "Rigidification",
               "contact solve 1", "contact solve 2", "connected components"]


class TimingData:
    """TimingData.m: the last step's counts and times, logged per frame."""

    def __init__(self):
        # discrete quantities
        self.contactCount = 0
        self.countParticles = 0
        self.countTris = 0
        self.countTotalParticles = 0
        self.countTotalTris = 0
        self.residual = 0.0
        self.residualPreSolve = 0.0
        self.rigidBodies = 0
        self.totalDofs = 0
        self.stepSum = 0.0
        # times (s)
        self.lastContact = 0.0
        self.lastSimulate = 0.0
        self.fullFCForces = 0.0
        self.lastElastification = 0.0
        self.lastElastifyQuickSolve = 0.0
        self.integrateForces = 0.0
        self.integrateContacts = 0.0
        self.lastRigidification = 0.0
        self.contactSolve1 = 0.0
        self.contactSolve2 = 0.0
        self.connectedComponents = 0.0
        self.labelsCountData = list(COUNT_LABELS)
        self.labels = list(TIME_LABELS)
        self.log = np.zeros((len(TIME_LABELS), 0))
        self.logCounts = np.zeros((len(COUNT_LABELS), 0))
        self.iterations = []

    def logData(self):
        """TimingData.logData: append this frame's column to both logs."""
        counts = [self.contactCount, self.countParticles, self.countTris, self.countTotalParticles,
                  self.countTotalTris, self.rigidBodies, self.totalDofs, self.stepSum, self.residual,
                  self.residualPreSolve]
        times = [self.lastContact, self.lastSimulate, self.fullFCForces, self.lastElastification,
                 self.lastElastifyQuickSolve, self.integrateForces, self.integrateContacts,
                 self.lastRigidification, self.contactSolve1, self.contactSolve2, self.connectedComponents]
        self.logCounts = np.hstack([self.logCounts, np.asarray(counts, np.float64)[:, None]])
        self.log = np.hstack([self.log, np.asarray(times, np.float64)[:, None]])


def matlab_d(x: float) -> str:
    """MATLAB's sprintf('%d', x): integral values as integers, others as %e."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Inf" if x > 0 else "-Inf"
    if x == int(x):
        return str(int(x))
    return f"{x:e}"


def write_td_csv(tds, testname, names):
    """writeTDcsv(td, testname, names): one file `testname + name + '.csv'`
    per TimingData."""
    assert len(tds) == len(names)
    paths = []
    for td, name in zip(tds, names):
        path = Path(f"{testname}{name}.csv")
        lines = [",".join(td.labelsCountData) + "," + ",".join(td.labels)]
        for j in range(td.log.shape[1]):
            row = np.concatenate([td.logCounts[:, j], td.log[:, j]])
            lines.append(",".join(matlab_d(v) for v in row))
        path.write_text("\n".join(lines) + "\n")
        paths.append(path)
    return paths


def simulate3d(mesh, integrator, h, steps, contact_finders=(), td=None, on_frame=None):
    """simulate3D's loop for one mesh: per frame the finders on the step-start
    positions (Collision Detection), integrate (Simulation Step Total,
    Integrate Forces, residuals), the counts, stepSum = h * frame, logData.
    Returns the TimingData."""
    from .contacts import find_contacts
    from .xpbd_layer3d import ContactSet, StepCache
    td = td or TimingData()
    cache = StepCache()
    for frame in range(1, steps + 1):
        t0 = time.perf_counter()
        if contact_finders:
            cs = find_contacts(integrator.solver(mesh), list(contact_finders), mesh.p)
        else:
            cs = ContactSet()
        td.contactCount = int(cs.vertex_ids.size)
        td.lastContact = time.perf_counter() - t0
        t1 = time.perf_counter()
        out = integrator.integrate(mesh, h, cs, cache, frame)
        td.lastSimulate = time.perf_counter() - t1
        td.integrateForces = out["integrateForces"]
        td.residual = out["residual"]
        td.residualPreSolve = out["residualPreSolve"]
        td.iterations.append(out["iterations"])
        td.countParticles = td.countTotalParticles = mesh.N
        td.countTris = td.countTotalTris = mesh.T
        td.rigidBodies = 0  # a plain Mesh3D (the layers' bodies live inside the step)
        td.totalDofs = int(mesh.unpinnedDOFs.size)  # activeDOFs of a plain Mesh3D
        td.stepSum = h * frame
        td.logData()
        if on_frame:
            on_frame(frame, mesh, td)
    return td
