"""simulate3D's loop (device contact finders, integrate, TimingData) on the
config-1 cantilever falling onto a plane and a sphere, against the oracle's
finders and integrate: positions FP64 <= 1e-9 of the bounding-box diagonal at
every frame, contact counts equal, and the TimingData log written in
writeTDcsv's format.  The single body-free layer runs on the component-group
path, so this also pins that path's projection of a host contact list."""
import numpy as np
import pytest

from multilayersolver2024_b200 import _lib, scenes
from multilayersolver2024_b200.contacts import PlaneContactFinder3D, SphereContactFinder
from multilayersolver2024_b200.simulate import simulate3d, write_td_csv
from multilayersolver2024_b200.xpbd_layer3d import StepCache, XpbdLayer3D

pytestmark = pytest.mark.gpu


def _finders():
    return [PlaneContactFinder3D([0, 0, 1.0], [0, 0, -0.06]), SphereContactFinder(0.05, [0.75, 0.1, -0.04])]


def _integ():
    it = XpbdLayer3D()
    it.setLayers([0])
    it.iterations = [20]
    it.precision = _lib.MLX_FP64
    return it


def test_simulate3d_matches_oracle(gpu, oracle, tmp_path):
    frames = 40
    sc = scenes.config1()
    traj = []
    integ = _integ()
    td = simulate3d(sc.mesh, integ, sc.h, frames, _finders(),
                    on_frame=lambda f, m, t: traj.append((m.p.copy(), t.contactCount)))
    assert "CTAs each owning whole components" in integ.solver(sc.mesh).launch_path
    ref_mesh = scenes.config1().mesh
    it, cache = _integ(), StepCache()
    d = ref_mesh.bbox_diagonal()
    oracle.load().orc_set_threads(4)
    seen = 0
    for frame in range(1, frames + 1):
        cs = oracle.find_contacts(_finders(), ref_mesh.p)
        oracle.integrate(it, ref_mesh, sc.h, cs, cache, frame)
        p, k = traj[frame - 1]
        assert k == cs.vertex_ids.size, frame
        seen = max(seen, k)
        assert np.abs(p - ref_mesh.p).max() / d <= 1e-9, frame
    assert seen > 0
    assert td.log.shape == (11, frames) and td.logCounts.shape == (10, frames)
    np.testing.assert_allclose(td.logCounts[7], sc.h * np.arange(1, frames + 1))
    (path,) = write_td_csv([td], str(tmp_path / "cantilever_"), ["b200"])
    assert len(path.read_text().splitlines()) == frames + 1
