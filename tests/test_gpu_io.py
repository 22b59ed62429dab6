"""GPU tests of output frames and restart through PhysBAM's viewer-directory
format (MPM_DRIVER.write_frame / read_frame, physbam_b200.io): a run written
at a frame and restarted from it continues as the uninterrupted run, plastic
state included, and the frame files hold the state the driver reports."""
import shutil
import tempfile

import numpy as np
import pytest

from physbam_b200 import io
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def D():
    from physbam_b200 import driver
    return driver


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), floor)


CASES = [("elastic-plain", S.small_3d, "plain"), ("snow-plain", S.small_snow_3d, "plain"),
         ("sand-fast", S.small_sand_3d, "fast"), ("elastic-fast", S.small_3d, "fast")]


@pytest.mark.parametrize("label,make,path", CASES, ids=[c[0] for c in CASES])
def test_restart_continues_the_run(cuda_device, label, make, path):
    scene = make(nsteps=10)
    p, prec = (D().PATH_PLAIN, D().FP64) if path == "plain" else (D().PATH_FAST, D().FP32)
    full = D().MPM_DRIVER(scene, precision=prec, path=p)
    full.set_scene_particles(scene)
    for _ in range(10):
        full.Advance_One_Time_Step()
    ref = full.get_particles()
    full.close()
    tmp = tempfile.mkdtemp()
    try:
        a = D().MPM_DRIVER(scene, precision=prec, path=p)
        a.set_scene_particles(scene)
        for _ in range(5):
            a.Advance_One_Time_Step()
        a.write_frame(tmp, 3)
        written = a.get_particles()
        a.close()
        f = io.read_frame(tmp, 3)
        np.testing.assert_array_equal(f["X"], written["X"])
        assert f["time"] == pytest.approx(5 * scene.dt)
        b = D().MPM_DRIVER(scene, precision=prec, path=p)
        b.read_frame(tmp, 3)
        assert b.time == pytest.approx(5 * scene.dt)
        for _ in range(5):
            b.Advance_One_Time_Step()
        got = b.get_particles()
        b.close()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    np.testing.assert_array_equal(got["valid"], ref["valid"])
    tol = 1e-12 if path == "plain" else 2e-6    # the fast path reorders its particles on reload
    assert rel(got["X"], ref["X"], 1.0) < tol
    assert rel(got["F"], ref["F"], 1.0) < tol * 10
