"""GPU tests of adaptive substeps (mpm_simulate_frame, mpm_set_dt_control):
MPM_DRIVER::Simulate_To_Frame with Compute_Dt, and Reduce_Dt's strong CFL
(Grid_To_Particle_Limit_Dt) and sound-speed CFL after the forces.

Against the reference's own frames (tests/golden/small{2,3}d_adaptive.npz):
the same number of substeps in every frame, and the state at the frame ends
node for node in FP64.
"""
import numpy as np
import pytest

from make_golden import CASES, load
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu

ADAPTIVE = sorted(n for n in CASES if "adaptive" in n)


def D():
    from physbam_b200 import driver
    return driver


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), floor)


@pytest.mark.parametrize("name", ADAPTIVE)
def test_frames_match_reference(cuda_device, name):
    scene, dumps = load(name)
    drv = D().MPM_DRIVER(scene, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(scene)
    counts = []
    for frame in range(max(dumps) + 1):
        counts.append(drv.simulate_frame())
        if frame not in dumps:
            continue
        ref = dumps[frame]
        got = drv.get_particles()
        np.testing.assert_array_equal(got["valid"], ref["valid"])
        vmax = float(np.abs(ref["V"]).max())
        assert rel(got["X"], ref["X"], 1.0) < 1e-12, frame
        assert rel(got["V"], ref["V"], vmax) < 1e-9, frame
        assert rel(got["F"], ref["F"], 1.0) < 1e-10, frame
    drv.close()
    print(name, counts, scene.frame_substeps)
    assert counts == scene.frame_substeps[:len(counts)]
    assert abs(drv.time - scene.dt_control.frame_dt * len(counts)) < 1e-15


def test_reduce_dt_shortens_and_fast_path_refuses(cuda_device):
    scene = S.small_3d_adaptive()
    drv = D().MPM_DRIVER(scene, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(scene)
    drv.Advance_One_Time_Step(5e-4)
    assert drv.last_dt() < 5e-4 * 0.99          # the sound speed of the stiff block
    drv.close()
    fast = D().MPM_DRIVER(S.small_3d(nsteps=1))
    with pytest.raises(D().MPMError):
        fast.set_dt_control(S.DtControl(strong_cfl=True))
    fast.set_dt_control(S.DtControl(max_dt=1e-4, cfl=0.5))   # Compute_Dt steps only
    fast.set_scene_particles(S.small_3d(nsteps=1))
    n = fast.simulate_frame(1e-3)
    assert n >= 10 and abs(fast.time - 1e-3) < 1e-15
    fast.close()
