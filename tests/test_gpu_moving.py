"""GPU tests of moving collision objects (mpm_set_object_motion).

Parity with the reference's own dumps of the moving-object scenes runs with the
other fixtures: test_gpu_parity.py (explicit substep, plain FP64 and the fast
path in every launch shape) and test_gpu_implicit.py (backward Euler).  Here:
the argument checks, that an object "moving" with the identity frame and no
twist equals the static object, that a failing callback fails the substep, and
that the fast path agrees with the plain path.
"""
import numpy as np
import pytest

from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def D():
    from physbam_b200 import driver
    return driver


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), floor)


PATHS = {"plain": lambda: (D().PATH_PLAIN, D().FP64), "fast": lambda: (D().PATH_FAST, D().FP32)}


def run(scene, path, nsteps):
    p, prec = PATHS[path]()
    drv = D().MPM_DRIVER(scene, precision=prec, path=p)
    drv.set_scene_particles(scene)
    for _ in range(nsteps):
        drv.Advance_One_Time_Step()
    out = drv.get_particles()
    drv.close()
    return out


def test_motion_arguments(cuda_device):
    s = S.small_3d(nsteps=1)
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    still = S.Motion([0, 0, 0], [0, 0, 0], [0, 0, 0])
    with pytest.raises(D().MPMError):
        drv.set_object_motion(len(s.objects), still)          # no such object
    drv.set_object_motion(0, still)
    drv.set_object_motion(0, None)
    drv.close()
    e = S.small_3d_moving(nsteps=1)
    with pytest.raises(ValueError):
        D().MPM_BATCH([e])


def test_failing_callback_fails_the_substep(cuda_device):
    s = S.small_3d(nsteps=1)
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(s)

    def broken(t):
        raise RuntimeError("no frame")

    drv.set_object_motion(0, broken)
    with pytest.raises(D().MPMError):
        drv.Advance_One_Time_Step()
    drv.close()


@pytest.mark.parametrize("implicit", [False, True])
@pytest.mark.parametrize("path", ["plain", "fast"])
def test_identity_motion_equals_static(cuda_device, path, implicit):
    """Every object given the identity frame and a zero twist: the static run
    (only the order of atomic sums differs)."""
    if implicit and path == "fast":
        pytest.skip("the implicit solve runs on the plain path")
    s = S.small_3d_sphere(nsteps=5)
    if implicit:
        s.implicit, s.dt = S.Implicit(), 1e-3
    moved = s.copy()
    moved.objects = [S.CollisionObject(o.kind, o.type, o.friction, o.a, o.b, motion=S.Motion([0, 0, 0], [0, 0, 0], [0, 0, 0]))
                     for o in s.objects]
    a, b = run(s, path, 5), run(moved, path, 5)
    # implicit: two runs of the same solve may take different Newton paths (the order of
    # the atomic sums), within the bounds of the implicit parity tests
    if implicit:
        tol = {"X": 2e-9, "V": 1e-6, "F": 1e-7}
    else:
        tol = dict.fromkeys(("X", "V", "F"), 1e-13 if path == "plain" else 1e-6)
    for k in ("X", "V", "F"):
        assert rel(b[k], a[k], 1.0) < tol[k], k


def test_sticky_nodes_follow_the_object(cuda_device):
    """Nodes held by the sliding sticky paddle carry its velocity (stuck_velocity)."""
    s = S.small_3d_moving(nsteps=1)
    pad = s.objects[-2]
    lin = [-4.0, 0.5, 0.0]
    s.objects = s.objects[:-2] + [S.CollisionObject(pad.kind, pad.type, pad.friction, pad.a, pad.b,
                                                    motion=S.Motion(pad.motion.center, lin, [0.0, 0.0, 0.0]))]
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(s)
    drv.Advance_One_Time_Step()
    g = drv.get_grid()
    drv.close()
    held = np.all(g["grid_vf"] == np.asarray(lin), axis=-1) & (g["grid_m"] > 0)
    assert held.sum() >= 4
    # velocity = dv + v0 with dv = V - v0, as the reference assembles it
    np.testing.assert_allclose(g["grid_v"][held], np.broadcast_to(lin, (int(held.sum()), 3)), rtol=1e-14, atol=1e-14)


def test_fast_matches_plain(cuda_device):
    s = S.small_3d_moving(nsteps=20)
    ref, fast = run(s, "plain", 20), run(s, "fast", 20)
    np.testing.assert_array_equal(fast["valid"], ref["valid"])
    vmax = float(np.abs(ref["V"]).max())
    assert rel(fast["X"], ref["X"], 1.0) < 2e-6
    assert rel(fast["V"], ref["V"], vmax) < 2e-3
    assert rel(fast["F"], ref["F"], 1.0) < 1e-4


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_advance_with_moving_objects(cuda_device, path):
    """mpm_advance over moving objects (every substep's frames evaluated into a
    device table first, then the captured graph replayed, its first kernel taking
    the next table slot) gives the substep-by-substep result: one advance of 12,
    and advance(5) then advance(12) (a second replay, whose slot counter the table
    upload resets, then a longer table: regrow, new capture) against 17 eager
    substeps."""
    s = S.small_3d_moving(nsteps=17)
    p, prec = PATHS[path]()
    tol = 1e-12 if path == "plain" else 1e-5
    for plan in ([12], [5, 12]):
        total = sum(plan)
        out = []
        for batched in (False, True):
            drv = D().MPM_DRIVER(s, precision=prec, path=p)
            drv.set_scene_particles(s)
            if batched:
                for k in plan:
                    drv.advance(k)
            else:
                for _ in range(total):
                    drv.Advance_One_Time_Step()
            out.append(drv.get_particles())
            drv.close()
        for k in ("X", "V", "F"):
            assert rel(out[1][k], out[0][k], 1.0) < tol, (plan, k)
