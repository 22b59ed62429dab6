"""GPU tests of the penalty collision objects (mpm_set_penalty_objects).

Parity with the reference's own dumps of the penalty scenes runs with the other
fixtures: test_gpu_parity.py (explicit substep: plain FP64 and the fast path in
every launch shape) and test_gpu_implicit.py (backward Euler, whose energy,
gradient and Hessian carry the penalty terms).  Here: the argument checks, that
objects no particle reaches change nothing, that the objects act, and that the
fast path's impulse form (V + dt f / m read by P2G) agrees with the plain
path's scattered force.
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


def test_penalty_arguments(cuda_device):
    s = S.small_3d(nsteps=1)
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    ball = S.CollisionObject(S.SPHERE, S.SLIP, 0.0, [0.5, 0.5, 0.5], [0.1, 0, 0])
    bad = [S.Penalty([S.CollisionObject(7, S.SLIP, 0.0, [0, 0, 0], [1, 1, 1])]),                 # kind
           S.Penalty([S.CollisionObject(S.SPHERE, S.SLIP, 0.0, [0.5, 0.5, 0.5], [0.0, 0, 0])]),  # radius
           S.Penalty([S.CollisionObject(S.BOX, S.SLIP, 0.0, [0.5, 0.5, 0.5], [0.4, 1, 1])]),     # empty box
           S.Penalty([ball], stiffness=-1.0),
           S.Penalty([ball], separation=float("nan")),
           S.Penalty([ball] * 9)]                                                              # > MPM_MAX_OBJECTS
    for pen in bad:
        with pytest.raises(D().MPMError):
            drv.set_penalty(pen)
    drv.set_penalty(S.Penalty([ball]))
    drv.set_penalty(None)
    drv.close()
    with pytest.raises(ValueError):
        e = S.small_3d(nsteps=1)
        e.penalty = S.Penalty([ball])
        D().MPM_BATCH([e])


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_unreached_objects_change_nothing(cuda_device, path):
    """Objects farther than the separation from every particle: the same motion
    (only the order of atomic sums differs between the runs)."""
    s = S.small_3d(nsteps=5)
    far = s.copy()
    far.penalty = S.Penalty([S.CollisionObject(S.SPHERE, S.SLIP, 0.0, [3.0, 3.0, 3.0], [0.5, 0, 0]),
                             S.CollisionObject(S.PLANE, S.SLIP, 0.0, [0.0, 1.0, 0.0], [0.0, -2.0, 0.0])])
    a, b = run(s, path, 5), run(far, path, 5)
    tol = 1e-13 if path == "plain" else 1e-6
    for k in ("X", "V", "F"):
        assert rel(b[k], a[k], 1.0) < tol, k


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_penalty_objects_push_particles_out(cuda_device, path):
    """The slab under the block and the ball beside it push the particles inside
    them outward: along +y under the slab's top and away from the ball's centre."""
    s = S.small_3d_penalty(nsteps=10)
    off = s.copy()
    off.penalty = None
    a, b = run(off, path, 10), run(s, path, 10)
    dv = b["V"] - a["V"]
    X0 = s.X
    slab = X0[:, 1] < 0.13          # under the slab's top (the sticky floor holds the lowest nodes)
    assert slab.sum() > 10 and (dv[slab, 1] > 0).mean() > 0.9 and dv[slab, 1].mean() > 1e-3
    c = np.array([0.62, 0.33, 0.52])
    inside = np.linalg.norm(X0 - c, axis=1) < 0.07
    assert inside.sum() > 5
    radial = np.einsum("ij,ij->i", dv[inside], (X0[inside] - c))
    assert (radial > 0).mean() > 0.9


def test_fast_matches_plain(cuda_device):
    s = S.small_3d_penalty(nsteps=20)
    ref, fast = run(s, "plain", 20), run(s, "fast", 20)
    np.testing.assert_array_equal(fast["valid"], ref["valid"])
    vmax = float(np.abs(ref["V"]).max())
    assert rel(fast["X"], ref["X"], 1.0) < 2e-6
    assert rel(fast["V"], ref["V"], vmax) < 2e-3
    assert rel(fast["F"], ref["F"], 1.0) < 1e-4


def test_fast_penalty_survives_a_new_particle_count(cuda_device):
    """The fast path's impulse buffer is rebuilt with the particle buffers: a
    second, smaller particle set on the same handle still feels the objects."""
    s = S.small_3d_penalty(nsteps=10)
    sub = s.subset(np.arange(0, s.n, 2))
    drv = D().MPM_DRIVER(s, precision=D().FP32, path=D().PATH_FAST)
    drv.set_scene_particles(s)
    drv.advance(3)
    drv.set_scene_particles(sub)                 # new count: every particle buffer is reallocated
    drv.time = 0.0
    for _ in range(10):
        drv.Advance_One_Time_Step()
    got = drv.get_particles()
    drv.close()
    ref = run(sub, "plain", 10)
    vmax = float(np.abs(ref["V"]).max())
    assert rel(got["X"], ref["X"], 1.0) < 2e-6
    assert rel(got["V"], ref["V"], vmax) < 2e-3
