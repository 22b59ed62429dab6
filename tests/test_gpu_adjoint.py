"""GPU tests of the hand-written adjoint (mpm_diff_forward / mpm_diff_backward).

Loss: squared distance of the final centre of mass to a seeded target (the
rollout loss; the v0 checks use it) and the same for the half of the body
that starts at x > 0.5 (it moves with the deformation, so the E checks use
it -- the whole-body centre of mass does not depend on E at all).  The
parameters are the initial velocity v0 (shared by all particles) and the
per-particle Young's modulus E.  Gradients are checked against central finite
differences of the FP64 forward (step scanned, best kept), in FP64 and FP32,
to the stated tolerance 1e-3.
"""
import numpy as np
import pytest

from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def setup(scene, prec):
    import torch
    from physbam_b200 import driver as D
    dtype = torch.float64 if prec == D.FP64 else torch.float32
    drv = D.MPM_DRIVER(scene, precision=prec, path=D.PATH_PLAIN)
    dev = "cuda"
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
    return drv, dtype, t


def loss_fn(drv, scene, t, dtype, v0, E, nsteps, every, want_grad, part=False):
    import torch
    from physbam_b200 import autograd as A
    nu = 0.3
    n = scene.n
    X = t(scene.X)
    F = t(scene.F)
    B = t(scene.B)
    mass, vol = t(scene.mass), t(scene.volume)
    target = t(scene.target)
    v0t = torch.tensor(v0, dtype=dtype, device="cuda", requires_grad=want_grad)
    Et = torch.tensor(E, dtype=dtype, device="cuda", requires_grad=want_grad)
    mu = Et / (2 * (1 + nu))
    lam = Et * nu / ((1 + nu) * (1 - 2 * nu))
    V = (v0t.expand(n, 3) + t(getattr(scene, "vfield", np.zeros((n, 3))))).contiguous()
    X1, V1, F1, B1, valid = A.rollout(drv, X, V, F, B, mu, lam, mass, vol, nsteps, every)
    if part:
        L = A.part_com_loss(X1, mass, t(scene.X[:, 0] > 0.5), target)
    else:
        L = A.com_loss(X1, mass, target)
    if not want_grad:
        return float(L)
    L.backward()
    return float(L.detach()), v0t.grad.detach().cpu().numpy().astype(np.float64), Et.grad.detach().cpu().numpy().astype(np.float64)


def fd(f, x0, direction, hs=(1e-3, 3e-4, 1e-4, 3e-5)):
    """Central differences over a scan of steps; returns all estimates."""
    return [(f(x0 + h * direction) - f(x0 - h * direction)) / (2 * h) for h in hs]


def closest(estimates, value):
    return min(estimates, key=lambda e: abs(e - value))


def deformed(scene, seed=5):
    """The same body pre-stressed (F != I) and spinning, so E matters."""
    rng = np.random.default_rng(seed)
    s = scene.copy()
    s.F = np.broadcast_to(np.eye(3) + 0.05 * rng.standard_normal((3, 3)), s.F.shape).copy()
    c = s.X.mean(0)
    s.vfield = 3.0 * np.cross(np.array([0.2, 1.0, -0.4]), s.X - c)
    s.target = scene.target
    return s


def check_case(scene, nsteps, every, tol=1e-3, E_dir_seed=0, check_E=True):
    from physbam_b200 import driver as D
    v0 = np.asarray(scene.V[0], float)
    E = scene.mu * 2 * (1 + 0.3)
    drv64, dt64, t64 = setup(scene, D.FP64)
    f_v = lambda v: loss_fn(drv64, scene, t64, dt64, v, E, nsteps, every, False)
    f_E = lambda e: loss_fn(drv64, scene, t64, dt64, v0, e, nsteps, every, False, part=True)
    L64, gv64, _ = loss_fn(drv64, scene, t64, dt64, v0, E, nsteps, every, True)
    _, _, gE64 = loss_fn(drv64, scene, t64, dt64, v0, E, nsteps, every, True, part=True)
    rng = np.random.default_rng(E_dir_seed)
    dirE = rng.standard_normal(scene.n) * E * 0.1
    ests_v = [fd(f_v, v0, np.eye(3)[k]) for k in range(3)]
    est_E = fd(lambda s: f_E(E + s * dirE), 0.0, 1.0, hs=(1e-2, 3e-3, 1e-3, 3e-4))
    drv32, dt32, t32 = setup(scene, D.FP32)
    L32, gv32, _ = loss_fn(drv32, scene, t32, dt32, v0, E, nsteps, every, True)
    _, _, gE32 = loss_fn(drv32, scene, t32, dt32, v0, E, nsteps, every, True, part=True)
    scale_v = np.linalg.norm(gv64)
    out = {}
    for name, gv, gE in (("fp64", gv64, gE64), ("fp32", gv32, gE32)):
        ev = max(abs(closest(ests_v[k], gv[k]) - gv[k]) for k in range(3)) / scale_v
        dE = float(np.dot(gE, dirE))
        eE = abs(closest(est_E, dE) - dE) / max(abs(closest(est_E, dE)), 1e-30)
        out[name] = (ev, eE)
        assert ev < tol, (name, "v0", ev, gv, ests_v)
        if check_E:
            assert eE < tol, (name, "E", eE, dE, est_E)
    drv64.close()
    drv32.close()
    print(scene.name, nsteps, every, {k: ("%.1e" % a, "%.1e" % b) for k, (a, b) in out.items()})
    return gv64, gE64


def test_adjoint_small_cube_fd(cuda_device):
    scene = deformed(S.cube_3d(G=16, nsteps=16))
    check_case(scene, 16, 4)


def test_adjoint_neohookean_fd(cuda_device):
    scene = deformed(S.cube_3d(G=16, nsteps=12, model=S.NEO_HOOKEAN, seed=3), seed=8)
    check_case(scene, 12, 3)


def test_checkpoint_interval_does_not_change_gradients(cuda_device):
    from physbam_b200 import driver as D
    scene = deformed(S.cube_3d(G=16, nsteps=12))
    v0 = np.asarray(scene.V[0], float)
    E = scene.mu * 2 * (1 + 0.3)
    res = []
    for every in (1, 5, 12):
        drv, dt, t = setup(scene, D.FP64)
        res.append(loss_fn(drv, scene, t, dt, v0, E, 12, every, True, part=True))
        drv.close()
    for r in res[1:]:
        np.testing.assert_allclose(r[1], res[0][1], rtol=1e-12)
        np.testing.assert_allclose(r[2], res[0][2], rtol=1e-10, atol=1e-12 * np.abs(res[0][2]).max())


def test_tape_budget_does_not_change_gradients(cuda_device):
    """A backward from every substep kept by the forward (the default budget) and
    one that recomputes each segment from its checkpoint (budget 0) agree."""
    from physbam_b200 import driver as D
    scene = deformed(S.cube_3d(G=16, nsteps=12))
    v0 = np.asarray(scene.V[0], float)
    E = scene.mu * 2 * (1 + 0.3)
    res = []
    for budget in (-1, 0):
        drv, dt, t = setup(scene, D.FP64)
        drv.set_diff_tape_budget(budget)
        res.append(loss_fn(drv, scene, t, dt, v0, E, 12, 4, True, part=True))
        drv.close()
    np.testing.assert_allclose(res[1][1], res[0][1], rtol=1e-12)
    np.testing.assert_allclose(res[1][2], res[0][2], rtol=1e-10, atol=1e-12 * np.abs(res[0][2]).max())


def test_adjoint_differentiable_config_fd(cuda_device):
    """The differentiable cube: 64^3, side-0.3 cube at 8 ppc, E log-uniform in
    [5e3, 5e4], v0 = (1, .5, 0), 64 substeps of 1e-4, checkpoint every 8."""
    scene = S.cube_3d()
    check_case(scene, 64, 8, check_E=False)
    # the body translates rigidly (uniform v0, gravity, F = I, no walls): E has no effect at all
    from physbam_b200 import driver as D
    drv, dt, t = setup(scene, D.FP32)
    E = scene.mu * 2 * (1 + 0.3)
    _, gv, gE = loss_fn(drv, scene, t, dt, np.asarray(scene.V[0], float), E, 64, 8, True, part=True)
    drv.close()
    assert np.max(np.abs(gE * E)) < 1e-6 * np.linalg.norm(gv)


def test_adjoint_differentiable_config_deformed_fd(cuda_device):
    """Same size and schedule, body pre-stressed and spinning so the E gradient is non-zero."""
    scene = deformed(S.cube_3d())
    check_case(scene, 64, 8)


def with_objects(scene):
    """The body meets static, frictionless collision objects during the rollout: a
    slip plane ahead of it in x (nodes beyond it are projected onto it), a
    separating sphere under its bottom face (curved: the projection's derivative
    has the curvature term) and a sticking box along its low-y face (nodes stop)."""
    s = scene.copy()
    s.target = scene.target
    if hasattr(scene, "vfield"):
        s.vfield = scene.vfield
    s.objects = [S.CollisionObject(S.PLANE, S.SLIP, 0.0, [-1.0, 0.0, 0.0], [0.66, 0.5, 0.5]),
                 S.CollisionObject(S.SPHERE, S.SEPARATE, 0.0, [0.5, 0.5, 0.25], [0.12, 0.0, 0.0]),
                 S.CollisionObject(S.BOX, S.STICK, 0.0, [-1.0, -1.0, -1.0], [2.0, 0.36, 2.0])]
    return s


def test_adjoint_with_collision_objects_fd(cuda_device):
    """The projection of MPM_OBJECTIVE::Test_Add_Collision (System/MPM_OBJECTIVE.cpp:150-183),
    transposed: gradients with a slip plane, a separating sphere and a sticking box."""
    scene = with_objects(deformed(S.cube_3d(G=16, nsteps=12)))
    check_case(scene, 12, 4)


def test_adjoint_differentiable_config_with_walls_fd(cuda_device):
    """The differentiable cube at full size (64^3, 64 substeps, checkpoint every 8) with the
    slip walls Add_Walls builds and a slip plane the cube runs into."""
    scene = S.cube_3d()
    s = scene.copy()
    s.target = scene.target
    s.objects = S.walls(3, s.counts, s.domain_min, s.domain_max, 63, S.SLIP, 0.0, 0.05) + [
        S.CollisionObject(S.PLANE, S.SLIP, 0.0, [-1.0, 0.0, 0.0], [0.653, 0.5, 0.5])]
    check_case(s, 64, 8, check_E=False)
