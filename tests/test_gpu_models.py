"""GPU tests of per-particle constitutive models (mpm_set_particle_models).

Parity with the reference's own dumps of a two-material scene (one
MPM_FINITE_ELEMENTS force per model over its particles) and of sand beside an
elastic body (the plasticity over the sand alone) runs with the other
fixtures: test_gpu_parity.py (explicit: plain FP64, fast FP32 in every launch
shape), test_gpu_plasticity.py and test_gpu_implicit.py (backward Euler).
Here: the argument checks, that a per-particle array naming the handle's model
everywhere reproduces the single-model run, and the particles outside the
plastic subset.
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


def test_model_arguments(cuda_device):
    s = S.small_3d(nsteps=1)
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    with pytest.raises(D().MPMError):
        drv.set_particle_models(np.zeros(s.n, np.uint8))          # before the particles
    drv.set_scene_particles(s)
    with pytest.raises(D().MPMError):
        drv.set_particle_models(np.zeros(s.n - 1, np.uint8))      # one per particle
    with pytest.raises(D().MPMError):
        drv.set_particle_models(np.full(s.n, 7, np.uint8))        # unknown model
    drv.set_particle_models(np.ones(s.n, np.uint8))
    drv.set_particle_models(None)
    drv.close()
    fast = D().MPM_DRIVER(s, precision=D().FP32, path=D().PATH_FAST)
    fast.set_scene_particles(s)
    with pytest.raises(D().MPMError):
        fast.set_particle_models(np.zeros(s.n + 1, np.uint8))
    fast.set_particle_models(np.zeros(s.n, np.uint8))
    fast.close()


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_uniform_models_equal_the_scene_model(cuda_device, path):
    s = S.small_3d(model=S.NEO_HOOKEAN, nsteps=5)
    p, prec = (D().PATH_PLAIN, D().FP64) if path == "plain" else (D().PATH_FAST, D().FP32)
    out = []
    for models in (None, np.full(s.n, S.NEO_HOOKEAN, np.uint8)):
        e = s.copy()
        e.models = models
        drv = D().MPM_DRIVER(e, precision=prec, path=p)
        drv.set_scene_particles(e)
        for _ in range(5):
            drv.Advance_One_Time_Step()
        out.append(drv.get_particles())
        drv.close()
    tol = 1e-13 if path == "plain" else 1e-6
    for k in ("X", "V", "F"):
        assert rel(out[1][k], out[0][k], 1.0) < tol, k


@pytest.mark.parametrize("implicit", [False, True])
def test_uniform_models_equal_the_handle_model(cuda_device, implicit):
    s = S.small_3d(model=S.NEO_HOOKEAN, nsteps=5)
    if implicit:
        s.implicit, s.dt = S.Implicit(), 1e-3
    out = []
    for models in (None, np.full(s.n, S.NEO_HOOKEAN, np.uint8)):
        e = s.copy()
        e.models = models
        drv = D().MPM_DRIVER(e, precision=D().FP64, path=D().PATH_PLAIN)
        drv.set_scene_particles(e)
        for _ in range(5):
            drv.Advance_One_Time_Step()
        out.append(drv.get_particles())
        drv.close()
    # implicit: two runs of the same solve may take different Newton paths (the order of
    # the atomic sums), within the bounds of the implicit parity tests
    tol = {"X": 2e-9, "V": 1e-6, "F": 1e-7} if implicit else dict.fromkeys(("X", "V", "F"), 1e-13)
    for k in ("X", "V", "F"):
        assert rel(out[1][k], out[0][k], 1.0) < tol[k], k


def test_plastic_particles(cuda_device):
    """mpm_set_plastic_particles: argument checks; a mask naming every particle
    reproduces the plasticity over all; the particles outside it keep Fp = I."""
    s = S.small_sand_3d(nsteps=5)
    out = []
    for mask in (None, np.ones(s.n, np.uint8)):
        e = s.copy()
        e.plastic_mask = mask
        drv = D().MPM_DRIVER(e, precision=D().FP64, path=D().PATH_PLAIN)
        drv.set_scene_particles(e)
        for _ in range(5):
            drv.Advance_One_Time_Step()
        out.append(drv.get_particles())
        out[-1].update(drv.get_plastic_state())
        drv.close()
    for k in ("X", "F", "Fp", "pdef"):
        assert rel(out[1][k], out[0][k], 1.0) < 1e-13, k
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(s)
    with pytest.raises(D().MPMError):
        drv.set_plastic_particles(np.ones(s.n + 1, np.uint8))
    half = (np.arange(s.n) % 2).astype(np.uint8)
    drv.set_plastic_particles(half)
    for _ in range(5):
        drv.Advance_One_Time_Step()
    st = drv.get_plastic_state()
    drv.close()
    off = half == 0
    np.testing.assert_array_equal(st["Fp"][off], np.broadcast_to(np.eye(3), (int(off.sum()), 3, 3)))
    assert np.all(st["pdef"][off] == 0) and np.all(st["rho_F"][off] == 0)
    fast = D().MPM_DRIVER(s, precision=D().FP32, path=D().PATH_FAST)
    fast.set_scene_particles(s)
    fast.set_plastic_particles(half)
    for _ in range(5):
        fast.Advance_One_Time_Step()
    st = fast.get_plastic_state()
    fast.close()
    np.testing.assert_array_equal(st["Fp"][off], np.broadcast_to(np.eye(3), (int(off.sum()), 3, 3)))
    assert np.all(st["pdef"][off] == 0) and np.all(st["rho_F"][off] == 0)
    assert np.abs(st["Fp"][~off] - np.eye(3)).max() > 1e-4   # the sand half did yield
