"""GPU tests of the FP64 diagnostics and the CFL time step (C ABI
mpm_particle_totals / mpm_grid_totals / mpm_compute_dt).

* Particle totals against the oracle's restatement of the reference's
  Total_Particle_* and Grid_V_Upper_Bound on the state read back from the GPU.
* Conservation: with no gravity and no collision objects, the grid after P2G and
  the force step carries the particles' mass, linear momentum and (APIC)
  angular momentum from before the substep, to roundoff.
* mpm_compute_dt against the reference's Compute_Dt formula.
"""
import numpy as np
import pytest

import oracle
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def D():
    from physbam_b200 import driver
    return driver


def quiet(scene):
    s = scene.copy()
    s.gravity = [0.0] * s.dim
    s.objects = []
    return s


def check_totals(got, want, rtol):
    scale_p = max(np.abs(want["momentum"]).max(), want["mass"] * 1e-3)
    assert got["count"] == want["count"]
    assert abs(got["mass"] - want["mass"]) <= rtol * want["mass"]
    assert np.abs(got["momentum"] - want["momentum"]).max() <= rtol * scale_p
    scale_l = max(np.abs(want["angular_momentum"]).max(), 1e-30)
    assert np.abs(got["angular_momentum"] - want["angular_momentum"]).max() <= rtol * scale_l
    assert abs(got["kinetic_energy"] - want["kinetic_energy"]) <= rtol * want["kinetic_energy"]


@pytest.mark.parametrize("path,precision", [("fast", "fp32"), ("plain", "fp64"), ("plain", "fp32")])
def test_particle_totals_match_oracle(cuda_device, path, precision):
    drv_mod = D()
    scene = S.small_3d(nsteps=5)
    pth = drv_mod.PATH_FAST if path == "fast" else drv_mod.PATH_PLAIN
    prec = drv_mod.FP32 if precision == "fp32" else drv_mod.FP64
    drv = drv_mod.MPM_DRIVER(scene, precision=prec, path=pth)
    drv.set_scene_particles(scene)
    drv.advance(5)
    got = drv.particle_totals()
    p = drv.get_particles()
    # the mass read back is the input mass, rounded to the path's precision
    m = scene.mass.astype(np.float32).astype(np.float64) if prec == drv_mod.FP32 else scene.mass
    want = oracle.particle_totals(p["X"], p["V"], p["B"], m, p["valid"], scene.dx)
    check_totals(got, want, 1e-9)
    assert abs(got["max_speed"] - want["max_speed"]) <= 1e-9 * want["max_speed"]
    assert abs(got["max_affine_speed"] - want["max_affine_speed"]) <= 1e-9 * want["max_affine_speed"]
    dt = drv.compute_dt(cfl=0.5, max_dt=1e-2)
    assert dt == pytest.approx(oracle.compute_dt(want["max_affine_speed"], scene.dx, 0.5, 1e-2), rel=1e-12)
    assert drv.compute_dt(cfl=0.5, max_dt=1e-9) == 1e-9     # below the critical speed: max_dt
    drv.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_plain_fp64_grid_conserves_momentum(cuda_device, dim):
    drv_mod = D()
    scene = quiet(S.small_3d() if dim == 3 else S.small_2d())
    drv = drv_mod.MPM_DRIVER(scene, precision=drv_mod.FP64, path=drv_mod.PATH_PLAIN)
    drv.set_scene_particles(scene)
    for _ in range(3):
        before = drv.particle_totals()
        drv.Particle_To_Grid()
        drv.Apply_Forces()
        grid = drv.grid_totals()
        check_totals({**grid, "count": before["count"], "kinetic_energy": before["kinetic_energy"]}, before, 1e-11)
        drv.Grid_To_Particle()
    drv.close()


def test_fast_grid_conserves_momentum(cuda_device):
    drv_mod = D()
    scene = quiet(S.small_3d())
    drv = drv_mod.MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    for _ in range(3):
        before = drv.particle_totals()
        drv.Particle_To_Grid()
        drv.Apply_Forces()
        grid = drv.grid_totals()
        g = drv.get_grid()
        assert grid["count"] == int((g["grid_m"] != 0).sum())
        check_totals({**grid, "count": before["count"], "kinetic_energy": before["kinetic_energy"]}, before, 2e-5)
        drv.Grid_To_Particle()
    drv.close()


def test_batch_totals_sum_scenes(cuda_device):
    drv_mod = D()
    scenes = S.batch_scenes(count=6)
    b = drv_mod.MPM_BATCH(scenes)
    b.set_scene_particles()
    b.advance(3)
    got = b.particle_totals()
    p = b.get_particles()
    parts = b.split({**p, "mass": np.concatenate([s.mass for s in scenes]).astype(np.float32).astype(np.float64)})
    mass = sum(q["mass"][q["valid"]].sum() for q in parts)
    mom = sum((q["mass"][q["valid"], None] * q["V"][q["valid"]]).sum(0) for q in parts)
    assert got["mass"] == pytest.approx(mass, rel=1e-12)
    np.testing.assert_allclose(got["momentum"], mom, rtol=1e-9, atol=1e-12 * mass)
    # per-scene xi = 6 sqrt(3) / dx of that scene; the batch reports the largest
    want = max(oracle.particle_totals(q["X"], q["V"], q["B"], q["mass"], q["valid"], s.dx)["max_affine_speed"]
               for q, s in zip(parts, scenes))
    assert got["max_affine_speed"] == pytest.approx(want, rel=1e-9)
    b.close()


def test_empty_totals(cuda_device):
    drv_mod = D()
    scene = S.small_3d().subset(np.arange(0))
    drv = drv_mod.MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    t = drv.particle_totals()
    assert t["count"] == 0 and t["mass"] == 0 and t["max_speed"] == 0
    assert drv.compute_dt(cfl=0.5, max_dt=1e-3) == 1e-3
    drv.close()
