"""GPU tests of plasticity after every G2P: snow (MPM_PLASTICITY_CLAMP) and
sand (MPM_DRUCKER_PRAGER with the St. Venant-Kirchhoff Hencky model).

* FP64 plain path vs the reference's own FP64 dumps of the snow and sand
  scenes (2D and 3D): F, Fp and the hardened mu, lambda (snow) or
  plastic_def, rho_F, sigma_Y, vc (sand) as well as X, V, B.
* FP32 fast path (plasticity fused into G2P) vs the same dumps at FP32 tolerances.
* A particle that leaves the domain in a substep is still updated by that
  substep's plasticity (MPM_DRIVER updates every simulated particle).
* The plastic state round-trips through the C ABI in the caller's order.
* Turning plasticity off restores the elastic substep; the autotuner restores
  the plastic state; the adjoint refuses plastic handles.
"""
import numpy as np
import pytest

import oracle
from make_golden import CASES, load
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu

SNOW = sorted(n for n in CASES if n.startswith("smallsnow"))
SAND = sorted(n for n in CASES if n.startswith("smallsand"))


def D():
    from physbam_b200 import driver
    return driver


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), floor)


def floors(scene, ref):
    vmax = max(float(np.max(np.abs(ref["V"]))), 1e-12)
    return {"X": 1.0, "V": vmax, "F": 1.0, "B": vmax / scene.dx, "Fp": 1.0, "mu": 1e-300, "lam": 1e-300,
            "pdef": 1e-300, "rho_F": 1e-300, "cohesion": 1.0, "vc": 1e-300}


TOL_FP64 = {"X": 1e-12, "V": 1e-9, "F": 1e-10, "B": 1e-8, "Fp": 1e-10, "mu": 1e-10, "lam": 1e-10,
            "pdef": 1e-10, "rho_F": 1e-10, "cohesion": 1e-12, "vc": 1e-10}
# FP32 after 20 substeps; the hardening exp(10 (1 - det Fp)) turns an FP32
# error of det Fp into ten times that in mu and lambda; the Drucker-Prager
# state is a sum of FP32 logarithms of the singular values.
# vc accumulates the log of the volume change over every yielding step (relative to its
# largest value); beside a stiff elastic body the FP32 sums reach 1.1e-4 after 20 steps.
TOL_FP32 = {"X": 2e-6, "V": 2e-3, "F": 1e-4, "B": 2e-3, "Fp": 1e-4, "mu": 1e-3, "lam": 1e-3,
            "pdef": 1e-4, "rho_F": 1e-5, "cohesion": 1e-6, "vc": 3e-4}


def run_snow(name, precision, path, tol, shape=None):
    scene, dumps = load(name)
    assert scene.plasticity is not None
    drv = D().MPM_DRIVER(scene, precision=precision, path=path)
    if shape is not None:
        drv.set_launch_shape(*shape)
    drv.set_scene_particles(scene)
    worst = {}
    for step in range(max(dumps) + 1):
        drv.Advance_One_Time_Step()
        if step not in dumps:
            continue
        ref = dumps[step]
        got = drv.get_particles()
        got.update(drv.get_plastic_state())
        np.testing.assert_array_equal(got["valid"], ref["valid"])
        fl = floors(scene, ref)
        for k in ("X", "V", "F", "B") + S.plastic_keys(scene.plasticity):
            e = rel(got[k], ref[k], fl[k])
            worst[k] = max(worst.get(k, 0), e)
            assert e < tol[k], (name, step, k, e)
    drv.close()
    print(name, {k: "%.1e" % v for k, v in worst.items()})
    return worst


@pytest.mark.parametrize("name", SNOW + SAND)
def test_plain_fp64_plastic_matches_reference(cuda_device, name):
    run_snow(name, D().FP64, D().PATH_PLAIN, TOL_FP64)


SHAPES = [(0, 128, 1), (2, 64, 2), (3, 256, 1)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "p2g%d-g2p%d-x%d" % s)
@pytest.mark.parametrize("name", [n for n in SNOW + SAND if "3d" in n])
def test_fast_fp32_plastic_matches_reference(cuda_device, name, shape):
    run_snow(name, D().FP32, D().PATH_FAST, TOL_FP32, shape)


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_drucker_prager_state_round_trip(cuda_device, path):
    s = S.small_sand_3d(nsteps=3)
    p, prec = (D().PATH_PLAIN, D().FP64) if path == "plain" else (D().PATH_FAST, D().FP32)
    drv = D().MPM_DRIVER(s, precision=prec, path=p)
    drv.set_scene_particles(s)
    st = drv.get_plastic_state()
    ref = oracle.State(s)
    for k in ("pdef", "rho_F", "cohesion", "vc"):
        np.testing.assert_allclose(st[k], getattr(ref, k), rtol=1e-6, atol=1e-30)
    drv.advance(3)
    before = drv.get_plastic_state()
    rng = np.random.default_rng(2)
    new = {"pdef": rng.uniform(0, 0.1, s.n), "vc": rng.uniform(-0.01, 0.01, s.n),
           "cohesion": rng.uniform(0, 50, s.n), "Fp": np.eye(3) + 0.01 * rng.standard_normal((s.n, 3, 3))}
    drv.set_plastic_state(**new)
    back = drv.get_plastic_state()
    r = 1e-15 if path == "plain" else 1e-7
    for k, v in new.items():
        np.testing.assert_allclose(back[k], v, rtol=r, atol=r * 1e-3)
    np.testing.assert_array_equal(back["rho_F"], before["rho_F"])     # not set: unchanged
    with pytest.raises(D().MPMError):          # the clamp's arrays on a Drucker-Prager handle
        drv.set_plastic_state(mu0=np.ones(s.n))
    drv.close()


def test_drucker_prager_fast_vs_plain_after_collision(cuda_device):
    """30 substeps of the sand block against the floor: the FP32 fast path (SVD-free
    return mapping in G2P) follows the FP64 plain path (the reference's SVD route)."""
    s = S.small_sand_3d(nsteps=30)
    out = {}
    for p, prec in ((D().PATH_PLAIN, D().FP64), (D().PATH_FAST, D().FP32)):
        drv = D().MPM_DRIVER(s, precision=prec, path=p)
        drv.set_scene_particles(s)
        drv.advance(s.nsteps)
        out[p] = (drv.get_particles(), drv.get_plastic_state())
        drv.close()
    (a, pa), (b, pb) = out[D().PATH_PLAIN], out[D().PATH_FAST]
    np.testing.assert_array_equal(a["valid"], b["valid"])
    assert rel(b["X"], a["X"], 1.0) < 2e-6
    assert rel(b["F"], a["F"], 1.0) < 1e-4
    assert rel(pb["pdef"], pa["pdef"]) < 1e-4
    assert (pa["pdef"] > 0).mean() > 0.5


def test_leaving_particle_gets_its_last_plastic_update(cuda_device):
    s = S.small_snow_3d(nsteps=1)
    s.objects = []
    s.X[0] = [0.5, 1.0 - 1e-5, 0.5]
    s.V[0] = [0.0, 50.0, 0.0]
    s.B[0] = 0
    st = oracle.State(s)
    oracle.substep(st)
    assert not st.valid[0]
    ref_Fp, ref_mu = st.Fp_rowmajor()[0], st.mu[0]
    assert np.abs(ref_Fp - np.eye(3)).max() > 1e-3, "the clamp must act on the leaving particle"
    for path, prec, tol in ((D().PATH_PLAIN, D().FP64, 1e-12), (D().PATH_FAST, D().FP32, 1e-5)):
        drv = D().MPM_DRIVER(s, precision=prec, path=path)
        drv.set_scene_particles(s)
        drv.Advance_One_Time_Step()
        got = drv.get_particles()
        np.testing.assert_array_equal(got["valid"], st.valid.astype(bool))
        pl = drv.get_plastic_state()
        assert np.abs(pl["Fp"][0] - ref_Fp).max() < tol, (path, pl["Fp"][0], ref_Fp)
        assert abs(pl["mu"][0] - ref_mu) < tol * ref_mu
        # the invalid particle keeps that state afterwards
        drv.Advance_One_Time_Step()
        np.testing.assert_array_equal(drv.get_plastic_state()["Fp"][0], pl["Fp"][0])
        drv.close()


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_plastic_state_round_trip(cuda_device, path):
    s = S.small_snow_3d(nsteps=4)
    p, prec = (D().PATH_PLAIN, D().FP64) if path == "plain" else (D().PATH_FAST, D().FP32)
    drv = D().MPM_DRIVER(s, precision=prec, path=p)
    drv.set_scene_particles(s)
    st = drv.get_plastic_state()
    np.testing.assert_array_equal(st["Fp"], np.broadcast_to(np.eye(3), st["Fp"].shape))
    np.testing.assert_allclose(st["mu0"], s.mu, rtol=1e-7)
    np.testing.assert_allclose(st["lam0"], s.lam, rtol=1e-7)
    drv.advance(3)      # the fast path reorders its particles
    rng = np.random.default_rng(9)
    Fp = np.eye(3) + 0.01 * rng.standard_normal((s.n, 3, 3))
    mu0 = s.mu * rng.uniform(0.5, 2.0, s.n)
    drv.set_plastic_state(Fp=Fp, mu0=mu0)
    back = drv.get_plastic_state()
    r = 1e-15 if path == "plain" else 1e-7
    np.testing.assert_allclose(back["Fp"], Fp, rtol=0, atol=r * 2)
    np.testing.assert_allclose(back["mu0"], mu0, rtol=r)
    np.testing.assert_allclose(back["lam0"], st["lam0"], rtol=r)
    drv.close()


def test_custom_plastic_state_fast_vs_plain(cuda_device):
    """A non-trivial plastic start, set through the ABI, evolves alike on both paths."""
    s = S.small_snow_3d(nsteps=6)
    rng = np.random.default_rng(4)
    Fp = np.eye(3) + 0.02 * rng.standard_normal((s.n, 3, 3))
    mu0, lam0 = s.mu * rng.uniform(0.8, 1.2, s.n), s.lam * rng.uniform(0.8, 1.2, s.n)
    out = {}
    for p, prec in ((D().PATH_PLAIN, D().FP64), (D().PATH_FAST, D().FP32)):
        drv = D().MPM_DRIVER(s, precision=prec, path=p)
        drv.set_scene_particles(s)
        drv.set_plastic_state(Fp=Fp, mu0=mu0, lam0=lam0)
        for _ in range(s.nsteps):
            drv.Advance_One_Time_Step()
        out[p] = (drv.get_particles(), drv.get_plastic_state())
        drv.close()
    (a, pa), (b, pb) = out[D().PATH_PLAIN], out[D().PATH_FAST]
    np.testing.assert_array_equal(a["valid"], b["valid"])
    assert rel(b["X"], a["X"], 1.0) < 2e-6
    assert rel(b["F"], a["F"], 1.0) < 1e-4
    assert rel(pb["Fp"], pa["Fp"], 1.0) < 1e-4
    assert rel(pb["mu"], pa["mu"]) < 1e-3


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_plasticity_off_is_elastic(cuda_device, path):
    s = S.small_snow_3d(nsteps=5)
    p, prec = (D().PATH_PLAIN, D().FP64) if path == "plain" else (D().PATH_FAST, D().FP32)
    res = []
    for toggle in (False, True):
        e = s.copy()
        e.plasticity = None if not toggle else s.plasticity
        drv = D().MPM_DRIVER(e, precision=prec, path=p)
        drv.set_scene_particles(e)
        if toggle:
            drv.set_plasticity(None)
        for _ in range(5):
            drv.Advance_One_Time_Step()
        res.append(drv.get_particles())
        drv.close()
    # same kernels, same inputs: only the order of atomic sums differs
    tol = 1e-13 if path == "plain" else 1e-6
    for k in ("X", "F"):
        assert rel(res[1][k], res[0][k], 1.0) < tol, k


def test_plasticity_changes_the_motion(cuda_device):
    s = S.small_snow_3d(nsteps=10)
    e = s.copy()
    e.plasticity = None
    out = []
    for sc in (s, e):
        drv = D().MPM_DRIVER(sc)
        drv.set_scene_particles(sc)
        drv.advance(10)
        out.append(drv.get_particles()["F"])
        drv.close()
    sv = np.linalg.svd(out[0], compute_uv=False)
    pl = s.plasticity
    assert sv.min() >= 1 - pl.theta_c - 1e-5 and sv.max() <= 1 + pl.theta_s + 1e-5
    assert np.abs(out[0] - out[1]).max() > 1e-3


def test_graph_advance_with_plasticity_matches_eager(cuda_device):
    s = S.small_snow_3d(nsteps=7)
    res = []
    for graph in (False, True):
        drv = D().MPM_DRIVER(s)
        drv.set_scene_particles(s)
        if graph:
            drv.advance(7)
        else:
            for _ in range(7):
                drv.Advance_One_Time_Step()
        res.append((drv.get_particles(), drv.get_plastic_state()))
        drv.close()
    assert rel(res[1][0]["X"], res[0][0]["X"], 1.0) < 1e-6
    assert rel(res[1][1]["Fp"], res[0][1]["Fp"], 1.0) < 1e-5


def test_autotune_restores_plastic_state(cuda_device):
    s = S.small_snow_3d(nsteps=6)
    drv = D().MPM_DRIVER(s)
    drv.set_scene_particles(s)
    drv.advance(2)
    before = drv.get_plastic_state()
    drv.autotune(substeps=1)
    after = drv.get_plastic_state()
    for k in before:
        np.testing.assert_array_equal(before[k], after[k])
    drv.close()


def test_batch_with_plasticity_matches_individual(cuda_device):
    scenes = [S.small_snow_3d(seed=21 + k, nsteps=6) for k in range(3)]
    batch = D().MPM_BATCH(scenes)
    batch.set_scene_particles()
    batch.advance(6)
    got = batch.split(batch.get_particles())
    batch.close()
    for sc, g in zip(scenes, got):
        drv = D().MPM_DRIVER(sc)
        drv.set_scene_particles(sc)
        drv.advance(6)
        ref = drv.get_particles()
        drv.close()
        np.testing.assert_array_equal(g["valid"], ref["valid"])
        assert rel(g["X"], ref["X"], 1.0) < 1e-6 and rel(g["F"], ref["F"], 1.0) < 1e-4


def test_bad_plasticity_arguments(cuda_device):
    s = S.small_snow_3d(nsteps=1)
    drv = D().MPM_DRIVER(s)
    for bad in (S.Plasticity(theta_c=1.5), S.Plasticity(theta_s=-1.0), S.Plasticity(kind=7),
                S.DruckerPrager(a0=10.0, a4=10.0), S.DruckerPrager(cohesion=float("nan"))):
        with pytest.raises(D().MPMError):
            drv.set_plasticity(bad)
    drv.set_plasticity(None)
    drv.set_scene_particles(s)
    with pytest.raises(D().MPMError):
        drv.get_plastic_state()
    drv.close()


def test_adjoint_refuses_plasticity(cuda_device):
    s = S.small_snow_3d(nsteps=2)
    drv = D().MPM_DRIVER(s, precision=D().FP64, path=D().PATH_PLAIN)
    drv.set_scene_particles(s)
    with pytest.raises(D().MPMError):
        drv.diff_forward(2)
    drv.close()
