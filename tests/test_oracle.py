"""CPU tests: the C restatement (oracle/) reproduces the reference's own dumps.

The fixtures in tests/golden/ were written by the reference's MPM_DRIVER
(compiled from its sources, driven by oracle/ref_scene.cpp) in FP64.  Passing
here pins the oracle that the GPU parity tests then use.
"""
import numpy as np
import pytest

import oracle
from make_golden import CASES, load
from physbam_b200 import scenes as S

# The restatement follows the reference's operation order, so it agrees to a
# few ulps per step; B carries a cancellation (sum w vf Z - Vpf X) that
# amplifies ulps by |Z|/dx, hence its looser bound.
TOL = {"X": 1e-13, "V": 1e-12, "F": 1e-12, "B": 1e-11, "grid_m": 1e-13, "grid_v0": 1e-12,
       "grid_v": 1e-12, "grid_vf": 1e-12, "Fp": 1e-12, "mu": 1e-12, "lam": 1e-12,
       "pdef": 1e-12, "rho_F": 1e-12, "cohesion": 1e-15, "vc": 1e-12}


def rel(a, b, floor=1e-300):
    """max |a-b| over max |b|; `floor` bounds the scale from below where b is pure roundoff (e.g. B of a body at rest)."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b))) / scale


def floors(scene, ref):
    vmax = max(float(np.max(np.abs(ref["V"]))), 1e-12)
    return {"X": 1.0, "V": vmax, "F": 1.0, "B": vmax / scene.dx, "grid_m": 1e-300, "grid_v0": vmax,
            "grid_v": vmax, "grid_vf": vmax, "Fp": 1.0, "mu": 1e-300, "lam": 1e-300,
            "pdef": 1e-300, "rho_F": 1e-300, "cohesion": 1.0, "vc": 1e-300}


# the backward-Euler, adaptive-frame, reflection and caller-force cases pin the
# GPU path directly against the reference's dumps; the C restatement covers the
# symplectic-Euler substep with its collision objects (static, moving and
# penalty), several materials and plasticity (also over a particle subset)
EXPLICIT = sorted(n for n in CASES if not any(k in n for k in ("implicit", "adaptive", "reflect", "node_force")))


@pytest.mark.parametrize("name", EXPLICIT)
def test_oracle_matches_reference_dumps(name):
    scene, dumps = load(name)
    st = oracle.State(scene)
    last = max(dumps)
    for step in range(last + 1):
        g = oracle.substep(st, want_grid=step in dumps)
        if step not in dumps:
            continue
        ref = dumps[step]
        np.testing.assert_array_equal(st.valid.astype(bool), ref["valid"])
        fl = floors(scene, ref)
        got = {"X": st.X, "V": st.V, "F": st.F_rowmajor(), "B": st.B_rowmajor()}
        if scene.plasticity is not None:
            got.update(st.plastic_state())
        for k, v in got.items():
            e = rel(v, ref[k], fl[k])
            assert e < TOL[k], (name, step, k, e)
        for k in ("grid_m", "grid_v0", "grid_v", "grid_vf"):
            if k in ref:
                e = rel(g[k], ref[k], fl[k])
                assert e < TOL[k], (name, step, k, e)


def test_fixture_scenes_exercise_collisions():
    """The fixtures must reach the collision and friction code: some nodes change velocity there."""
    scene, dumps = load("small3d_neohookean_friction")
    st = oracle.State(scene)
    g = oracle.substep(st, want_grid=True)
    m = g["grid_m"] > 0
    v_unconstrained_close = np.all(np.isclose(g["grid_v"][m], g["grid_vf"][m]))
    assert not v_unconstrained_close, "friction never acted"
    assert len(scene.objects) >= 3


def test_svd3_reconstructs_and_signs():
    rng = np.random.default_rng(3)
    for trial in range(200):
        A = rng.standard_normal((3, 3))
        if trial % 3 == 0:
            A[:, 2] = A[:, 0] * 0.999 + 1e-9 * rng.standard_normal(3)   # nearly singular
        if trial % 5 == 0:
            A = -A                                                      # inverted
        U, s, V = np.zeros(9), np.zeros(3), np.zeros(9)
        Fc = np.ascontiguousarray(A.T.reshape(-1))
        it = oracle.lib().oracle_svd3(oracle._ptr(Fc), oracle._ptr(U), oracle._ptr(s), oracle._ptr(V))
        assert it >= 0
        Um, Vm = U.reshape(3, 3).T, V.reshape(3, 3).T
        np.testing.assert_allclose(Um @ np.diag(s) @ Vm.T, A, atol=1e-12 * np.abs(A).max())
        assert np.linalg.det(Um) > 0 and np.linalg.det(Vm) > 0
        assert s[0] >= s[1] >= abs(s[2]) - 1e-15


def test_pft_matches_closed_forms():
    """P F^T from the SVD route equals the SVD-free forms the fast path uses."""
    rng = np.random.default_rng(5)
    for _ in range(100):
        A = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if np.linalg.det(A) <= 0.3:
            continue
        mu, la = 1e4 * rng.uniform(0.5, 2), 2e4 * rng.uniform(0.5, 2)
        Fc = np.ascontiguousarray(A.T.reshape(-1))
        b = A @ A.T
        J = np.linalg.det(A)
        w, Q = np.linalg.eigh(b)
        sqrt_b = Q @ np.diag(np.sqrt(w)) @ Q.T
        coro = 2 * mu * (b - sqrt_b) + la * J * (J - 1) * np.eye(3)
        nh = mu * (b - np.eye(3)) + la * np.log(J) * np.eye(3)
        got_c = oracle.pft(3, 0, Fc, mu, la).reshape(3, 3).T
        got_n = oracle.pft(3, 1, Fc, mu, la).reshape(3, 3).T
        np.testing.assert_allclose(got_c, coro, rtol=1e-9, atol=1e-9 * np.abs(coro).max())
        np.testing.assert_allclose(got_n, nh, rtol=1e-9, atol=1e-9 * np.abs(nh).max())


@pytest.mark.skipif(not oracle.ref_available(), reason="reference runner not built (no reference sources)")
@pytest.mark.parametrize("dim", [2, 3])
def test_totals_match_reference(dim):
    """oracle.particle_totals / compute_dt against the reference's own
    Total_Particle_*, Grid_V_Upper_Bound and Compute_Dt on the same final state."""
    scene = S.small_3d(nsteps=4) if dim == 3 else S.small_2d(nsteps=4)
    # a CFL small enough that the affine speed bound decides the step
    cfl, max_dt = 1e-3, 1e-2
    dumps, ref = oracle.run_reference(scene, [scene.nsteps - 1], threads=2, totals=(cfl, max_dt))
    last = dumps[scene.nsteps - 1]
    got = oracle.particle_totals(last["X"], last["V"], last["B"], scene.mass, last["valid"], scene.dx)
    assert got["count"] == ref["count"]
    assert got["mass"] == pytest.approx(ref["mass"], rel=1e-13)
    np.testing.assert_allclose(got["momentum"][:dim], ref["momentum"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(got["angular_momentum"][:len(ref["angular_momentum"])], ref["angular_momentum"],
                               rtol=1e-12, atol=1e-14)
    assert got["kinetic_energy"] == pytest.approx(ref["kinetic_energy"], rel=1e-12)
    assert got["max_speed"] == pytest.approx(ref["max_speed"], rel=1e-13)
    assert got["max_affine_speed"] == pytest.approx(ref["max_affine_speed"], rel=1e-13)
    dt = oracle.compute_dt(got["max_affine_speed"], scene.dx, cfl, max_dt)
    assert dt < max_dt
    assert dt == pytest.approx(ref["dt"], rel=1e-13)


def test_snow_fixtures_exercise_plasticity():
    """The snow fixtures clamp singular values and harden: Fp leaves the identity
    and mu grows for some particles."""
    for name in ("smallsnow3d_corotated", "smallsnow2d_corotated"):
        scene, dumps = load(name)
        ref = dumps[max(dumps)]
        d = scene.dim
        assert np.abs(ref["Fp"] - np.eye(d)).max() > 1e-3, name
        assert (ref["mu"] / scene.mu).max() > 1.05, name
        sv = np.linalg.svd(ref["F"], compute_uv=False)
        pl = scene.plasticity
        assert sv.min() >= 1 - pl.theta_c - 1e-12 and sv.max() <= 1 + pl.theta_s + 1e-12, name


def test_sand_fixtures_exercise_every_branch():
    """The sand fixtures leave particles in all three cases of the Drucker-Prager
    return mapping: elastic (no plastic deformation yet), the tip (vc != 0) and
    the cone (plastic deformation, vc = 0)."""
    for name in ("smallsand3d_hencky", "smallsand2d_hencky"):
        scene, dumps = load(name)
        ref = dumps[max(dumps)]
        elastic = ref["pdef"] == 0
        assert 0.05 < elastic.mean() < 0.95, name
        if scene.plasticity.use_vc:
            assert (ref["vc"] != 0).mean() > 0.05, name
        assert ((ref["pdef"] > 0) & (ref["vc"] == 0)).mean() > 0.05, name
        assert scene.model == S.HENCKY


def test_drucker_prager_parameter_forms():
    """Add_Drucker_Prager_Case and the friction-angle form of Add_Drucker_Prager
    (STANDARD_TESTS_BASE.cpp:437-464) map onto the hardening constants."""
    assert S.DruckerPrager.mast_case(2) == S.DruckerPrager(a0=35.0, a1=9.0, a3=0.3, a4=10.0)
    assert S.sand_3d(G=16).plasticity == S.DruckerPrager.mast_case(2)
    assert len(S.MAST_CASES) == 10 and all(len(c) == 4 for c in S.MAST_CASES)
    f = S.DruckerPrager.friction_angle(30.0, cohesion=5.0)
    assert (f.a0, f.a1, f.a3, f.a4, f.cohesion) == (30.0, 0.0, 0.0, 0.0, 5.0)
