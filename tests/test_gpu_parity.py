"""GPU parity tests: the CUDA paths, called through the C ABI, against the reference.

* FP64 plain path vs the reference's own FP64 dumps (tests/golden), node for node.
* FP32 fast path vs the same dumps, at FP32 tolerances stated per quantity.
* Radix sort and the fast path's cell keys bit-exact against a CPU stable sort.
* Full-size two-sphere case (128^3, 200 substeps): FP32 fast path
  within 1e-4 relative position error of the FP64 plain path.
* Edge cases: empty particle set, particles leaving the domain, NaN input,
  particles outside the grid.
"""
import numpy as np
import pytest

import oracle
from make_golden import CASES, load
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def D():
    from physbam_b200 import driver
    return driver


def rel(a, b, floor=1e-300):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), floor)


def floors(scene, ref):
    vmax = max(float(np.max(np.abs(ref["V"]))), 1e-12)
    return {"X": 1.0, "V": vmax, "F": 1.0, "B": vmax / scene.dx, "grid_m": 1e-300, "grid_v0": vmax,
            "grid_v": vmax, "grid_vf": vmax}


# FP64 GPU vs FP64 reference: FMA contraction and atomic summation order are
# the only differences, so agreement is near machine precision.
TOL_FP64 = {"X": 1e-12, "V": 1e-9, "F": 1e-10, "B": 1e-8, "grid_m": 1e-12, "grid_v0": 1e-10,
            "grid_v": 1e-9, "grid_vf": 1e-9}
# FP32 GPU vs FP64 reference after up to 20 substeps (relative to the floors above).
TOL_FP32 = {"X": 2e-6, "V": 2e-3, "F": 1e-4, "B": 2e-3, "grid_m": 1e-5, "grid_v": 1e-3, "grid_vf": 1e-3}


def run_case(name, precision, path, tol, shape=None):
    scene, dumps = load(name)
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
        np.testing.assert_array_equal(got["valid"], ref["valid"])
        fl = floors(scene, ref)
        for k in ("X", "V", "F", "B"):
            e = rel(got[k], ref[k], fl[k])
            worst[k] = max(worst.get(k, 0), e)
            assert e < tol[k], (name, step, k, e)
        if "grid_m" in ref:
            g = drv.get_grid(want_v0=(path == D().PATH_PLAIN))
            for k in ("grid_m", "grid_v0", "grid_v", "grid_vf"):
                if k in g and k in tol:
                    e = rel(g[k], ref[k], fl[k])
                    worst[k] = max(worst.get(k, 0), e)
                    assert e < tol[k], (name, step, k, e)
    drv.synchronize()
    drv.close()
    print(name, {k: "%.1e" % v for k, v in worst.items()})
    return worst


# fixed-step symplectic-Euler cases (the implicit and adaptive-frame fixtures
# have their own tests)
FIXED = sorted(n for n in CASES if "implicit" not in n and "adaptive" not in n)
# the fast path has no reflection boundary conditions
FAST = sorted(n for n in FIXED if n.startswith("small3d") and "reflect" not in n)


@pytest.mark.parametrize("name", FIXED)
def test_plain_fp64_matches_reference(cuda_device, name):
    run_case(name, D().FP64, D().PATH_PLAIN, TOL_FP64)


# launch shapes: (P2G variant, G2P threads per CTA, CTA multiplier)
SHAPES = [(0, 128, 1), (1, 64, 2), (2, 256, 1), (2, 128, 2), (3, 64, 1), (3, 128, 2)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "p2g%d-g2p%d-x%d" % s)
@pytest.mark.parametrize("name", FAST)
def test_fast_fp32_matches_reference(cuda_device, name, shape):
    run_case(name, D().FP32, D().PATH_FAST, TOL_FP32, shape)


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "p2g%d-g2p%d-x%d" % s)
@pytest.mark.parametrize("model", [S.COROTATED, S.NEO_HOOKEAN])
def test_fast_stress_fallback_matches_plain_fp64(cuda_device, model, shape):
    """Inverted and nearly flat F take the FP64 SVD route on the fast path
    (the P2G launch adds their force once every part is done, in every launch shape)."""
    scene = S.small_3d(model=model, nsteps=3)
    rng = np.random.default_rng(5)
    n = scene.n
    F = scene.F.copy()
    inv = rng.random(n) < 0.3
    F[inv, :, 0] *= -1.0                                  # det < 0
    flat = (~inv) & (rng.random(n) < 0.15)
    F[flat, :, 2] *= 5e-3                                 # sigma_min / sigma_max < 1e-2
    scene.F = F
    got = {}
    for prec, path, sh in ((D().FP64, D().PATH_PLAIN, None), (D().FP32, D().PATH_FAST, shape)):
        drv = D().MPM_DRIVER(scene, precision=prec, path=path)
        if sh is not None:
            drv.set_launch_shape(*sh)
        drv.set_scene_particles(scene)
        for _ in range(scene.nsteps):
            drv.Advance_One_Time_Step()
        got[path] = drv.get_particles()
        drv.close()
    ref, fast = got[D().PATH_PLAIN], got[D().PATH_FAST]
    np.testing.assert_array_equal(fast["valid"], ref["valid"])
    vmax = float(np.abs(ref["V"]).max())
    assert rel(fast["X"], ref["X"], 1.0) < 2e-6
    assert rel(fast["V"], ref["V"], vmax) < 2e-3
    assert rel(fast["F"], ref["F"], 1.0) < 1e-4


def test_launch_shape_round_trip(cuda_device):
    scene = S.small_3d(nsteps=1)
    drv = D().MPM_DRIVER(scene)
    drv.set_launch_shape(2, 64, 2)
    assert drv.get_launch_shape() == (2, 64, 2)
    for bad in [(4, 128, 1), (-1, 128, 1), (0, 96, 1), (0, 128, 3)]:
        with pytest.raises(D().MPMError):
            drv.set_launch_shape(*bad)
    assert drv.get_launch_shape() == (2, 64, 2)
    drv.close()


@pytest.mark.parametrize("n,bits", [(0, 8), (1, 8), (2047, 11), (2048, 16), (2049, 17), (100_003, 25),
                                    (1_000_000, 32), (300_000, 6), (3_000_001, 30)])
def test_radix_sort_bit_exact(cuda_device, n, bits):
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    if n > 10:
        keys[::7] = keys[3]              # many duplicates, to test stability
    sk, perm = D().radix_sort_u32(keys, bits)
    mask = np.uint32((1 << bits) - 1) if bits < 32 else np.uint32(0xffffffff)
    ref = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(perm, ref.astype(np.uint32))
    np.testing.assert_array_equal(sk, keys[ref])


def cpu_cell_keys(scene, X32):
    """The fast path's key, in the same float32 arithmetic: block of 4^3 cells << 6 | cell in block."""
    dx = np.float32(scene.dx)
    inv = np.float32(1.0 / scene.dx)
    dmin = np.float32(scene.domain_min[0])
    cc = np.floor(((X32 - dx) - dmin) * inv).astype(np.int64) + S.GHOST
    NB = (np.asarray(scene.counts) + 4 + 3) // 4
    b = ((cc[:, 0] >> 2) * NB[1] + (cc[:, 1] >> 2)) * NB[2] + (cc[:, 2] >> 2)
    return ((b << 6) | ((cc[:, 0] & 3) << 4) | ((cc[:, 1] & 3) << 2) | (cc[:, 2] & 3)).astype(np.uint32)


def test_fast_cell_keys_and_sort_bit_exact(cuda_device):
    """The fast path's cell keys equal the CPU's (same float32 arithmetic).
    Freshly set particles are radix-sorted by their full keys once; from then on
    every substep's order is the previous one routed by the moves G2P counted,
    which must equal a CPU stable sort of the slots' keys by block (key >> 6)."""
    scene = S.spheres_3d(G=64, ppc=4, nsteps=3)
    drv = D().MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    drv.Particle_To_Grid()
    keys, sk, perm = drv.sort_state()
    X32 = scene.X.astype(np.float32)
    np.testing.assert_array_equal(keys, np.sort(cpu_cell_keys(scene, X32), kind="stable"))
    ref = np.argsort(keys >> 6, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(sk, keys[ref])
    drv.Apply_Forces()
    drv.Grid_To_Particle()
    for step in range(8):
        drv.Particle_To_Grid()
        keys, sk, perm = drv.sort_state()
        ref = np.argsort(keys >> 6, kind="stable").astype(np.uint32)
        np.testing.assert_array_equal(perm, ref, err_msg="substep %d" % step)
        np.testing.assert_array_equal(sk, keys[ref])
        drv.Apply_Forces()
        drv.Grid_To_Particle()
    drv.close()


def test_fast_vs_plain_fp64_full_size_spheres(cuda_device):
    """The full-size two-sphere case (128^3, NEO_HOOKEAN, 200 substeps):
    FP32 fast path within 1e-4 relative position error of the FP64 plain path."""
    scene = S.spheres_3d()
    out = {}
    for prec, path in ((D().FP64, D().PATH_PLAIN), (D().FP32, D().PATH_FAST)):
        drv = D().MPM_DRIVER(scene, precision=prec, path=path)
        drv.set_scene_particles(scene)
        drv.advance(scene.nsteps)
        out[path] = drv.get_particles()
        drv.close()
    ref, got = out[D().PATH_PLAIN], out[D().PATH_FAST]
    np.testing.assert_array_equal(got["valid"], ref["valid"])
    err = np.linalg.norm(got["X"] - ref["X"]) / np.linalg.norm(ref["X"])
    disp = np.linalg.norm(got["X"] - ref["X"]) / np.linalg.norm(ref["X"] - scene.X)
    assert err <= 1e-4, err
    assert disp <= 1e-2, disp    # also small against the distance actually travelled
    vrel = np.linalg.norm(got["V"] - ref["V"]) / np.linalg.norm(ref["V"])
    frel = np.linalg.norm(got["F"] - ref["F"]) / np.linalg.norm(ref["F"])
    print("spheres3d: X %.2e  disp %.2e  V %.2e  F %.2e" % (err, disp, vrel, frel))
    assert vrel < 1e-2 and frel < 1e-4


def test_graph_advance_matches_eager(cuda_device):
    scene = S.small_3d(nsteps=9)
    res = []
    for graph in (False, True):
        drv = D().MPM_DRIVER(scene)
        drv.set_scene_particles(scene)
        if graph:
            drv.advance(9)
        else:
            for _ in range(9):
                drv.Advance_One_Time_Step()
        res.append(drv.get_particles())
        drv.close()
    for k in ("X", "F"):
        assert rel(res[1][k], res[0][k], 1.0) < 1e-6


@pytest.mark.parametrize("path", ["fast", "plain"])
def test_timed_substeps_match_untimed(cuda_device, path):
    """With per-kernel timing on, the substeps run eagerly with events around
    each kernel: the state equals the untimed (graph-replayed) run's, and every
    kernel of the substep is timed once per substep."""
    scene = S.small_3d(nsteps=6)
    p = D().PATH_FAST if path == "fast" else D().PATH_PLAIN
    prec = D().FP32 if path == "fast" else D().FP64
    res, timers = [], None
    for timed in (False, True):
        drv = D().MPM_DRIVER(scene, precision=prec, path=p)
        drv.set_scene_particles(scene)
        drv.advance(2)
        drv.set_timing(timed)
        for _ in range(4):
            drv.Advance_One_Time_Step()
        drv.synchronize()
        if timed:
            timers = drv.get_timing()
        res.append(drv.get_particles())
        drv.close()
    for k in ("X", "V", "F"):
        assert rel(res[1][k], res[0][k], 1.0) < 1e-6, k
    names = ("fast_bins", "fast_route", "fast_p2g", "fast_grid", "fast_g2p") if path == "fast" else \
        ("plain_p2g", "plain_g2p")
    for name in names:
        assert name in timers and timers[name][1] == 4 and timers[name][0] > 0, (name, timers.get(name))


def test_empty_and_leaving_particles(cuda_device):
    scene = S.small_3d(with_walls=False)
    for path, prec in ((D().PATH_FAST, D().FP32), (D().PATH_PLAIN, D().FP64)):
        drv = D().MPM_DRIVER(scene.subset(slice(0, 0)), precision=prec, path=path)
        drv.set_scene_particles(scene.subset(slice(0, 0)))
        drv.Advance_One_Time_Step()
        drv.synchronize()
        assert drv.count_valid() == 0
        drv.close()
    # a fast particle next to the top face leaves the domain in one substep and is invalidated
    s = scene.copy()
    s.X[0] = [0.5, 1.0 - 1e-5, 0.5]
    s.V[0] = [0.0, 50.0, 0.0]
    s.B[0] = 0
    st = oracle.State(s)
    oracle.substep(st)
    for path, prec in ((D().PATH_FAST, D().FP32), (D().PATH_PLAIN, D().FP64)):
        drv = D().MPM_DRIVER(s, precision=prec, path=path)
        drv.set_scene_particles(s)
        drv.Advance_One_Time_Step()
        got = drv.get_particles()
        assert not got["valid"][0]
        np.testing.assert_array_equal(got["valid"], st.valid.astype(bool))
        assert drv.count_valid() == s.n - 1
        for _ in range(3):      # invalid particles keep their last state
            drv.Advance_One_Time_Step()
        later = drv.get_particles()
        np.testing.assert_array_equal(later["X"][0], got["X"][0])
        drv.close()


def test_bad_inputs_are_reported(cuda_device):
    scene = S.small_3d(with_walls=False)
    s = scene.copy()
    s.X[5] = [2.0, 0.5, 0.5]               # outside the ghosted grid
    drv = D().MPM_DRIVER(s)
    with pytest.raises(D().MPMError) as e:
        drv.set_scene_particles(s)
    assert e.value.code == 4
    drv.close()
    s = scene.copy()
    s.F[3] = np.nan
    drv = D().MPM_DRIVER(s)
    drv.set_scene_particles(s)
    drv.Advance_One_Time_Step()
    with pytest.raises(D().MPMError) as e:
        drv.synchronize()
    assert e.value.code == 3
    drv.close()


def test_grid_mass_conservation_full_size(cuda_device):
    """Size-independent property at full size: grid mass after P2G equals particle mass."""
    scene = S.spheres_3d()
    drv = D().MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    drv.Advance_One_Time_Step()
    g = drv.get_grid()
    total = float(np.sum(g["grid_m"]))
    assert abs(total - scene.mass.sum()) / scene.mass.sum() < 1e-5
    drv.close()


def test_native_layout_round_trip(cuda_device):
    """set_particles_native / get_particles_native (C-ABI layout, no host copies)
    give the same state as the numpy-matrix calls."""
    scene = S.small_3d(nsteps=3)
    n = scene.n
    col = lambda M: np.ascontiguousarray(np.swapaxes(M, 1, 2).reshape(n, 9), np.float32)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    a = D().MPM_DRIVER(scene)
    a.set_particles_native(f32(scene.X), f32(scene.V), col(scene.F), col(scene.B), f32(scene.mass),
                           f32(scene.volume), f32(scene.mu), f32(scene.lam))
    b = D().MPM_DRIVER(scene)
    b.set_scene_particles(scene, dtype=np.float32)
    for drv in (a, b):
        drv.advance(scene.nsteps)
    X, V = np.empty((n, 3), np.float32), np.empty((n, 3), np.float32)
    Fc, Bc, valid = np.empty((n, 9), np.float32), np.empty((n, 9), np.float32), np.empty(n, np.uint8)
    a.get_particles_native(X, V, Fc, Bc, valid)
    ref = b.get_particles(dtype=np.float32)
    # the two runs differ only in the order of float atomics
    vmax = float(np.abs(ref["V"]).max())
    assert rel(X, ref["X"], 1.0) < 1e-6
    assert rel(V, ref["V"], vmax) < 1e-4
    assert rel(Fc.reshape(n, 3, 3).transpose(0, 2, 1), ref["F"], 1.0) < 1e-5
    assert rel(Bc.reshape(n, 3, 3).transpose(0, 2, 1), ref["B"], vmax / scene.dx) < 1e-4
    np.testing.assert_array_equal(valid.astype(bool), ref["valid"])
    with pytest.raises(ValueError):
        a.get_particles_native(X, V, Fc.reshape(n, 3, 3), Bc, valid)
    a.close()
    b.close()


def test_reupload_keeps_buffers_and_matches_fresh_handle(cuda_device):
    """Re-uploading the same number of particles reuses the buffers and the
    captured substeps; a P2G left without its grid update is discarded."""
    scene = S.small_3d(nsteps=5)
    fresh = D().MPM_DRIVER(scene)
    fresh.set_scene_particles(scene)
    fresh.advance(5)
    ref = fresh.get_particles()
    fresh.close()
    drv = D().MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    drv.advance(5)
    drv.set_scene_particles(scene)          # same count: buffers and graphs kept
    drv.advance(5)
    got = drv.get_particles()
    assert rel(got["X"], ref["X"], 1.0) < 1e-6
    drv.Particle_To_Grid()                   # P2G with no grid update ...
    drv.set_scene_particles(scene)          # ... then a re-upload
    drv.advance(5)
    got = drv.get_particles()
    vmax = float(np.abs(ref["V"]).max())
    assert rel(got["X"], ref["X"], 1.0) < 1e-6
    assert rel(got["V"], ref["V"], vmax) < 1e-4
    drv.close()
