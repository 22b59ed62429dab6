"""GPU tests of the device-side failure paths, made to happen without faulting
the GPU: every wait that runs out is bounded and reports a status, after which
the same process keeps sorting and simulating correctly.

* The radix sort's decoupled look-back waits on a predecessor tile that never
  publishes (its ticket is taken before the pass starts): the bounded wait
  gives up and the call returns MPM_ERR_TIMEOUT.
* The look-back status words of the radix sort and of the block scan carry a
  30-bit epoch: sorts across its wrap stay bit-exact against a CPU stable sort.
* The FP64 SVD (the reference's unbounded implicit-shift QR,
  Core/Matrices/MATRIX_3X3.cpp:202-236) gets a one-sweep bound: the substep
  reports MPM_ERR_NOT_CONVERGED.
The reference's counterparts are assertion failures that throw
(Core/Log/DEBUG_UTILITIES.cpp:95-103); here they are status codes.
"""
import numpy as np
import pytest

from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu

TIMEOUT, NOT_CONVERGED = 5, 8


def D():
    from physbam_b200 import driver
    return driver


def test_sort_lookback_timeout_is_reported(cuda_device):
    L = D().load_library()
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 16, 10_000, dtype=np.uint32)
    rc = L.mpm_debug_sort_stall(keys.ctypes.data, keys.size, 16, 1024)
    assert rc == TIMEOUT
    # the context is still usable: a normal sort right after is bit-exact
    sk, perm = D().radix_sort_u32(keys, 16)
    ref = np.argsort(keys, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(sk, keys[ref])


def test_sort_across_epoch_wrap(cuda_device):
    scene = S.small_3d(nsteps=8)
    drv = D().MPM_DRIVER(scene)
    drv.set_scene_particles(scene)
    drv._check(drv.L.mpm_debug_set_sort_epoch(drv.h, (1 << 30) - 3), "mpm_debug_set_sort_epoch")
    for it in range(6):
        if it % 2 == 0:
            drv.set_scene_particles(scene)     # a full sort of freshly uploaded keys next
        drv.Particle_To_Grid()
        keys, sk, perm = drv.sort_state()
        ref = np.argsort(keys >> 6, kind="stable").astype(np.uint32)
        np.testing.assert_array_equal(perm, ref, err_msg="sort %d" % it)
        np.testing.assert_array_equal(sk, keys[ref])
        drv.Apply_Forces()
        drv.Grid_To_Particle()
    drv.synchronize()
    drv.close()


@pytest.mark.parametrize("path", ["plain", "fast"])
def test_svd_non_convergence_is_reported(cuda_device, path):
    L = D().load_library()
    scene = S.small_3d(nsteps=2)
    if path == "fast":         # inverted F takes the FP64 SVD route on the fast path
        F = scene.F.copy()
        F[::3, :, 0] *= -1.0
        scene.F = F
    prec, p = (D().FP64, D().PATH_PLAIN) if path == "plain" else (D().FP32, D().PATH_FAST)
    assert L.mpm_debug_set_svd_iterations(1) == 0
    try:
        drv = D().MPM_DRIVER(scene, precision=prec, path=p)
        drv.set_scene_particles(scene)
        drv.Advance_One_Time_Step()
        with pytest.raises(D().MPMError) as e:
            drv.synchronize()
        assert e.value.code == NOT_CONVERGED
        drv.close()
    finally:
        assert L.mpm_debug_set_svd_iterations(64) == 0
    drv = D().MPM_DRIVER(scene, precision=prec, path=p)
    drv.set_scene_particles(scene)
    drv.advance(2)
    drv.synchronize()
    assert drv.count_valid() == scene.n
    drv.close()
