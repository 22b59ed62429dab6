"""The reference-side binding, compiled and run on the GPU.

include/mpm_physbam.hpp (B200_SUBSTEP<TV>, the adapter a PhysBAM maintainer
adds beside MPM_DRIVER, Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.h:41-78)
is compiled against the reference's own headers and library by oracle/ref.mk
into oracle/_ref/ref_b200.  That program sets a scene up as the reference's
MPM_EXAMPLE, hands its MPM_PARTICLES arrays to the C ABI, runs the substeps on
the GPU and downloads the particles back into MPM_PARTICLES.

* The two-sphere scene at full size (128^3, 242,742 particles, 200 substeps,
  one mpm_advance): the particles it gets back match the reference's own FP64
  driver within the FP32 path's bounds, and the Python-side run of the same
  kernels through the same C ABI.
* A small scene with one mpm_substep per substep (double arrays in and out)
  against the FP64 C oracle.
"""
import numpy as np
import pytest

import oracle
from oracle import parity
from physbam_b200 import scenes as S

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.b200_binding_available(), reason="oracle/_ref/ref_b200 is not built")]


def test_binding_full_size_spheres(cuda_device):
    scene = S.spheres_3d()
    got, report = oracle.run_b200_binding(scene, use_float=True)
    assert report["particles"] == scene.n and report["substeps"] == scene.nsteps
    ref = parity.reference_final(scene)
    e = parity.errors(got, ref)
    assert "valid_mismatch" not in e
    assert e["X"]["rel_l2"] <= 1e-4 and e["V"]["rel_l2"] <= 1e-4 and e["F"]["rel_l2"] <= 1e-4, e
    same = parity.fast_final(scene)
    e2 = parity.errors(got, same)
    assert e2["X"]["max_abs"] <= 1e-5 and e2["F"]["max_abs"] <= 1e-4, e2
    print("binding: %.3f s for %d substeps; vs reference FP64: %s" % (report["gpu_seconds"], scene.nsteps,
                                                                    parity.compact({"x": e})["x"]))


def test_binding_per_substep_small(cuda_device):
    scene = S.small_3d(nsteps=10)
    got, _ = oracle.run_b200_binding(scene, use_float=False, per_substep=True)
    st = oracle.State(scene)
    oracle.run(st, scene.nsteps)
    np.testing.assert_array_equal(got["valid"], st.valid.astype(bool))
    assert np.max(np.abs(got["X"] - st.X)) < 2e-6
    assert np.max(np.abs(got["F"] - st.F_rowmajor())) < 1e-4
