"""GPU tests of the batched path (mpm_batch_create): many independent scenes,
different grid sizes and models, advanced together.  Each scene of the batch
is checked against the FP64 oracle (oracle/mpm_oracle.c, itself pinned to the
reference's dumps) run on that scene alone, at the FP32 path's tolerances; the
full-size batch scenes are pinned to the reference's own build in
test_gpu_baseline_parity.py."""
import numpy as np
import pytest

import oracle
from physbam_b200 import scenes as S

pytestmark = pytest.mark.gpu


def small_batch(count=6, seed=77):
    scenes = S.batch_scenes(seed=seed, count=count)
    out = []
    for s in scenes:   # keep the test quick: subsample big scenes
        if s.n > 20000:
            s = s.subset(slice(0, 20000))
        out.append(s)
    out[1].objects = S.walls(3, out[1].counts, out[1].domain_min, out[1].domain_max, 1 << 3, S.STICK, 0.0, 0.3)
    return out


def test_batch_matches_individual_scenes(cuda_device):
    from physbam_b200 import driver as D
    scenes = small_batch()
    nsteps = 12
    batch = D.MPM_BATCH(scenes)
    batch.set_scene_particles()
    batch.advance(nsteps)
    got = batch.split(batch.get_particles())
    batch.close()
    for s, g in zip(scenes, got):
        st = oracle.State(s)
        oracle.run(st, nsteps)
        np.testing.assert_array_equal(g["valid"], st.valid.astype(bool))
        ex = np.max(np.abs(g["X"] - st.X))
        ef = np.max(np.abs(g["F"] - st.F_rowmajor()))
        ev = np.max(np.abs(g["V"] - st.V)) / max(np.max(np.abs(st.V)), 1e-12)
        assert ex < 2e-6 and ef < 1e-4 and ev < 2e-3, (s.name, s.counts, ex, ef, ev)


@pytest.mark.parametrize("cold", [False, True])
def test_autotune_keeps_state_and_results(cuda_device, cold):
    from physbam_b200 import driver as D
    scenes = small_batch(count=4, seed=3)
    b1 = D.MPM_BATCH(scenes)
    b1.set_scene_particles()
    before = b1.get_particles()
    report = b1.autotune(substeps=2, cold_l2=cold)
    assert "chosen" in report and (("cold L2" in report) == cold)
    after = b1.get_particles()
    np.testing.assert_array_equal(before["X"], after["X"])
    b1.advance(6)
    x1 = b1.get_particles()["X"]
    b1.close()
    b2 = D.MPM_BATCH(scenes)
    b2.set_scene_particles()
    b2.advance(6)
    x2 = b2.get_particles()["X"]
    b2.close()
    assert np.max(np.abs(x1 - x2)) < 1e-6
