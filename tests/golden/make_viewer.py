"""Keep a few files of the reference's own viewer output for the format tests.

Runs the reference's MPM_DRIVER (oracle/ref.mk, oracle/ref_scene.cpp) on the
small 2D scene for two frames of one 1e-4 substep each, with its own
Write_Output_Files, and keeps common/grid.gz, common/last_frame and frame 2's
deformable_object_particles.gz and restart_data.gz in viewer_small2d/.

    python tests/golden/make_viewer.py
"""
import os
import shutil
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from physbam_b200 import scenes as S  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "viewer_small2d")


def main():
    if not oracle.ref_available():
        oracle.build_ref()
    s = S.small_2d(nsteps=2)
    s.dt_control = S.DtControl(frame_dt=1e-4, cfl=0.5, min_dt=1e-4, max_dt=1e-4)
    tmp = tempfile.mkdtemp(prefix="viewer_")
    try:
        oracle.run_reference(s, [], output=tmp)
        for rel in ("common/grid.gz", "common/last_frame", "2/deformable_object_particles.gz", "2/restart_data.gz"):
            dst = os.path.join(OUT, rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            shutil.copyfile(os.path.join(tmp, rel), dst)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
