"""CPU tests of PhysBAM's on-disk formats (physbam_b200.io).

* The reference's own viewer output (tests/golden/viewer_small2d, written by
  its Write_Output_Files) reads back to the reference's state, and writing it
  again gives the same bytes.
* Where the reference is built here: it restarts (Read_Output_Files) from a
  frame we write and continues exactly as its own uninterrupted run, for
  elastic, snow and sand scenes.
"""
import gzip
import os
import shutil
import tempfile

import numpy as np
import pytest

import oracle
from make_golden import load
from physbam_b200 import io
from physbam_b200 import scenes as S

HERE = os.path.dirname(os.path.abspath(__file__))
VIEWER = os.path.join(HERE, "golden", "viewer_small2d")


def test_reads_the_references_frame():
    scene, dumps = load("small2d_corotated")      # same seeded scene; frame 2 = after two substeps
    f = io.read_frame(VIEWER, 2)
    assert f["time"] == pytest.approx(2e-4, abs=1e-18)
    ref = dumps[1]
    for k in ("X", "V", "F", "B"):
        np.testing.assert_array_equal(f[k], ref[k])
    np.testing.assert_array_equal(f["valid"], ref["valid"])
    np.testing.assert_array_equal(f["mass"], scene.mass)
    counts, lo, hi, mac = io.read_grid(VIEWER, 2)
    assert counts == list(scene.counts) and lo == list(scene.domain_min) and hi == list(scene.domain_max) and mac == .5


def test_rewrite_is_byte_identical():
    f = io.read_particles(os.path.join(VIEWER, "2", "deformable_object_particles.gz"))
    tmp = tempfile.mkdtemp()
    try:
        p = os.path.join(tmp, "p.gz")
        io.write_particles(p, f)
        with gzip.open(p) as a, gzip.open(os.path.join(VIEWER, "2", "deformable_object_particles.gz")) as b:
            assert a.read() == b.read()
        io.write_frame(tmp, 2, 2e-4, f, counts=[16, 16], domain_min=[0, 0], domain_max=[1, 1])
        for rel in ("2/restart_data.gz", "common/grid.gz"):
            with gzip.open(os.path.join(tmp, rel)) as a, gzip.open(os.path.join(VIEWER, rel)) as b:
                assert a.read() == b.read(), rel
        with open(os.path.join(tmp, "common", "last_frame")) as a, open(os.path.join(VIEWER, "common", "last_frame")) as b:
            assert a.read() == b.read()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


@pytest.mark.parametrize("use_doubles", [True, False])
def test_round_trip(use_doubles):
    rng = np.random.default_rng(0)
    n = 37
    arrays = {"X": rng.random((n, 3)), "F": rng.random((n, 3, 3)), "mass": rng.random(n),
              "valid": rng.random(n) > 0.3, "Fp": rng.random((n, 3, 3))}
    tmp = tempfile.mkdtemp()
    try:
        p = os.path.join(tmp, "p.gz")
        io.write_particles(p, arrays, use_doubles)
        back = io.read_particles(p)
        assert set(back) == set(arrays)
        for k, v in arrays.items():
            if v.dtype == bool:
                np.testing.assert_array_equal(back[k], v)
            else:
                assert back[k].dtype == (np.float64 if use_doubles else np.float32)
                np.testing.assert_array_equal(back[k], v.astype(back[k].dtype))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def particle_arrays(scene, st, plastic=None):
    out = {"X": st["X"], "V": st["V"], "F": st["F"], "B": st["B"], "mass": scene.mass, "volume": scene.volume,
           "mu": st.get("mu", scene.mu), "lambda": st.get("lam", scene.lam), "valid": st["valid"]}
    if plastic is not None:
        out.update(plastic)
    return out


@pytest.mark.skipif(not oracle.ref_available(), reason="reference runner not built (no reference sources)")
@pytest.mark.parametrize("name", ["small3d_corotated", "smallsnow3d_corotated", "smallsand2d_hencky"])
def test_reference_restarts_from_our_frame(name):
    """Our frame of the state after the first substep (the reference's own dump, with
    its plastic arrays) -> the reference restarts from it -> after 19 more substeps it
    equals its uninterrupted run, bit for bit."""
    scene, dumps = load(name)
    st = dumps[0]
    plastic = None
    pl = scene.plasticity
    if pl is not None:
        plastic = {"Fp": st["Fp"]}
        if pl.kind == S.PLASTICITY_CLAMP:
            plastic.update(mu0=scene.mu, lambda0=scene.lam)
        else:
            plastic.update(plastic_deformation=st["pdef"], dp_rho_f=st["rho_F"], dp_cohesion=st["cohesion"],
                           vcp=st["vc"])
    tmp = tempfile.mkdtemp()
    try:
        io.write_frame(tmp, 1, scene.dt, particle_arrays(scene, st, plastic), counts=scene.counts,
                       domain_min=scene.domain_min, domain_max=scene.domain_max)
        s = scene.copy()
        s.nsteps = 19
        r = oracle.run_reference(s, [18], restart=(tmp, 1))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    ref = dumps[19]
    for k in ("X", "V", "F", "B") + S.plastic_keys(pl):
        np.testing.assert_array_equal(r[18][k], ref[k], err_msg=k)
