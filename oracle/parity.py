"""Per-quantity error of the FP32 fast path against the reference's own FP64
build on the full-size 3D configurations -- TEST INFRASTRUCTURE ONLY.

Used by ``tests/test_gpu_baseline_parity.py`` and by the parity leg of
``bench.py`` (outside its timed region) as the checker; the product never
imports it.  The reference side is ``oracle/_ref/ref_scene`` (the reference's
``MPM_DRIVER<VECTOR<double,3>>`` compiled from its own sources by
``oracle/ref.mk``) run on the same seeded scene file; it dumps the state after
the last substep (``Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.cpp:141-157``:
``Advance_One_Time_Step``; X, V, F, B from ``Grid_To_Particle``, l.450-515; the
grids of that substep from ``Particle_To_Grid`` and ``Apply_Forces``).

Quantities and their error measures (after the last substep):
  X, V, F           relative L2 over all particles (||a - r|| / ||r||) and max |a - r|
  grid_m            mass of every node of the ghosted grid, same two measures
  grid_mv           node momentum after the grid update, mass x velocity (the
                    velocity G2P reads: ``MPM_EXAMPLE::velocity`` after Apply_Forces)
"""
from __future__ import annotations

import os

import numpy as np

from physbam_b200 import scenes as S

# The full-size configurations: name -> (scene builder, description).  The
# batch scenes are checked per scene, each run inside one 256-scene batch
# handle on the device and alone on the reference.
BATCH_CHECKED = (0, 1, 2, 3, 4, 5, 6, 7, 128, 200, 255)


def _cfg2():
    return S.spheres_3d()


def _cfg3_64():
    return S.dam_3d(G=64)


def _cfg4():
    return S.cube_3d()


SINGLE = {
    "spheres3d-128": (_cfg2, "two spheres, 128^3, neo-Hookean, 200 substeps"),
    "dam3d-64": (_cfg3_64, "dam break, 64^3 copy of the 256^3 scene, corotated, 100 substeps"),
    "cube3d-64": (_cfg4, "differentiable cube forward, 64^3, corotated, 64 substeps"),
}


def measures(got: np.ndarray, ref: np.ndarray) -> dict:
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    nr = float(np.linalg.norm(ref))
    diff = got - ref
    return {"rel_l2": float(np.linalg.norm(diff)) / (nr if nr > 0 else 1.0),
            "max_abs": float(np.max(np.abs(diff))) if diff.size else 0.0}


def errors(got: dict, ref: dict) -> dict:
    """Error table of one configuration; `got` and `ref` carry X, V, F, valid, grid_m, grid_v."""
    out = {}
    if not np.array_equal(np.asarray(got["valid"], bool), np.asarray(ref["valid"], bool)):
        out["valid_mismatch"] = int(np.sum(np.asarray(got["valid"], bool) != np.asarray(ref["valid"], bool)))
    ok = np.asarray(ref["valid"], bool)
    for k in ("X", "V", "F"):
        out[k] = measures(np.asarray(got[k])[ok], np.asarray(ref[k])[ok])
    if "grid_m" in got and "grid_m" in ref:
        out["grid_m"] = measures(got["grid_m"], ref["grid_m"])
        out["grid_mv"] = measures(np.asarray(got["grid_m"])[..., None] * np.asarray(got["grid_v"]),
                                  np.asarray(ref["grid_m"])[..., None] * np.asarray(ref["grid_v"]))
    return out


def reference_final(scene, threads: int = 0) -> dict:
    """The reference's FP64 state and grids after the scene's last substep."""
    import oracle
    if not oracle.ref_available():
        raise RuntimeError("the reference build (oracle/_ref/ref_scene) is absent")
    threads = threads or (os.cpu_count() or 1)
    dumps = oracle.run_reference(scene, [scene.nsteps - 1], threads=threads)
    rec = dumps[scene.nsteps - 1]
    return {k: rec[k] for k in ("X", "V", "F", "B", "valid", "grid_m", "grid_v", "grid_vf")}


def fast_final(scene) -> dict:
    """The FP32 fast path's state and grids after the scene's substeps (one handle, graph replay)."""
    from physbam_b200 import driver as D
    drv = D.MPM_DRIVER(scene, precision=D.FP32, path=D.PATH_FAST)
    try:
        drv.set_scene_particles(scene)
        drv.advance(scene.nsteps)
        out = drv.get_particles()
        g = drv.get_grid()
        out["grid_m"], out["grid_v"] = g["grid_m"], g["grid_v"]
        return out
    finally:
        drv.close()


def batch_final(scenes, checked) -> list:
    """All scenes advanced together in one batch handle; the state and grids of the `checked` ones."""
    from physbam_b200 import driver as D
    drv = D.MPM_BATCH(scenes)
    try:
        drv.set_scene_particles()
        drv.advance(scenes[0].nsteps)
        parts = drv.split(drv.get_particles())
        out = []
        for i in checked:
            rec = parts[i]
            g = drv.get_scene_grid(i)
            rec["grid_m"], rec["grid_v"] = g["grid_m"], g["grid_v"]
            out.append(rec)
        return out
    finally:
        drv.close()


def single_table(name: str, threads: int = 0) -> dict:
    scene = SINGLE[name][0]()
    ref = reference_final(scene, threads)
    got = fast_final(scene)
    e = errors(got, ref)
    e["particles"] = scene.n
    e["substeps"] = scene.nsteps
    return e


def batch_table(threads: int = 0, checked=BATCH_CHECKED) -> dict:
    scenes = S.batch_scenes(seed=1234, count=256)
    got = batch_final(scenes, checked)
    out = {}
    for i, g in zip(checked, got):
        e = errors(g, reference_final(scenes[i], threads))
        e["particles"] = scenes[i].n
        e["grid"] = scenes[i].counts[0]
        e["substeps"] = scenes[i].nsteps
        out["batch256-scene%d" % i] = e
    return out


def compact(table: dict) -> dict:
    """{config: {quantity: rel_l2}} for a one-line report."""
    out = {}
    for cfg, e in table.items():
        out[cfg] = {k: float("%.3g" % v["rel_l2"]) for k, v in e.items() if isinstance(v, dict)}
        if "valid_mismatch" in e:
            out[cfg]["valid_mismatch"] = e["valid_mismatch"]
    return out
