"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own MPM_DRIVER (compiled from its sources by
``oracle/ref.mk``, driven by ``oracle/ref_scene.cpp``) in FP64 on small seeded
scenes and freezes inputs plus dumps into ``<name>.npz``.  Needs the reference
tree, so it runs only where that is present; the fixtures are committed so the
tests never need it.

    python tests/golden/make_golden.py [case ...]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from physbam_b200 import scenes as S  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (scene factory, dumps, steps whose grids are kept)
    "small2d_corotated": (lambda: S.small_2d(), [0, 1, 19], [0, 19]),
    "small2d_neohookean": (lambda: S.small_2d(model=S.NEO_HOOKEAN, seed=5), [0, 19], [0]),
    "small3d_corotated": (lambda: S.small_3d(), [0, 1, 19], [0, 19]),
    "small3d_neohookean_friction": (lambda: S.small_3d(model=S.NEO_HOOKEAN, seed=9, friction=0.4), [0, 19], [0]),
    # the 2D block case: 64^2, block 0.25^2 at (0.5,0.6), 4 ppc, corotated, sticky ground, 100 substeps
    "block2d_cfg": (lambda: S.block_2d(), [0, 9, 99], [0, 99]),
    # snow: MPM_PLASTICITY_CLAMP after every G2P (Fp, hardened mu and lambda dumped too)
    "smallsnow3d_corotated": (lambda: S.small_snow_3d(), [0, 19], [0, 19]),
    "smallsnow2d_corotated": (lambda: S.small_snow_2d(), [0, 19], [19]),
    "small3d_hencky": (lambda: S.small_3d(model=S.HENCKY, seed=13, E=(1e5, 3e5)), [0, 19], [0]),
    # backward Euler (the reference's default solve), Newton tolerances as MPM_EXAMPLE's defaults
    "small3d_implicit": (lambda: S.small_3d_implicit(), [0, 1, 9], [0, 9]),
    "small2d_implicit": (lambda: S.small_2d_implicit(), [0, 9], [0, 9]),
    # spherical collision objects (SPHERE): explicit (3D separate, 2D stick) and implicit
    "small3d_sphere": (lambda: S.small_3d_sphere(), [0, 1, 19], [0, 19]),
    "small2d_sphere": (lambda: S.small_2d_sphere(), [0, 19], [19]),
    "small3d_sphere_implicit": (lambda: S.small_3d_sphere(implicit=True), [0, 7], [0, 7]),
    # Simulate_To_Frame with Compute_Dt and Reduce_Dt (steps are frames; substep counts kept)
    "small3d_adaptive": (lambda: S.small_3d_adaptive(), [0, 2], [2]),
    "small2d_adaptive": (lambda: S.small_2d_adaptive(), [0, 2], [2]),
    # reflection boundary conditions on the domain faces (no wall objects)
    "small3d_reflect": (lambda: S.small_3d_reflect(), [0, 1, 19], [0, 19]),
    "small2d_reflect": (lambda: S.small_2d_reflect(), [0, 19], [0, 19]),
    # sand: ST_VENANT_KIRCHHOFF_HENCKY_STRAIN + MPM_DRUCKER_PRAGER (Fp, plastic_def, rho_F, sigma_Y, vc dumped)
    "smallsand3d_hencky": (lambda: S.small_sand_3d(), [0, 1, 19], [0, 19]),
    "smallsand2d_hencky": (lambda: S.small_sand_2d(), [0, 19], [19]),
    # penalty collision objects (IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES): explicit and implicit
    "small3d_penalty": (lambda: S.small_3d_penalty(), [0, 1, 19], [0, 19]),
    "small2d_penalty": (lambda: S.small_2d_penalty(), [0, 19], [0, 19]),
    "small3d_penalty_implicit": (lambda: S.small_3d_penalty(implicit=True), [0, 7], [0, 7]),
    # moving collision objects (func_frame / func_twist): explicit 3D/2D and implicit 3D
    "small3d_moving": (lambda: S.small_3d_moving(), [0, 1, 19], [0, 19]),
    "small2d_moving": (lambda: S.small_2d_moving(), [0, 19], [0, 19]),
    "small3d_moving_implicit": (lambda: S.small_3d_moving(implicit=True), [0, 7], [0, 7]),
    # two materials: one MPM_FINITE_ELEMENTS force per model over its particles
    "small3d_mixed": (lambda: S.small_3d_mixed(), [0, 19], [0, 19]),
    "small3d_mixed_implicit": (lambda: S.small_3d_mixed(implicit=True), [0, 7], [0, 7]),
    # sand beside an elastic body: the plasticity over the sand's particles alone
    "smallsandwater3d_mixed": (lambda: S.small_sand_water_3d(), [0, 1, 19], [0, 19]),
    # a force the library does not model (a constant vector at every node with mass), which
    # the GPU path receives from the caller through mpm_add_grid_forces
    "small3d_node_force": (lambda: S.small_3d_node_force(), [0, 1, 19], [0, 19]),
}


def main(names=None):
    oracle.build()
    if not oracle.ref_available():
        oracle.build_ref()
    for name, (make, dumps, grid_steps) in CASES.items():
        if names and name not in names:
            continue
        scene = make()
        ref = oracle.run_reference(scene, dumps, threads=1)
        frames = None
        if scene.dt_control is not None:
            ref, frames = ref
        arrays = dict(
            dim=scene.dim, counts=np.array(scene.counts), dmin=np.array(scene.domain_min),
            dmax=np.array(scene.domain_max), model=scene.model, gravity=np.array(scene.gravity),
            dt=scene.dt, nsteps=scene.nsteps,
            obj_kind=np.array([o.kind for o in scene.objects], np.int32),
            obj_type=np.array([o.type for o in scene.objects], np.int32),
            obj_friction=np.array([o.friction for o in scene.objects]),
            obj_a=np.array([o.a for o in scene.objects]).reshape(-1, scene.dim),
            obj_b=np.array([o.b for o in scene.objects]).reshape(-1, scene.dim),
            X=scene.X, V=scene.V, F=scene.F, B=scene.B, mass=scene.mass, volume=scene.volume,
            mu=scene.mu, lam=scene.lam, dumps=np.array(dumps))
        if any(o.motion is not None for o in scene.objects):   # center, linear, angular (3 each, zero padded)
            pad = lambda v: list(v) + [0.0] * (3 - len(v))
            arrays["obj_motion"] = np.array([pad(o.motion.center) + pad(o.motion.linear) + pad(o.motion.angular)
                                             if o.motion is not None else [np.nan] * 9 for o in scene.objects])
        if scene.models is not None:
            arrays["models"] = np.asarray(scene.models, np.uint8)
        if scene.plastic_mask is not None:
            arrays["plastic_mask"] = np.asarray(scene.plastic_mask, np.uint8)
        pl = scene.plasticity
        if pl is not None:
            arrays["plasticity"] = np.array(S.plastic_params(pl), np.float64)
        rf = scene.reflection
        if rf is not None:
            arrays["reflection"] = np.array(list(rf.side_type) + [rf.friction, float(rf.full)], np.float64)
        dc = scene.dt_control
        if dc is not None:
            arrays["dt_control"] = np.array([dc.frame_dt, dc.cfl, dc.min_dt, dc.max_dt, float(dc.strong_cfl), dc.cfl_F,
                                             float(dc.sound_cfl), dc.cfl_sound])
            arrays["frame_substeps"] = np.array(frames["frame_substeps"], np.int32)
        pn = scene.penalty
        if pn is not None:
            arrays["penalty"] = np.array([pn.stiffness, pn.separation], np.float64)
            arrays["pen_kind"] = np.array([o.kind for o in pn.objects], np.int32)
            arrays["pen_type"] = np.array([o.type for o in pn.objects], np.int32)
            arrays["pen_friction"] = np.array([o.friction for o in pn.objects])
            arrays["pen_a"] = np.array([o.a for o in pn.objects]).reshape(-1, scene.dim)
            arrays["pen_b"] = np.array([o.b for o in pn.objects]).reshape(-1, scene.dim)
        if scene.node_force is not None:
            arrays["node_force"] = np.array(scene.node_force, np.float64)
        im = scene.implicit
        if im is not None:
            arrays["implicit"] = np.array([im.newton_tolerance, im.newton_iterations, im.solver_tolerance,
                                           im.solver_iterations], np.float64)
        for step in dumps:
            r = ref[step]
            for k in ("X", "V", "F", "B", "valid") + S.plastic_keys(pl):
                arrays["s%d_%s" % (step, k)] = r[k]
            if step in grid_steps:
                for k in ("grid_m", "grid_v0", "grid_v", "grid_vf"):
                    arrays["s%d_%s" % (step, k)] = r[k]
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
        print(name, scene.n, "particles", os.path.getsize(os.path.join(OUT, name + ".npz")), "bytes")


def load(name):
    """Load a fixture back into a Scene plus its reference dumps {step: {key: array}}."""
    z = np.load(os.path.join(OUT, name + ".npz"))
    dim = int(z["dim"])
    objs = [S.CollisionObject(int(k), int(t), float(f), list(a), list(b))
            for k, t, f, a, b in zip(z["obj_kind"], z["obj_type"], z["obj_friction"], z["obj_a"], z["obj_b"])]
    scene = S.Scene(name, dim, [int(c) for c in z["counts"]], list(z["dmin"]), list(z["dmax"]), int(z["model"]),
                    list(z["gravity"]), float(z["dt"]), int(z["nsteps"]), objs,
                    z["X"].copy(), z["V"].copy(), z["F"].copy(), z["B"].copy(), z["mass"].copy(),
                    z["volume"].copy(), z["mu"].copy(), z["lam"].copy())
    if "obj_motion" in z:
        for o, m in zip(objs, z["obj_motion"]):
            if not np.isnan(m[0]):
                o.motion = S.Motion(list(m[0:dim]), list(m[3:3 + dim]), list(m[6:9] if dim == 3 else m[6:7]))
    if "models" in z:
        scene.models = z["models"].copy()
    if "plastic_mask" in z:
        scene.plastic_mask = z["plastic_mask"].copy()
    if "plasticity" in z:
        scene.plasticity = S.plastic_from_params(z["plasticity"])
    if "reflection" in z:
        r = z["reflection"]
        scene.reflection = S.Reflection(tuple(int(x) for x in r[:-2]), float(r[-2]), bool(r[-1]))
    if "dt_control" in z:
        c = z["dt_control"]
        scene.dt_control = S.DtControl(float(c[0]), float(c[1]), float(c[2]), float(c[3]), bool(c[4]), float(c[5]),
                                       bool(c[6]), float(c[7]))
        dumps_meta = {"frame_substeps": [int(x) for x in z["frame_substeps"]]}
        scene.frame_substeps = dumps_meta["frame_substeps"]
    if "penalty" in z:
        pobjs = [S.CollisionObject(int(k), int(t), float(f), list(a), list(b))
                 for k, t, f, a, b in zip(z["pen_kind"], z["pen_type"], z["pen_friction"], z["pen_a"], z["pen_b"])]
        scene.penalty = S.Penalty(pobjs, float(z["penalty"][0]), float(z["penalty"][1]))
    if "node_force" in z:
        scene.node_force = [float(x) for x in z["node_force"]]
    if "implicit" in z:
        im = z["implicit"]
        scene.implicit = S.Implicit(float(im[0]), int(im[1]), float(im[2]), int(im[3]))
    dumps = {}
    for step in z["dumps"]:
        step = int(step)
        rec = {}
        for k in ("X", "V", "F", "B", "valid", "grid_m", "grid_v0", "grid_v", "grid_vf") + S.plastic_keys(scene.plasticity):
            key = "s%d_%s" % (step, k)
            if key in z:
                rec[k] = z[key]
        dumps[step] = rec
    return scene, dumps


if __name__ == "__main__":
    main(sys.argv[1:])
