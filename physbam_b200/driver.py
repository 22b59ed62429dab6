"""Host-side mirror of the reference's explicit MPM driver over the C ABI.

`MPM_DRIVER` here plays the part of PhysBAM's ``MPM_DRIVER<TV>``
(``Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.h:22-80``) for the explicit
path: the same step names, one handle per simulation, state kept on the GPU
between calls.  Every call goes through ``libphysbam_mpm.so``; there is no
CPU fallback, and importing this module on a machine without the library
raises.  Errors come back as `MPMError`, the way PHYSBAM_FATAL_ERROR surfaces
as ``std::runtime_error`` in the reference (``Core/Log/DEBUG_UTILITIES.cpp:95-103``).
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import scenes as S

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphysbam_mpm.so")

MPM_OK = 0
FP32, FP64 = 0, 1
P2G_CELLS, P2G_INTERLEAVED, P2G_PAIRS, P2G_PAIRX = 0, 1, 2, 3
PATH_FAST, PATH_PLAIN = 0, 1
MAX_OBJECTS = 8
STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "non-finite value", 4: "particle outside the grid",
          5: "device wait timed out", 6: "out of device memory", 7: "call out of order", 8: "SVD did not converge"}


class MPMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("counts", ctypes.c_int * 3), ("domain_min", ctypes.c_double * 3),
                ("domain_max", ctypes.c_double * 3), ("ghost", ctypes.c_int)]


class ModelDesc(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("precision", ctypes.c_int), ("path", ctypes.c_int),
                ("gravity", ctypes.c_double * 3)]


class CollisionObject(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("type", ctypes.c_int), ("friction", ctypes.c_double),
                ("a", ctypes.c_double * 3), ("b", ctypes.c_double * 3)]


class Totals(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("momentum", ctypes.c_double * 3), ("angular_momentum", ctypes.c_double * 3),
                ("kinetic_energy", ctypes.c_double), ("max_speed", ctypes.c_double),
                ("max_affine_speed", ctypes.c_double), ("count", ctypes.c_int64)]

    def as_dict(self):
        return {"mass": self.mass, "momentum": np.array(self.momentum[:]),
                "angular_momentum": np.array(self.angular_momentum[:]), "kinetic_energy": self.kinetic_energy,
                "max_speed": self.max_speed, "max_affine_speed": self.max_affine_speed, "count": self.count}


class ParticlesView(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dtype", ctypes.c_int), ("on_device", ctypes.c_int),
                ("X", ctypes.c_void_p), ("V", ctypes.c_void_p), ("F", ctypes.c_void_p), ("B", ctypes.c_void_p),
                ("mass", ctypes.c_void_p), ("volume", ctypes.c_void_p), ("mu", ctypes.c_void_p),
                ("lambda_", ctypes.c_void_p), ("valid", ctypes.c_void_p)]


class PlasticityDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("theta_c", ctypes.c_double), ("theta_s", ctypes.c_double),
                ("max_hardening", ctypes.c_double), ("hardening_factor", ctypes.c_double),
                ("dp_a0", ctypes.c_double), ("dp_a1", ctypes.c_double), ("dp_a3", ctypes.c_double),
                ("dp_a4", ctypes.c_double), ("cohesion", ctypes.c_double), ("use_vc", ctypes.c_int)]


class PlasticView(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dtype", ctypes.c_int), ("on_device", ctypes.c_int),
                ("Fp", ctypes.c_void_p), ("mu", ctypes.c_void_p), ("lambda_", ctypes.c_void_p),
                ("mu0", ctypes.c_void_p), ("lambda0", ctypes.c_void_p), ("plastic_def", ctypes.c_void_p),
                ("rho_F", ctypes.c_void_p), ("cohesion", ctypes.c_void_p), ("vc", ctypes.c_void_p)]


class ImplicitDesc(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int), ("newton_tolerance", ctypes.c_double), ("newton_iterations", ctypes.c_int),
                ("solver_tolerance", ctypes.c_double), ("solver_iterations", ctypes.c_int)]


class ImplicitStats(ctypes.Structure):
    _fields_ = [("newton_iterations", ctypes.c_int), ("krylov_iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("residual", ctypes.c_double)]


class DtControlDesc(ctypes.Structure):
    _fields_ = [("cfl", ctypes.c_double), ("min_dt", ctypes.c_double), ("max_dt", ctypes.c_double),
                ("strong_cfl", ctypes.c_int), ("cfl_F", ctypes.c_double), ("sound_cfl", ctypes.c_int),
                ("cfl_sound", ctypes.c_double)]


class ReflectionDesc(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int), ("side_type", ctypes.c_int * 6), ("friction", ctypes.c_double),
                ("full_reflection", ctypes.c_int)]


# plastic-state keys (scenes.plastic_keys and the mu/lam pair) -> PlasticView fields
_PLASTIC_FIELDS = {"Fp": "Fp", "mu": "mu", "lam": "lambda_", "mu0": "mu0", "lam0": "lambda0",
                   "pdef": "plastic_def", "rho_F": "rho_F", "cohesion": "cohesion", "vc": "vc"}


class ObjectState(ctypes.Structure):
    _fields_ = [("translation", ctypes.c_double * 3), ("rotation", ctypes.c_double * 4),
                ("linear", ctypes.c_double * 3), ("angular", ctypes.c_double * 3)]


MOTION_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ObjectState))


EXPORTS = ["mpm_create", "mpm_destroy", "mpm_set_stream", "mpm_set_collision_objects", "mpm_set_particles",
           "mpm_get_particles", "mpm_substep", "mpm_advance", "mpm_particle_to_grid", "mpm_apply_forces",
           "mpm_grid_to_particle", "mpm_synchronize", "mpm_get_grid", "mpm_count_valid", "mpm_set_timing",
           "mpm_get_timing", "mpm_last_error", "mpm_status_string", "mpm_radix_sort_u32", "mpm_debug_sort_state",
           "mpm_diff_forward", "mpm_diff_backward", "mpm_set_diff_tape_budget", "mpm_batch_create", "mpm_autotune", "mpm_particle_totals",
           "mpm_grid_totals", "mpm_compute_dt", "mpm_set_launch_shape", "mpm_get_launch_shape", "mpm_autotune_ex",
           "mpm_set_plasticity", "mpm_get_plastic_state", "mpm_set_plastic_state", "mpm_set_implicit",
           "mpm_get_implicit_stats", "mpm_set_dt_control", "mpm_simulate_frame", "mpm_last_dt",
           "mpm_set_reflection", "mpm_set_penalty_objects", "mpm_set_object_motion", "mpm_set_particle_models",
           "mpm_set_plastic_particles", "mpm_batch_get_grid", "mpm_debug_sort_stall", "mpm_debug_set_sort_epoch",
           "mpm_debug_set_svd_iterations", "mpm_add_grid_forces"]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libphysbam_mpm.so.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libphysbam_mpm.so is not built (run __graft_entry__.build()); "
                           "the MPM path has no CPU fallback")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    L.mpm_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(ModelDesc), ctypes.POINTER(P)]
    L.mpm_destroy.argtypes = [P]
    L.mpm_set_stream.argtypes = [P, P]
    L.mpm_set_collision_objects.argtypes = [P, ctypes.POINTER(CollisionObject), ctypes.c_int]
    L.mpm_set_particles.argtypes = [P, ctypes.POINTER(ParticlesView)]
    L.mpm_get_particles.argtypes = [P, ctypes.POINTER(ParticlesView)]
    for f in ("mpm_substep", "mpm_particle_to_grid", "mpm_apply_forces", "mpm_grid_to_particle"):
        getattr(L, f).argtypes = [P, ctypes.c_double, ctypes.c_double]
    L.mpm_advance.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    L.mpm_synchronize.argtypes = [P]
    L.mpm_get_grid.argtypes = [P, P, P, P, P]
    L.mpm_batch_get_grid.argtypes = [P, ctypes.c_int, P, P, P]
    L.mpm_debug_sort_stall.argtypes = [P, ctypes.c_int64, ctypes.c_int, ctypes.c_uint32]
    L.mpm_debug_set_sort_epoch.argtypes = [P, ctypes.c_uint32]
    L.mpm_debug_set_svd_iterations.argtypes = [ctypes.c_int]
    L.mpm_add_grid_forces.argtypes = [P, ctypes.c_double, P, ctypes.c_int, ctypes.c_int]
    L.mpm_count_valid.argtypes = [P, ctypes.POINTER(ctypes.c_int64)]
    L.mpm_set_timing.argtypes = [P, ctypes.c_int]
    L.mpm_get_timing.argtypes = [P, ctypes.c_char_p, ctypes.c_int, P, P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.mpm_last_error.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
    L.mpm_diff_forward.argtypes = [P, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.mpm_set_diff_tape_budget.argtypes = [P, ctypes.c_int64]
    L.mpm_diff_backward.argtypes = [P, ctypes.POINTER(ParticlesView), ctypes.POINTER(ParticlesView), P, P]
    L.mpm_radix_sort_u32.argtypes = [P, ctypes.c_int64, ctypes.c_int, P, P]
    L.mpm_autotune.argtypes = [P, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.mpm_autotune_ex.argtypes = [P, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
    L.mpm_set_launch_shape.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.mpm_get_launch_shape.argtypes = [P] + [ctypes.POINTER(ctypes.c_int)] * 3
    L.mpm_particle_totals.argtypes = [P, ctypes.POINTER(Totals)]
    L.mpm_grid_totals.argtypes = [P, ctypes.POINTER(Totals)]
    L.mpm_compute_dt.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    L.mpm_debug_sort_state.argtypes = [P, P, P, P]
    L.mpm_set_plasticity.argtypes = [P, ctypes.POINTER(PlasticityDesc)]
    L.mpm_get_plastic_state.argtypes = [P, ctypes.POINTER(PlasticView)]
    L.mpm_set_plastic_state.argtypes = [P, ctypes.POINTER(PlasticView)]
    L.mpm_set_implicit.argtypes = [P, ctypes.POINTER(ImplicitDesc)]
    L.mpm_get_implicit_stats.argtypes = [P, ctypes.POINTER(ImplicitStats)]
    L.mpm_set_dt_control.argtypes = [P, ctypes.POINTER(DtControlDesc)]
    L.mpm_simulate_frame.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_int)]
    L.mpm_last_dt.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
    L.mpm_set_reflection.argtypes = [P, ctypes.POINTER(ReflectionDesc)]
    L.mpm_set_penalty_objects.argtypes = [P, ctypes.POINTER(CollisionObject), ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double]
    L.mpm_set_object_motion.argtypes = [P, ctypes.c_int, MOTION_FN, P]
    L.mpm_set_particle_models.argtypes = [P, P, ctypes.c_int64]
    L.mpm_set_plastic_particles.argtypes = [P, P, ctypes.c_int64]
    L.mpm_status_string.argtypes = [ctypes.c_int]
    L.mpm_status_string.restype = ctypes.c_char_p
    for f in EXPORTS:
        if f != "mpm_status_string":
            getattr(L, f).restype = ctypes.c_int
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class MPM_DRIVER:
    """Explicit MPM substep on one GPU, keyed to a `scenes.Scene` (grid, model, gravity, objects)."""

    def __init__(self, scene: S.Scene, precision: int = FP32, path: int = PATH_FAST):
        self.L = load_library()
        self.scene = scene
        self.dim = scene.dim
        self.precision = precision
        self.path = path
        g = GridDesc()
        g.dim = scene.dim
        for a in range(3):
            g.counts[a] = scene.counts[a] if a < scene.dim else 1
            g.domain_min[a] = scene.domain_min[a] if a < scene.dim else 0.0
            g.domain_max[a] = scene.domain_max[a] if a < scene.dim else 1.0
        g.ghost = S.GHOST
        m = ModelDesc()
        m.model, m.precision, m.path = scene.model, precision, path
        for a in range(scene.dim):
            m.gravity[a] = scene.gravity[a]
        self.h = ctypes.c_void_p()
        self._check(self.L.mpm_create(ctypes.byref(g), ctypes.byref(m), ctypes.byref(self.h)), "mpm_create")
        self.set_collision_objects(scene.objects)
        if scene.plasticity is not None:
            self.set_plasticity(scene.plasticity)
        if scene.implicit is not None:
            self.set_implicit(scene.implicit)
        if scene.dt_control is not None:
            self.set_dt_control(scene.dt_control)
        if scene.reflection is not None:
            self.set_reflection(scene.reflection)
        if scene.penalty is not None:
            self.set_penalty(scene.penalty)
        self.time = 0.0
        self.n = 0

    # -- errors ---------------------------------------------------------------
    def _check(self, rc, what):
        if rc != MPM_OK:
            buf = ctypes.create_string_buffer(512)
            if self.__dict__.get("h"):
                self.L.mpm_last_error(self.h, buf, 512)
            raise MPMError(rc, "%s: %s" % (what, buf.value.decode(errors="replace")))

    def close(self):
        if getattr(self, "h", None):
            self.L.mpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- scene ----------------------------------------------------------------
    def set_collision_objects(self, objects: Sequence[S.CollisionObject]):
        arr = (CollisionObject * max(len(objects), 1))()
        for i, o in enumerate(objects):
            arr[i].kind, arr[i].type, arr[i].friction = o.kind, o.type, o.friction
            for a in range(self.dim):
                arr[i].a[a], arr[i].b[a] = o.a[a], o.b[a]
        self._check(self.L.mpm_set_collision_objects(self.h, arr, len(objects)), "mpm_set_collision_objects")
        self._motion_fns = {}
        for j, o in enumerate(objects):
            if getattr(o, "motion", None) is not None:
                self.set_object_motion(j, o.motion)

    def set_object_motion(self, j: int, motion):
        """Make collision object j move (mpm_set_object_motion).  `motion` is an
        S.Motion or any callable time -> (translation, quaternion (w, x, y, z) -- in 2D
        (cos, sin, 0, 0) --, linear, angular); None makes it static."""
        if motion is None:
            self._motion_fns.pop(j, None)
            self._check(self.L.mpm_set_object_motion(self.h, j, MOTION_FN(), None), "mpm_set_object_motion")
            return
        at = (lambda t: motion.state(self.dim, t)) if isinstance(motion, S.Motion) else motion

        def fn(user, obj, time, state):
            try:
                tr, q, lin, ang = at(time)
                st = state.contents
                for k in range(3):
                    st.translation[k] = tr[k] if k < len(tr) else 0.0
                    st.linear[k] = lin[k] if k < len(lin) else 0.0
                    st.angular[k] = ang[k] if k < len(ang) else 0.0
                for k in range(4):
                    st.rotation[k] = q[k]
                return 0
            except Exception:
                return 1

        cb = MOTION_FN(fn)
        self._motion_fns[j] = cb   # the library holds the pointer: keep the callback alive
        self._check(self.L.mpm_set_object_motion(self.h, j, cb, None), "mpm_set_object_motion")

    def set_penalty(self, penalty: Optional[S.Penalty]):
        """Penalty collision objects (IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES, one per object);
        None removes them."""
        objects = penalty.objects if penalty is not None else []
        arr = (CollisionObject * max(len(objects), 1))()
        for i, o in enumerate(objects):
            arr[i].kind, arr[i].type, arr[i].friction = o.kind, o.type, o.friction
            for a in range(self.dim):
                arr[i].a[a], arr[i].b[a] = o.a[a], o.b[a]
        k, sep = (penalty.stiffness, penalty.separation) if penalty is not None else (0.0, 0.0)
        self._check(self.L.mpm_set_penalty_objects(self.h, arr, len(objects), k, sep), "mpm_set_penalty_objects")

    def set_particles(self, X, V, F, B, mass, volume, mu, lam, valid=None, dtype=np.float64):
        """Arrays in the reference layout: X,V (n,d); F,B (n,d,d) row/col as numpy matrices."""
        d = self.dim
        n = X.shape[0]
        self._keep = [np.ascontiguousarray(X, dtype), np.ascontiguousarray(V, dtype),
                      np.ascontiguousarray(np.swapaxes(F, 1, 2).reshape(n, d * d), dtype),
                      np.ascontiguousarray(np.swapaxes(B, 1, 2).reshape(n, d * d), dtype),
                      np.ascontiguousarray(mass, dtype), np.ascontiguousarray(volume, dtype),
                      np.ascontiguousarray(mu, dtype), np.ascontiguousarray(lam, dtype)]
        v = ParticlesView()
        v.n, v.dtype, v.on_device = n, FP64 if dtype == np.float64 else FP32, 0
        v.X, v.V, v.F, v.B, v.mass, v.volume, v.mu, v.lambda_ = [a.ctypes.data for a in self._keep]
        vv = None
        if valid is not None:
            vv = np.ascontiguousarray(valid, np.uint8)
            v.valid = vv.ctypes.data
        self._check(self.L.mpm_set_particles(self.h, ctypes.byref(v)), "mpm_set_particles")
        self._keep = None
        self.n = n

    def _native(self, arrays, n, what):
        dtype = arrays[0].dtype
        if dtype not in (np.float32, np.float64):
            raise ValueError("%s: float32 or float64 arrays" % what)
        d = self.dim
        shapes = [(n, d), (n, d), (n, d * d), (n, d * d)] + [(n,)] * (len(arrays) - 4)
        for arr, shp in zip(arrays, shapes):
            if arr.dtype != dtype or arr.shape != shp or not arr.flags.c_contiguous:
                raise ValueError("%s: arrays must be C-contiguous %s of shapes %s" % (what, dtype, shapes))
        return FP64 if dtype == np.float64 else FP32

    def set_particles_native(self, X, V, Fc, Bc, mass, volume, mu, lam, valid=None):
        """Arrays already in the C-ABI (PhysBAM) layout, passed by pointer with no
        host-side copy: X, V (n, d); Fc, Bc (n, d*d) with F[i + d*j] = F(i, j);
        mass, volume, mu, lambda (n,); all one float dtype, C-contiguous.  With
        page-locked (pinned) arrays the upload is a plain DMA."""
        n = X.shape[0]
        v = ParticlesView()
        v.n, v.dtype, v.on_device = n, self._native([X, V, Fc, Bc, mass, volume, mu, lam], n, "set_particles_native"), 0
        v.X, v.V, v.F, v.B, v.mass, v.volume, v.mu, v.lambda_ = [a.ctypes.data for a in (X, V, Fc, Bc, mass, volume, mu, lam)]
        if valid is not None:
            if valid.dtype != np.uint8 or valid.shape != (n,) or not valid.flags.c_contiguous:
                raise ValueError("set_particles_native: valid must be a contiguous uint8 array of n")
            v.valid = valid.ctypes.data
        self._check(self.L.mpm_set_particles(self.h, ctypes.byref(v)), "mpm_set_particles")
        self.n = n

    def get_particles_native(self, X, V, Fc, Bc, valid=None):
        """Fill caller arrays in the C-ABI layout (as set_particles_native) with
        the particle state, in the caller's particle order, no host-side copy."""
        n = self.n
        v = ParticlesView()
        v.n, v.dtype, v.on_device = n, self._native([X, V, Fc, Bc], n, "get_particles_native"), 0
        v.X, v.V, v.F, v.B = X.ctypes.data, V.ctypes.data, Fc.ctypes.data, Bc.ctypes.data
        if valid is not None:
            if valid.dtype != np.uint8 or valid.shape != (n,) or not valid.flags.c_contiguous:
                raise ValueError("get_particles_native: valid must be a contiguous uint8 array of n")
            v.valid = valid.ctypes.data
        self._check(self.L.mpm_get_particles(self.h, ctypes.byref(v)), "mpm_get_particles")

    def set_scene_particles(self, scene: Optional[S.Scene] = None, dtype=np.float64):
        s = scene or self.scene
        self.set_particles(s.X, s.V, s.F, s.B, s.mass, s.volume, s.mu, s.lam, dtype=dtype)
        self._attrs = {"mass": s.mass, "volume": s.volume, "mu": s.mu, "lam": s.lam}
        if getattr(s, "models", None) is not None:
            self.set_particle_models(s.models)
        if getattr(s, "plastic_mask", None) is not None:
            self.set_plastic_particles(s.plastic_mask)

    def set_plastic_particles(self, mask: Optional[np.ndarray]):
        """The particles the plasticity acts on (mpm_set_plastic_particles); None: all.
        Restarts the plastic state."""
        if mask is None:
            self._check(self.L.mpm_set_plastic_particles(self.h, None, 0), "mpm_set_plastic_particles")
            return
        m = np.ascontiguousarray(mask, np.uint8)
        self._check(self.L.mpm_set_plastic_particles(self.h, m.ctypes.data_as(ctypes.c_void_p), m.shape[0]),
                    "mpm_set_plastic_particles")

    def set_particle_models(self, models: Optional[np.ndarray]):
        """A constitutive model per particle (mpm_set_particle_models); None: the scene's."""
        if models is None:
            self._check(self.L.mpm_set_particle_models(self.h, None, 0), "mpm_set_particle_models")
            return
        m = np.ascontiguousarray(models, np.uint8)
        self._check(self.L.mpm_set_particle_models(self.h, m.ctypes.data_as(ctypes.c_void_p), m.shape[0]),
                    "mpm_set_particle_models")

    def get_particles(self, dtype=np.float64):
        d, n = self.dim, self.n
        X = np.empty((n, d), dtype)
        V = np.empty((n, d), dtype)
        F = np.empty((n, d * d), dtype)
        B = np.empty((n, d * d), dtype)
        valid = np.empty(n, np.uint8)
        v = ParticlesView()
        v.n, v.dtype, v.on_device = n, FP64 if dtype == np.float64 else FP32, 0
        v.X, v.V, v.F, v.B = X.ctypes.data, V.ctypes.data, F.ctypes.data, B.ctypes.data
        v.valid = valid.ctypes.data
        self._check(self.L.mpm_get_particles(self.h, ctypes.byref(v)), "mpm_get_particles")
        F = np.swapaxes(F.reshape(n, d, d), 1, 2)
        B = np.swapaxes(B.reshape(n, d, d), 1, 2)
        return {"X": X, "V": V, "F": F, "B": B, "valid": valid.astype(bool)}

    # -- device-resident arrays (torch tensors on the handle's device) ------------
    def _dev_view(self, X, V, Fc, Bc, mass=None, volume=None, mu=None, lam=None, valid=None):
        import torch
        ts = [X, V, Fc, Bc, mass, volume, mu, lam]
        dt = X.dtype
        for t in ts:
            if t is not None:
                assert t.is_cuda and t.is_contiguous() and t.dtype == dt, "contiguous CUDA tensors of one dtype"
        v = ParticlesView()
        v.n, v.on_device = X.shape[0], 1
        v.dtype = FP64 if dt == torch.float64 else FP32
        v.X, v.V, v.F, v.B = X.data_ptr(), V.data_ptr(), Fc.data_ptr(), Bc.data_ptr()
        if mass is not None:
            v.mass, v.volume, v.mu, v.lambda_ = mass.data_ptr(), volume.data_ptr(), mu.data_ptr(), lam.data_ptr()
        if valid is not None:
            v.valid = valid.data_ptr()
        return v

    def set_particles_device(self, X, V, Fc, Bc, mass, volume, mu, lam):
        """Device tensors; F and B column-major per particle (i.e. F[p].T flattened)."""
        import torch
        torch.cuda.current_stream().synchronize()
        v = self._dev_view(X, V, Fc, Bc, mass, volume, mu, lam)
        self._check(self.L.mpm_set_particles(self.h, ctypes.byref(v)), "mpm_set_particles")
        self.n = X.shape[0]

    def get_particles_device(self, dtype):
        import torch
        n, d = self.n, self.dim
        X = torch.empty((n, d), dtype=dtype, device="cuda")
        V = torch.empty_like(X)
        Fc = torch.empty((n, d * d), dtype=dtype, device="cuda")
        Bc = torch.empty_like(Fc)
        valid = torch.empty(n, dtype=torch.uint8, device="cuda")
        torch.cuda.current_stream().synchronize()
        v = self._dev_view(X, V, Fc, Bc, valid=valid)
        self._check(self.L.mpm_get_particles(self.h, ctypes.byref(v)), "mpm_get_particles")
        return X, V, Fc, Bc, valid

    # -- output frames and restart (PhysBAM's viewer directory) ---------------------
    def write_frame(self, directory: str, frame: int, use_doubles: bool = True):
        """Write the particle state as the reference's Write_Output_Files does
        (physbam_b200.io): <directory>/<frame>/mpm_particles.gz, restart_data.gz and
        common/grid.gz, readable by the reference and by read_frame."""
        from . import io
        p = self.get_particles()
        sc = self.scene
        parts = {"X": p["X"], "V": p["V"], "F": p["F"], "B": p["B"], "valid": p["valid"],
                 "mass": self._attr("mass"), "volume": self._attr("volume")}
        if getattr(self, "plasticity", None) is not None:
            st = self.get_plastic_state()
            parts["mu"], parts["lambda"] = st["mu"], st["lam"]
            for k, name in io.PLASTIC_NAMES.items():
                if k in st:
                    parts[name] = st[k]
        else:
            parts["mu"], parts["lambda"] = self._attr("mu"), self._attr("lam")
        io.write_frame(directory, frame, self.time, parts, counts=sc.counts[:self.dim],
                       domain_min=sc.domain_min[:self.dim], domain_max=sc.domain_max[:self.dim], use_doubles=use_doubles)

    def read_frame(self, directory: str, frame: int):
        """Restart from a frame (MPM_EXAMPLE::Read_Output_Files): the particles of
        mpm_particles.gz (the plastic arrays too, where the file has them) and the time."""
        from . import io
        f = io.read_frame(directory, frame)
        self.set_particles(f["X"], f["V"], f["F"], f["B"], f["mass"], f["volume"], f["mu"], f["lambda"],
                           valid=f["valid"])
        self._attrs = {"mass": f["mass"], "volume": f["volume"], "mu": f["mu"], "lam": f["lambda"]}
        if getattr(self, "plasticity", None) is not None:
            keys = {k: f[name] for k, name in io.PLASTIC_NAMES.items() if name in f and k in self._plastic_keys()}
            if keys:
                self.set_plastic_state(**keys)
        self.time = f["time"]

    def _attr(self, name):
        """Per-particle constants as last set (mass, volume, mu, lam)."""
        a = getattr(self, "_attrs", None)
        if a is not None:
            return a[name]
        return getattr(self.scene, name)

    # -- reflection boundary conditions -----------------------------------------
    def set_reflection(self, reflection: Optional[S.Reflection]):
        r = ReflectionDesc()
        if reflection is not None:
            r.enabled = 1
            for k, t in enumerate(reflection.side_type):
                r.side_type[k] = int(t)
            r.friction, r.full_reflection = reflection.friction, 1 if reflection.full else 0
        self._check(self.L.mpm_set_reflection(self.h, ctypes.byref(r)), "mpm_set_reflection")

    # -- adaptive substeps (Simulate_To_Frame) -------------------------------------
    def set_dt_control(self, control: S.DtControl):
        c = DtControlDesc()
        c.cfl, c.min_dt, c.max_dt = control.cfl, control.min_dt, control.max_dt
        c.strong_cfl, c.cfl_F = 1 if control.strong_cfl else 0, control.cfl_F
        c.sound_cfl, c.cfl_sound = 1 if control.sound_cfl else 0, control.cfl_sound
        self._check(self.L.mpm_set_dt_control(self.h, ctypes.byref(c)), "mpm_set_dt_control")
        self.dt_control = control

    def simulate_frame(self, frame_dt: Optional[float] = None) -> int:
        """MPM_DRIVER::Simulate_To_Frame for one frame; returns the substeps taken."""
        frame_dt = self.dt_control.frame_dt if frame_dt is None else frame_dt
        t, n = ctypes.c_double(), ctypes.c_int()
        self._check(self.L.mpm_simulate_frame(self.h, self.time, frame_dt, ctypes.byref(t), ctypes.byref(n)),
                    "mpm_simulate_frame")
        self.time = t.value
        return n.value

    def last_dt(self) -> float:
        x = ctypes.c_double()
        self._check(self.L.mpm_last_dt(self.h, ctypes.byref(x)), "mpm_last_dt")
        return x.value

    # -- backward Euler ---------------------------------------------------------
    def set_implicit(self, implicit: Optional[S.Implicit]):
        """Newton backward-Euler force solve (a `scenes.Implicit`) or symplectic Euler (None)."""
        d = ImplicitDesc()
        if implicit is not None:
            d.enabled = 1
            d.newton_tolerance, d.newton_iterations = implicit.newton_tolerance, int(implicit.newton_iterations)
            d.solver_tolerance, d.solver_iterations = implicit.solver_tolerance, int(implicit.solver_iterations)
        self._check(self.L.mpm_set_implicit(self.h, ctypes.byref(d)), "mpm_set_implicit")

    def implicit_stats(self):
        st = ImplicitStats()
        self._check(self.L.mpm_get_implicit_stats(self.h, ctypes.byref(st)), "mpm_get_implicit_stats")
        return {"newton_iterations": st.newton_iterations, "krylov_iterations": st.krylov_iterations,
                "converged": bool(st.converged), "residual": st.residual}

    # -- plasticity (MPM_PLASTICITY_CLAMP) -------------------------------------
    def set_plasticity(self, plasticity):
        """Plasticity after every G2P: a `scenes.Plasticity` (snow clamp), a
        `scenes.DruckerPrager` (sand) or None (off).  Particles start unplastic."""
        d = PlasticityDesc()
        if plasticity is not None:
            d.kind = plasticity.kind
            if isinstance(plasticity, S.Plasticity):
                d.theta_c, d.theta_s = plasticity.theta_c, plasticity.theta_s
                d.max_hardening, d.hardening_factor = plasticity.max_hardening, plasticity.hardening_factor
            else:
                d.dp_a0, d.dp_a1, d.dp_a3, d.dp_a4 = plasticity.a0, plasticity.a1, plasticity.a3, plasticity.a4
                d.cohesion, d.use_vc = plasticity.cohesion, 1 if plasticity.use_vc else 0
        self._check(self.L.mpm_set_plasticity(self.h, ctypes.byref(d)), "mpm_set_plasticity")
        self.plasticity = plasticity

    def _plastic_keys(self):
        pl = getattr(self, "plasticity", None)
        if pl is None:
            return ("Fp", "mu", "lam")   # the library reports "plasticity is off"
        if pl.kind == S.PLASTICITY_CLAMP:
            return ("Fp", "mu", "lam", "mu0", "lam0")
        return ("Fp", "mu", "lam") + S.plastic_keys(pl)[1:]

    def get_plastic_state(self, dtype=np.float64):
        """The plastic state in the caller's particle order: "Fp" (n,d,d), the current
        "mu", "lam", and per kind "mu0", "lam0" (clamp) or "pdef", "rho_F",
        "cohesion", "vc" (Drucker-Prager), each (n,)."""
        d, n = self.dim, self.n
        v = PlasticView()
        v.n, v.dtype, v.on_device = n, FP64 if dtype == np.float64 else FP32, 0
        out = {}
        for k in self._plastic_keys():
            out[k] = np.empty((n, d * d) if k == "Fp" else n, dtype)
            setattr(v, _PLASTIC_FIELDS[k], out[k].ctypes.data)
        self._check(self.L.mpm_get_plastic_state(self.h, ctypes.byref(v)), "mpm_get_plastic_state")
        out["Fp"] = np.swapaxes(out["Fp"].reshape(n, d, d), 1, 2)
        return out

    def set_plastic_state(self, dtype=np.float64, **arrays):
        """Overwrite any subset of the plastic state, by the keys of get_plastic_state
        (Fp as (n,d,d) matrices)."""
        d, n = self.dim, self.n
        v = PlasticView()
        v.n, v.dtype, v.on_device = n, FP64 if dtype == np.float64 else FP32, 0
        keep = []
        for k, a in arrays.items():
            if a is None:
                continue
            if k not in _PLASTIC_FIELDS:
                raise ValueError("set_plastic_state: unknown array %r" % k)
            a = np.asarray(a)
            if k == "Fp":
                a = np.swapaxes(a, 1, 2).reshape(n, d * d)
            a = np.ascontiguousarray(a, dtype)
            if a.shape[0] != n:
                raise ValueError("set_plastic_state: arrays of n = %d particles" % n)
            keep.append(a)
            setattr(v, _PLASTIC_FIELDS[k], a.ctypes.data)
        self._check(self.L.mpm_set_plastic_state(self.h, ctypes.byref(v)), "mpm_set_plastic_state")

    # -- differentiation -------------------------------------------------------
    def set_diff_tape_budget(self, nbytes):
        """Memory the next diff_forward may keep for a backward without recomputation
        (< 0: a quarter of the free device memory, 0: checkpoints only)."""
        self._check(self.L.mpm_set_diff_tape_budget(self.h, int(nbytes)), "mpm_set_diff_tape_budget")

    def diff_forward(self, nsteps, checkpoint_every=8, dt=None):
        dt = self.scene.dt if dt is None else dt
        self._check(self.L.mpm_diff_forward(self.h, dt, nsteps, checkpoint_every), "mpm_diff_forward")
        self.time += nsteps * dt

    def diff_backward(self, gX, gV, gFc, gBc):
        """Device tensors of dL/d(final X, V, F col-major, B col-major); returns the initial-state grads + mu, lambda."""
        import torch
        n = self.n
        out = [torch.empty_like(gX), torch.empty_like(gV), torch.empty_like(gFc), torch.empty_like(gBc)]
        gmu = torch.empty(n, dtype=gX.dtype, device="cuda")
        glam = torch.empty_like(gmu)
        torch.cuda.current_stream().synchronize()
        vin = self._dev_view(gX.contiguous(), gV.contiguous(), gFc.contiguous(), gBc.contiguous())
        vout = self._dev_view(*out)
        self._check(self.L.mpm_diff_backward(self.h, ctypes.byref(vin), ctypes.byref(vout),
                                             ctypes.c_void_p(gmu.data_ptr()), ctypes.c_void_p(glam.data_ptr())),
                    "mpm_diff_backward")
        return (*out, gmu, glam)

    # -- the substep (MPM_DRIVER.cpp:141-157) --------------------------------
    def Advance_One_Time_Step(self, dt: Optional[float] = None):
        dt = self.scene.dt if dt is None else dt
        if getattr(self.scene, "node_force", None) is not None:   # the caller's force between the phases
            self.Particle_To_Grid(dt)
            self.add_grid_forces(self._node_force_array(), dt)
            self.Apply_Forces(dt)
            self.Grid_To_Particle(dt)
            return
        self._check(self.L.mpm_substep(self.h, dt, self.time), "mpm_substep")
        self.time += dt

    def _node_force_array(self):
        shape = tuple(c + 2 * S.GHOST for c in self.scene.counts[:self.dim])
        f = np.empty(shape + (self.dim,))
        f[...] = np.asarray(self.scene.node_force, np.float64)[:self.dim]
        return f

    def add_grid_forces(self, force: np.ndarray, dt: Optional[float] = None):
        """Extra node forces (ghosted grid, d per node) for the next grid update (mpm_add_grid_forces)."""
        dt = self.scene.dt if dt is None else dt
        f = np.ascontiguousarray(force, np.float64)
        shape = tuple(c + 2 * S.GHOST for c in self.scene.counts[:self.dim]) + (self.dim,)
        if f.shape != shape:
            raise ValueError("node forces must have shape %s" % (shape,))
        self._check(self.L.mpm_add_grid_forces(self.h, dt, _ptr(f), FP64, 0), "mpm_add_grid_forces")

    def Particle_To_Grid(self, dt=None):
        self._check(self.L.mpm_particle_to_grid(self.h, self.scene.dt if dt is None else dt, self.time), "p2g")

    def Apply_Forces(self, dt=None):
        self._check(self.L.mpm_apply_forces(self.h, self.scene.dt if dt is None else dt, self.time), "forces")

    def Grid_To_Particle(self, dt=None):
        dt = self.scene.dt if dt is None else dt
        self._check(self.L.mpm_grid_to_particle(self.h, dt, self.time), "g2p")
        self.time += dt

    def advance(self, nsteps: int, dt: Optional[float] = None):
        """Fixed-dt substep loop (Simulate_To_Frame with min_dt = max_dt), CUDA-graph replay."""
        dt = self.scene.dt if dt is None else dt
        if getattr(self.scene, "node_force", None) is not None:
            for _ in range(nsteps):
                self.Advance_One_Time_Step(dt)
            return
        self._check(self.L.mpm_advance(self.h, dt, self.time, nsteps), "mpm_advance")
        self.time += nsteps * dt

    def synchronize(self):
        self._check(self.L.mpm_synchronize(self.h), "mpm_synchronize")

    def set_stream(self, stream_ptr: int):
        self._check(self.L.mpm_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "mpm_set_stream")

    # -- inspection -----------------------------------------------------------
    def get_grid(self, want_v0=False):
        shape = tuple(c + 2 * S.GHOST for c in self.scene.counts[:self.dim])
        gn = int(np.prod(shape))
        m = np.zeros(gn)
        v0 = np.zeros(gn * self.dim) if want_v0 else None
        v = np.zeros(gn * self.dim)
        vf = np.zeros(gn * self.dim)
        self._check(self.L.mpm_get_grid(self.h, _ptr(m), _ptr(v0), _ptr(v), _ptr(vf)), "mpm_get_grid")
        out = {"grid_m": m.reshape(shape), "grid_v": v.reshape(shape + (self.dim,)),
               "grid_vf": vf.reshape(shape + (self.dim,))}
        if want_v0:
            out["grid_v0"] = v0.reshape(shape + (self.dim,))
        return out

    def sort_state(self):
        n = self.n
        keys, sk, perm = (np.empty(n, np.uint32) for _ in range(3))
        self._check(self.L.mpm_debug_sort_state(self.h, _ptr(keys), _ptr(sk), _ptr(perm)), "mpm_debug_sort_state")
        return keys, sk, perm

    def autotune(self, substeps=3, dt=None, cold_l2=False):
        """Time every launch-shape choice of the fast path on the current state
        (restored after each trial) and keep the fastest; returns the report.
        cold_l2: scrub the L2 before every timed substep."""
        dt = self.scene.dt if dt is None else dt
        buf = ctypes.create_string_buffer(4096)
        self._check(self.L.mpm_autotune_ex(self.h, dt, substeps, 1 if cold_l2 else 0, buf, 4096), "mpm_autotune_ex")
        return buf.value.decode()

    def set_launch_shape(self, p2g_variant, g2p_threads=128, cta_mult=1):
        self._check(self.L.mpm_set_launch_shape(self.h, p2g_variant, g2p_threads, cta_mult), "mpm_set_launch_shape")

    def get_launch_shape(self):
        v = [ctypes.c_int() for _ in range(3)]
        self._check(self.L.mpm_get_launch_shape(self.h, *[ctypes.byref(x) for x in v]), "mpm_get_launch_shape")
        return tuple(x.value for x in v)

    def particle_totals(self):
        t = Totals()
        self._check(self.L.mpm_particle_totals(self.h, ctypes.byref(t)), "mpm_particle_totals")
        return t.as_dict()

    def grid_totals(self):
        t = Totals()
        self._check(self.L.mpm_grid_totals(self.h, ctypes.byref(t)), "mpm_grid_totals")
        return t.as_dict()

    def compute_dt(self, cfl=1.0, max_dt=None):
        out = ctypes.c_double()
        max_dt = self.scene.dt if max_dt is None else max_dt
        self._check(self.L.mpm_compute_dt(self.h, cfl, max_dt, ctypes.byref(out)), "mpm_compute_dt")
        return out.value

    def count_valid(self) -> int:
        c = ctypes.c_int64()
        self._check(self.L.mpm_count_valid(self.h, ctypes.byref(c)), "mpm_count_valid")
        return int(c.value)

    def set_timing(self, on: bool):
        self._check(self.L.mpm_set_timing(self.h, 1 if on else 0), "mpm_set_timing")

    def get_timing(self):
        names = ctypes.create_string_buffer(4096)
        ms = (ctypes.c_double * 64)()
        launches = (ctypes.c_int64 * 64)()
        count = ctypes.c_int()
        self._check(self.L.mpm_get_timing(self.h, names, 4096, ctypes.cast(ms, ctypes.c_void_p),
                                          ctypes.cast(launches, ctypes.c_void_p), 64, ctypes.byref(count)),
                    "mpm_get_timing")
        keys = names.value.decode().split(",") if count.value else []
        return {k: (ms[i], launches[i]) for i, k in enumerate(keys)}


def radix_sort_u32(keys: np.ndarray, bits: int = 32):
    """Sort uint32 keys by their low `bits` bits on the GPU; returns (sorted_keys, perm)."""
    L = load_library()
    k = np.ascontiguousarray(keys, np.uint32)
    out = np.empty_like(k)
    perm = np.empty_like(k)
    rc = L.mpm_radix_sort_u32(_ptr(k), k.size, bits, _ptr(out), _ptr(perm))
    if rc != MPM_OK:
        raise MPMError(rc, "mpm_radix_sort_u32")
    return out, perm


class SceneDesc(ctypes.Structure):
    _fields_ = [("grid", GridDesc), ("model", ctypes.c_int), ("gravity", ctypes.c_double * 3),
                ("particle_count", ctypes.c_int64), ("first_object", ctypes.c_int), ("object_count", ctypes.c_int)]


class MPM_BATCH(MPM_DRIVER):
    """Many independent 3D scenes advanced together (mpm_batch_create): every phase
    of the substep is one persistent launch over all scenes.  FP32 fast path."""

    def __init__(self, scenes_list):
        self.L = load_library()
        L = self.L
        L.mpm_batch_create.argtypes = [ctypes.POINTER(SceneDesc), ctypes.c_int, ctypes.POINTER(CollisionObject),
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mpm_batch_create.restype = ctypes.c_int
        self.scenes = list(scenes_list)
        self.scene = self.scenes[0]
        if any(s.penalty is not None for s in self.scenes):
            raise ValueError("a batch takes no penalty collision objects")
        if any(o.motion is not None for s in self.scenes for o in s.objects):
            raise ValueError("a batch takes no moving collision objects")
        self.dim = 3
        self.precision, self.path = FP32, PATH_FAST
        descs = (SceneDesc * len(self.scenes))()
        objs = []
        for i, s in enumerate(self.scenes):
            if s.dim != 3:
                raise ValueError("batched scenes are 3D")
            d = descs[i]
            d.grid.dim, d.grid.ghost = 3, S.GHOST
            for a in range(3):
                d.grid.counts[a] = s.counts[a]
                d.grid.domain_min[a], d.grid.domain_max[a] = s.domain_min[a], s.domain_max[a]
                d.gravity[a] = s.gravity[a]
            d.model = s.model
            d.particle_count = s.n
            d.first_object, d.object_count = len(objs), len(s.objects)
            objs += list(s.objects)
        arr = (CollisionObject * max(len(objs), 1))()
        for i, o in enumerate(objs):
            arr[i].kind, arr[i].type, arr[i].friction = o.kind, o.type, o.friction
            for a in range(3):
                arr[i].a[a], arr[i].b[a] = o.a[a], o.b[a]
        self.h = ctypes.c_void_p()
        self._check(L.mpm_batch_create(descs, len(self.scenes), arr, len(objs), ctypes.byref(self.h)), "mpm_batch_create")
        # one plasticity per handle: the scenes of a batch share it
        pl = self.scenes[0].plasticity
        if any(s.plasticity != pl for s in self.scenes):
            raise ValueError("the scenes of a batch share one plasticity (or none)")
        if pl is not None:
            self.set_plasticity(pl)
        self.time = 0.0
        self.n = 0
        self.offsets = np.cumsum([0] + [s.n for s in self.scenes])

    def set_scene_particles(self, scene=None, dtype=np.float64):
        cat = lambda name: np.concatenate([getattr(s, name) for s in self.scenes])
        self.set_particles(cat("X"), cat("V"), cat("F"), cat("B"), cat("mass"), cat("volume"), cat("mu"), cat("lam"),
                           dtype=dtype)

    def split(self, arrays):
        return [{k: v[self.offsets[i]:self.offsets[i + 1]] for k, v in arrays.items()} for i in range(len(self.scenes))]

    def get_scene_grid(self, i):
        """Scene i's ghosted grid of the last substep (mpm_batch_get_grid): mass, velocity, friction velocity."""
        s = self.scenes[i]
        shape = tuple(c + 2 * S.GHOST for c in s.counts[:3])
        gn = int(np.prod(shape))
        m, v, vf = np.zeros(gn), np.zeros(gn * 3), np.zeros(gn * 3)
        self._check(self.L.mpm_batch_get_grid(self.h, int(i), _ptr(m), _ptr(v), _ptr(vf)), "mpm_batch_get_grid")
        return {"grid_m": m.reshape(shape), "grid_v": v.reshape(shape + (3,)), "grid_vf": vf.reshape(shape + (3,))}


