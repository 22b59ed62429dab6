"""CPU oracle for the explicit MPM substep -- TEST INFRASTRUCTURE ONLY.

Two checkers live here, used only by tests/, the smoke check and bench.py's
CPU-baseline leg, never by the product path:

* ``mpm_oracle.c``: a plain-C FP64 restatement of the reference's substep
  (``PhysBAM Hybrid_Methods MPM_DRIVER``), built to ``oracle/liboracle.so``.
* ``_ref/ref_scene``: the reference itself (its own sources compiled by
  ``ref.mk``) driven by ``ref_scene.cpp`` on a scene file.  Present only where
  the reference sources were available at build time; its dumps are frozen into
  ``tests/golden/`` by ``tests/golden/make_golden.py``.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SCENE = os.path.join(REF_DIR, "ref_scene")
MAXOBJ = 32


class _Obj(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("type", ctypes.c_int), ("friction", ctypes.c_double),
                ("a", ctypes.c_double * 3), ("b", ctypes.c_double * 3), ("moving", ctypes.c_int),
                ("R0", ctypes.c_double * 9), ("x0", ctypes.c_double * 3), ("R1", ctypes.c_double * 9),
                ("x1", ctypes.c_double * 3), ("v", ctypes.c_double * 3), ("w", ctypes.c_double * 3)]


class _Scene(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("counts", ctypes.c_int * 3), ("dmin", ctypes.c_double * 3),
                ("dmax", ctypes.c_double * 3), ("model", ctypes.c_int), ("gravity", ctypes.c_double * 3),
                ("nobj", ctypes.c_int), ("obj", _Obj * MAXOBJ), ("npen", ctypes.c_int),
                ("pen_stiffness", ctypes.c_double), ("pen_separation", ctypes.c_double), ("pen", _Obj * MAXOBJ),
                ("models", ctypes.POINTER(ctypes.c_ubyte))]


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc, no FMA contraction so it rounds like the reference's x86-64 build)."""
    src = os.path.join(HERE, "mpm_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off",
                               "-o", LIB, src, "-lm"])
    return LIB


def reference_root():
    """The PhysBAM checkout: $PHYSBAM_REFERENCE, else a directory named
    ``reference`` beside this repository; None when neither holds Public_Library."""
    cands = [os.environ.get("PHYSBAM_REFERENCE"), os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "Public_Library")):
            return c
    return None


def build_ref(ref_root: str = None, jobs: int = os.cpu_count() or 8) -> bool:
    """Compile the reference's MPM path from its sources (minutes on first run)."""
    ref_root = ref_root or reference_root()
    if not ref_root or not os.path.isdir(ref_root):
        return os.path.exists(REF_SCENE)
    subprocess.check_call(["make", "-f", os.path.join(HERE, "ref.mk"), "-j%d" % jobs, "REF=" + ref_root,
                           "OUT=" + REF_DIR], cwd=os.path.dirname(HERE))
    return True


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        P = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_substep.argtypes = [ctypes.POINTER(_Scene), ctypes.c_longlong, P, P, P, P, P, P, P, P,
                                        ctypes.POINTER(ctypes.c_ubyte), ctypes.c_double, ctypes.c_double,
                                        P, P, P, P]
        _lib.oracle_substep.restype = ctypes.c_int
        _lib.oracle_run.argtypes = [ctypes.POINTER(_Scene), ctypes.c_longlong, P, P, P, P, P, P, P, P,
                                    ctypes.POINTER(ctypes.c_ubyte), ctypes.c_double, ctypes.c_double, ctypes.c_int]
        _lib.oracle_run.restype = ctypes.c_int
        _lib.oracle_pft.argtypes = [ctypes.c_int, ctypes.c_int, P, ctypes.c_double, ctypes.c_double, P]
        _lib.oracle_svd3.argtypes = [P, P, P, P]
        _lib.oracle_svd3.restype = ctypes.c_int
        _lib.oracle_plastic_clamp.argtypes = [ctypes.c_int, ctypes.c_longlong, P, P, P, P, P, P,
                                              ctypes.POINTER(ctypes.c_ubyte), P]
        _lib.oracle_dp_init.argtypes = [ctypes.c_longlong, P, P, P, P, ctypes.c_double, P]
        _lib.oracle_plastic_dp.argtypes = [ctypes.c_int, ctypes.c_longlong, P, P, P, P, P, P, P, P,
                                           ctypes.POINTER(ctypes.c_ubyte), P]
    return _lib


def _rotation(dim, q):
    """ROTATION<TV>::Rotation_Matrix of a unit quaternion (w, x, y, z), in 2D of (cos, sin),
    column-major."""
    if dim == 2:
        m = np.hypot(q[0], q[1])
        c, s = (q[0] / m, q[1] / m) if m > 0 else (1.0, 0.0)
        return [c, s, -s, c]
    m = float(np.sqrt(sum(x * x for x in q[:4])))
    w, x, y, z = (q[0] / m, q[1] / m, q[2] / m, q[3] / m) if m > 0 else (1.0, 0.0, 0.0, 0.0)
    return [1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y),
            2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x),
            2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)]


def _scene_struct(s, time: float = 0.0) -> _Scene:
    c = _Scene()
    c.dim = s.dim
    for a in range(3):
        c.counts[a] = s.counts[a] if a < s.dim else 1
        c.dmin[a] = s.domain_min[a] if a < s.dim else 0.0
        c.dmax[a] = s.domain_max[a] if a < s.dim else 1.0
        c.gravity[a] = s.gravity[a] if a < s.dim else 0.0
    c.model = s.model
    if len(s.objects) > MAXOBJ:
        raise ValueError("too many collision objects")
    c.nobj = len(s.objects)
    for i, o in enumerate(s.objects):
        c.obj[i].kind, c.obj[i].type, c.obj[i].friction = o.kind, o.type, o.friction
        for a in range(s.dim):
            c.obj[i].a[a], c.obj[i].b[a] = o.a[a], o.b[a]
        m = getattr(o, "motion", None)
        if m is not None:   # the frames at the substep's start and end, the twist at its end
            t0, q0, _, _ = m.state(s.dim, time)
            t1, q1, lin, ang = m.state(s.dim, time + s.dt)
            c.obj[i].moving = 1
            for k, val in enumerate(_rotation(s.dim, q0)):
                c.obj[i].R0[k] = val
            for k, val in enumerate(_rotation(s.dim, q1)):
                c.obj[i].R1[k] = val
            for k in range(s.dim):
                c.obj[i].x0[k], c.obj[i].x1[k], c.obj[i].v[k] = t0[k], t1[k], lin[k]
            for k in range(len(ang)):
                c.obj[i].w[k] = ang[k]
    models = getattr(s, "models", None)
    if models is not None:
        c._models = np.ascontiguousarray(models, np.uint8)   # kept alive with the struct
        c.models = c._models.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
    pn = getattr(s, "penalty", None)
    if pn is not None and pn.objects:
        if len(pn.objects) > MAXOBJ:
            raise ValueError("too many penalty objects")
        c.npen, c.pen_stiffness, c.pen_separation = len(pn.objects), pn.stiffness, pn.separation
        for i, o in enumerate(pn.objects):
            c.pen[i].kind, c.pen[i].type, c.pen[i].friction = o.kind, o.type, o.friction
            for a in range(s.dim):
                c.pen[i].a[a], c.pen[i].b[a] = o.a[a], o.b[a]
    return c


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class State:
    """Particle state in the reference layout: X,V (n,d); F,B column-major (n,d*d)."""

    def __init__(self, scene):
        d = scene.dim
        self.scene = scene
        self.X = np.ascontiguousarray(scene.X, np.float64).copy()
        self.V = np.ascontiguousarray(scene.V, np.float64).copy()
        self.F = np.ascontiguousarray(np.swapaxes(scene.F, 1, 2).reshape(-1, d * d), np.float64)
        self.B = np.ascontiguousarray(np.swapaxes(scene.B, 1, 2).reshape(-1, d * d), np.float64)
        self.mass = np.ascontiguousarray(scene.mass, np.float64)
        self.vol = np.ascontiguousarray(scene.volume, np.float64)
        self.mu = np.ascontiguousarray(scene.mu, np.float64)
        self.lam = np.ascontiguousarray(scene.lam, np.float64)
        self.valid = np.ones(scene.n, np.uint8)
        self.time = 0.0
        pl = scene.plasticity
        if pl is not None:   # as the reference seeds them (STANDARD_TESTS_BASE.cpp:299,568-586)
            self.Fp = np.ascontiguousarray(np.tile(np.eye(d).reshape(1, d * d), (scene.n, 1)), np.float64)
            self.mu0, self.lam0 = self.mu.copy(), self.lam.copy()
            self.mu, self.lam = self.mu.copy(), self.lam.copy()
        if pl is not None and pl.kind == 2:   # MPM_DRUCKER_PRAGER::Initialize_Particles
            n = scene.n
            self.pdef, self.rho_F, self.cohesion, self.vc = (np.zeros(n) for _ in range(4))
            lib().oracle_dp_init(n, _ptr(self.pdef), _ptr(self.rho_F), _ptr(self.cohesion), _ptr(self.vc),
                                 pl.cohesion, _ptr(self._dp_prm()))
            mask = getattr(scene, "plastic_mask", None)
            if mask is not None:   # over the model's affected particles only; the rest keep zeros
                off = np.asarray(mask) == 0
                for a in (self.pdef, self.rho_F, self.cohesion, self.vc):
                    a[off] = 0.0

    def _dp_prm(self):
        pl = self.scene.plasticity
        return np.array([pl.a0, pl.a1, pl.a3, pl.a4, 1.0 if pl.use_vc else 0.0], np.float64)

    def plastic_state(self):
        """The plastic state with the keys of `scenes.plastic_keys` (Fp as (n,d,d) matrices)."""
        from physbam_b200 import scenes as S
        out = {}
        for k in S.plastic_keys(self.scene.plasticity):
            out[k] = self.Fp_rowmajor() if k == "Fp" else getattr(self, k)
        return out

    def Fp_rowmajor(self):
        d = self.scene.dim
        return np.swapaxes(self.Fp.reshape(-1, d, d), 1, 2)

    def plasticity(self, simulated):
        """Update_Plasticity_And_Hardening (MPM_DRIVER.cpp:922-928) after G2P, over the particles
        simulated in the substep (valid at its start, MPM_DRIVER::Update_Simulated_Particles)."""
        pl = self.scene.plasticity
        if pl is None:
            return
        sim = np.ascontiguousarray(simulated, np.uint8)
        mask = getattr(self.scene, "plastic_mask", None)
        if mask is not None:   # the plasticity's own particles (its gather_scatter's)
            sim = np.ascontiguousarray(sim & (np.asarray(mask) != 0), np.uint8)
        if pl.kind == 2:
            lib().oracle_plastic_dp(self.scene.dim, self.scene.n, _ptr(self.F), _ptr(self.Fp), _ptr(self.mu),
                                    _ptr(self.lam), _ptr(self.pdef), _ptr(self.rho_F), _ptr(self.cohesion),
                                    _ptr(self.vc), sim.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                    _ptr(self._dp_prm()))
            return
        prm = np.array([pl.theta_c, pl.theta_s, pl.max_hardening, pl.hardening_factor], np.float64)
        lib().oracle_plastic_clamp(self.scene.dim, self.scene.n, _ptr(self.F), _ptr(self.Fp), _ptr(self.mu),
                                   _ptr(self.lam), _ptr(self.mu0), _ptr(self.lam0),
                                   sim.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), _ptr(prm))

    def F_rowmajor(self):
        d = self.scene.dim
        return np.swapaxes(self.F.reshape(-1, d, d), 1, 2)

    def B_rowmajor(self):
        d = self.scene.dim
        return np.swapaxes(self.B.reshape(-1, d, d), 1, 2)


def substep(state: State, want_grid: bool = False):
    s = state.scene
    L = lib()
    sc = _scene_struct(s, state.time)
    gn = int(np.prod([c + 6 for c in s.counts[:s.dim]]))
    grids = None
    args = [None] * 4
    if want_grid:
        grids = [np.zeros(gn), np.zeros(gn * s.dim), np.zeros(gn * s.dim), np.zeros(gn * s.dim)]
        args = [_ptr(g) for g in grids]
    simulated = state.valid.copy()
    rc = L.oracle_substep(ctypes.byref(sc), s.n, _ptr(state.X), _ptr(state.V), _ptr(state.F), _ptr(state.B),
                          _ptr(state.mass), _ptr(state.vol), _ptr(state.mu), _ptr(state.lam),
                          state.valid.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), s.dt, state.time, *args)
    if rc:
        raise RuntimeError("oracle_substep failed: %d" % rc)
    state.plasticity(simulated)
    state.time += s.dt
    if want_grid:
        shape = tuple(c + 6 for c in s.counts[:s.dim])
        return {"grid_m": grids[0].reshape(shape), "grid_v0": grids[1].reshape(shape + (s.dim,)),
                "grid_v": grids[2].reshape(shape + (s.dim,)), "grid_vf": grids[3].reshape(shape + (s.dim,))}
    return None


def run(state: State, nsteps: int):
    s = state.scene
    if s.plasticity is not None or any(getattr(o, "motion", None) is not None for o in s.objects):
        for _ in range(nsteps):   # per-substep work on the host: plasticity, object frames
            substep(state)
        return
    sc = _scene_struct(s)
    rc = lib().oracle_run(ctypes.byref(sc), s.n, _ptr(state.X), _ptr(state.V), _ptr(state.F), _ptr(state.B),
                          _ptr(state.mass), _ptr(state.vol), _ptr(state.mu), _ptr(state.lam),
                          state.valid.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), s.dt, state.time, nsteps)
    if rc:
        raise RuntimeError("oracle_run failed: %d" % rc)
    state.time += nsteps * s.dt


def pft(dim, model, F_colmajor, mu, lam):
    out = np.zeros(dim * dim)
    Fc = np.ascontiguousarray(F_colmajor, np.float64)
    lib().oracle_pft(dim, model, _ptr(Fc), mu, lam, _ptr(out))
    return out


def ref_available() -> bool:
    return os.path.exists(REF_SCENE)


REF_B200 = os.path.join(REF_DIR, "ref_b200")


def b200_binding_available() -> bool:
    return os.path.exists(REF_B200)


def run_b200_binding(scene, use_float: bool = True, per_substep: bool = False):
    """Run ``scene`` through the reference-side binding (``oracle/ref_b200``: the
    reference's MPM_EXAMPLE set up from the scene file, its substeps run on the GPU
    by include/mpm_physbam.hpp).  Returns (state dict with X, V, F, B as (n,3,3)
    row-major matrices and valid, the runner's JSON report)."""
    import json
    from physbam_b200 import scenes as S
    tmp = tempfile.mkdtemp(prefix="mpmb200_")
    try:
        sp, dp = os.path.join(tmp, "scene.bin"), os.path.join(tmp, "dump.bin")
        S.write_scene(sp, scene, [])
        cmd = [REF_B200, sp, dp] + (["-float"] if use_float else []) + (["-substeps"] if per_substep else [])
        out = subprocess.run(cmd, check=True, capture_output=True, text=True)
        report = json.loads(out.stdout.strip().splitlines()[-1])
        with open(dp, "rb") as f:
            n = int(np.frombuffer(f.read(4), np.int32)[0])
            X = np.frombuffer(f.read(8 * n * 3), np.float64).reshape(n, 3)
            V = np.frombuffer(f.read(8 * n * 3), np.float64).reshape(n, 3)
            F = np.swapaxes(np.frombuffer(f.read(8 * n * 9), np.float64).reshape(n, 3, 3), 1, 2)
            B = np.swapaxes(np.frombuffer(f.read(8 * n * 9), np.float64).reshape(n, 3, 3), 1, 2)
            valid = np.frombuffer(f.read(n), np.uint8).astype(bool)
        return {"X": X, "V": V, "F": F, "B": B, "valid": valid}, report
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_reference(scene, dumps, threads: int = 1, use_float: bool = False, timing: bool = False, totals=None,
                  output: str = None, restart=None):
    """Run the reference's own driver on ``scene``; return {step: dump} (and timing JSON if asked).

    ``output`` keeps the viewer directory the driver writes; ``restart=(dir, frame)``
    starts from that frame's files (MPM_EXAMPLE::Read_Output_Files).
    With ``scene.dt_control`` the steps are frames of Simulate_To_Frame and the
    result is ``(dumps, {"frame_substeps": [...], "time": t})``.
    ``totals=(cfl, max_dt)`` returns instead ``(dumps, diagnostics)``: the
    reference's Total_Particle_* momenta and energy, Max_Particle_Speed,
    Grid_V_Upper_Bound and Compute_Dt on the final state."""
    from physbam_b200 import scenes as S
    tmp = tempfile.mkdtemp(prefix="mpmref_")
    try:
        sp, dp = os.path.join(tmp, "scene.bin"), os.path.join(tmp, "dump.bin")
        S.write_scene(sp, scene, dumps)
        cmd = [REF_SCENE, sp, dp, "-threads", str(threads)]
        if use_float:
            cmd.append("-float")
        if timing:
            cmd.append("-time")
        if totals is not None:
            cmd += ["-totals", repr(float(totals[0])), repr(float(totals[1]))]
        if output is not None:
            cmd += ["-output", output]
        if restart is not None:      # (viewer directory, frame): Read_Output_Files, then the substeps
            cmd += ["-restart", restart[0], str(int(restart[1]))]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True)
        res = S.read_dump(dp, scene.dim, scene.n, scene.counts, plastic=S.plastic_keys(scene.plasticity)) if dumps else {}
        if scene.dt_control is not None:   # frames: the substeps Simulate_To_Frame took per frame
            import json
            lines = [ln for ln in out.stdout.splitlines() if ln.startswith('{"frame_substeps"')]
            res = (res, json.loads(lines[-1]))
        if totals is not None:
            import json
            lines = [ln for ln in out.stdout.splitlines() if ln.startswith('{"mass"')]
            return res, json.loads(lines[-1])
        if timing:
            import json
            return res, json.loads(out.stdout.strip().splitlines()[-1])
        return res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def particle_totals(X, V, B, mass, valid, dx):
    """FP64 particle diagnostics in the reference's form.

    MPM_EXAMPLE::Total_Particle_Linear_Momentum / Angular_Momentum /
    Kinetic_Energy (Hybrid_Methods/Examples_And_Drivers/MPM_EXAMPLE.cpp:209-327)
    and MPM_DRIVER::Max_Particle_Speed / Grid_V_Upper_Bound
    (Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.cpp:1107-1138).  ``B`` is
    (n, d, d) with B[p, r, c]; ``dx`` the cell size per axis.
    """
    ok = np.asarray(valid, bool)
    X, V, B, m = (np.asarray(a, np.float64)[ok] for a in (X, V, B, mass))
    d = X.shape[1]
    dx = np.broadcast_to(np.asarray(dx, np.float64), (d,))
    if d == 3:
        eps = np.stack([B[:, 1, 2] - B[:, 2, 1], B[:, 2, 0] - B[:, 0, 2], B[:, 0, 1] - B[:, 1, 0]], 1)
        L = (m[:, None] * (np.cross(X, V) - eps)).sum(0)
    else:
        L = np.array([(m * (X[:, 0] * V[:, 1] - X[:, 1] * V[:, 0] - (B[:, 0, 1] - B[:, 1, 0]))).sum(), 0.0, 0.0])
    Dp_inv = 4.0 / dx ** 2                       # quadratic B-spline Dp^-1, one entry per axis
    ke = 0.5 * (m * (V ** 2).sum(1)).sum() + 0.5 * (m * (B ** 2 * Dp_inv[None, None, :]).sum((1, 2))).sum()
    speed = np.sqrt((V ** 2).sum(1))
    xi = 6.0 * np.sqrt(d) / dx.max()
    affine = speed + np.sqrt((B ** 2).sum((1, 2))) * xi
    mom = np.zeros(3)
    mom[:d] = (m[:, None] * V).sum(0)
    return {"mass": m.sum(), "momentum": mom, "angular_momentum": L, "kinetic_energy": ke,
            "max_speed": speed.max(initial=0.0), "max_affine_speed": affine.max(initial=0.0), "count": int(ok.sum())}


def compute_dt(max_affine_speed, dx_min, cfl, max_dt):
    """MPM_DRIVER::Compute_Dt (Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.cpp:1098-1105)."""
    critical = cfl * dx_min / max_dt
    v = max_affine_speed
    return cfl * dx_min / v if v > critical else max_dt
