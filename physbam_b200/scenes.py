"""Seeded synthetic MPM scenes and the binary scene-file format.

The reference has no public dataset for its MPM path: scenes are built in C++
by `Projects/mpm/STANDARD_TESTS_BASE.cpp` (seeding, Lame parameters l.567-586,
walls l.487-511).  This module builds the benchmark scenes the same way, from
one numpy seed, so the CUDA path, the CPU oracle and the reference's own
driver all start from bit-identical particle arrays:

* particles are seeded ``ppc`` per cell, each uniform in its cell, and kept
  when inside the body (box or sphere);
* ``volume = dx^d / ppc``, ``mass = density * volume``, ``F = I``, ``B = 0``;
* ``mu = E / (2 (1 + nu))``, ``lambda = E nu / ((1 + nu)(1 - 2 nu))`` per
  particle, as `STANDARD_TESTS_BASE::Set_Lame_On_Particles` computes them;
* walls are RANGE boxes over the domain thickened by ``dx (2 ghost + 1)``,
  cut at ``inset`` from one face, as `STANDARD_TESTS_BASE::Add_Walls` builds
  them.

Layout follows `MPM_PARTICLES` (`Hybrid_Methods/Examples_And_Drivers/
MPM_PARTICLES.h:18-44`): ``X, V`` are (N, d); ``F, B`` are (N, d, d) stored
column-major per particle, i.e. ``F[p].T`` in numpy row-major terms (the
reference's ``MATRIX<T,3>`` keeps ``x[i + d*j]``, `Core/Matrices/MATRIX_3X3.h:115-119`).
Arrays here are kept as plain (N, d, d) with ``F[p][i, j]`` = row i, col j;
the writer transposes when it serialises.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional, Sequence

import numpy as np

COROTATED = 0
NEO_HOOKEAN = 1
HENCKY = 2          # ST_VENANT_KIRCHHOFF_HENCKY_STRAIN (the sand scenes' elastic model)

STICK = 0
SLIP = 1
SEPARATE = 2

BOX = 0
PLANE = 1
SPHERE = 2          # a = center, b[0] = radius

GHOST = 3


@dataclasses.dataclass
class Motion:
    """A collision object moving with a constant twist: `func_frame(t)` =
    FRAME(center + linear t, ROTATION::From_Rotation_Vector(angular t)) and
    `func_twist(t)` = TWIST(linear, angular), the form of the reference's rotating
    and translating objects (e.g. `Projects/mpm/STANDARD_TESTS_3D.cpp:1560-1561`).
    The object's geometry is then given about the origin of its own frame.  In 2D
    ``angular`` has one entry (the spin)."""
    center: Sequence[float]
    linear: Sequence[float]
    angular: Sequence[float]

    def state(self, dim, t):
        """(translation, unit quaternion w, x, y, z -- in 2D (cos, sin, 0, 0) --, linear, angular) at t."""
        tr = [float(self.center[k]) + float(self.linear[k]) * t for k in range(dim)]
        if dim == 2:
            th = float(self.angular[0]) * t
            q = [np.cos(th), np.sin(th), 0.0, 0.0]
        else:
            r = np.asarray(self.angular[:3], float) * t
            th = float(np.sqrt(r @ r))
            if th > 0:
                q = [np.cos(th / 2)] + list(np.sin(th / 2) / th * r)
            else:
                q = [1.0, 0.0, 0.0, 0.0]
        return tr, q, list(self.linear[:dim]), list(self.angular[:3 if dim == 3 else 1])


@dataclasses.dataclass
class CollisionObject:
    """A collision object (`Hybrid_Methods/Collisions/MPM_COLLISION_OBJECT.h:13-37`).

    ``kind`` BOX: ``a`` = min corner, ``b`` = max corner (`Core/Math_Tools/RANGE.cpp:37-63`).
    ``kind`` PLANE: ``a`` = unit normal, ``b`` = a point on the plane
    (`Geometry/Basic_Geometry/PLANE.h:52-63`); inside is behind the normal.
    ``motion`` (optional): the object moves, its geometry given in its own frame.
    """
    kind: int
    type: int
    friction: float
    a: Sequence[float]
    b: Sequence[float]
    motion: Optional[Motion] = None


PLASTICITY_NONE, PLASTICITY_CLAMP, PLASTICITY_DRUCKER_PRAGER = 0, 1, 2


@dataclasses.dataclass
class Plasticity:
    """Snow-like plasticity, MPM_PLASTICITY_CLAMP (`Hybrid_Methods/Forces/MPM_PLASTICITY_CLAMP.cpp:28-45`):
    the singular values of F are clamped to [1 - theta_c, 1 + theta_s] after each G2P, the
    clamped-off part goes to the plastic deformation Fp, and mu, lambda harden as
    mu0 exp(min(max_hardening, hardening_factor (1 - det Fp)))."""
    kind: int = PLASTICITY_CLAMP
    theta_c: float = 2.5e-2
    theta_s: float = 7.5e-3
    max_hardening: float = 5.0
    hardening_factor: float = 10.0


@dataclasses.dataclass
class DruckerPrager:
    """Sand plasticity, MPM_DRUCKER_PRAGER (`Hybrid_Methods/Forces/MPM_DRUCKER_PRAGER.cpp:60-125`):
    the Hencky strain is projected onto the Drucker-Prager cone after each G2P.  Friction
    angle (degrees) a0 + (a1 q - a4) exp(-a3 q) of the accumulated plastic deformation q
    (the Mast et al. hardening of `Update_Hardening`); `cohesion` is the initial sigma_Y
    (`Initialize_Particles`); `use_vc` keeps the volume-correction term."""
    kind: int = PLASTICITY_DRUCKER_PRAGER
    a0: float = 35.0
    a1: float = 0.0
    a3: float = 0.2
    a4: float = 10.0
    cohesion: float = 0.0
    use_vc: bool = True

    @classmethod
    def friction_angle(cls, phi_F: float, cohesion: float = 0.0, use_vc: bool = True) -> "DruckerPrager":
        """A constant friction angle phi_F (degrees), no hardening: the reference's
        Add_Drucker_Prager(E, nu, phi_F) (`Projects/mpm/STANDARD_TESTS_BASE.cpp:437-441`)."""
        return cls(a0=phi_F, a1=0.0, a3=0.0, a4=0.0, cohesion=cohesion, use_vc=use_vc)

    @classmethod
    def mast_case(cls, case: int, use_vc: bool = True) -> "DruckerPrager":
        """The hardening constants (a0, a1, a3, a4) of Mast et al.'s cases 0-9, as
        Add_Drucker_Prager_Case selects them (`Projects/mpm/STANDARD_TESTS_BASE.cpp:445-464`)."""
        a0, a1, a3, a4 = (float(x) for x in MAST_CASES[case])
        return cls(a0=a0, a1=a1, a3=a3, a4=a4, use_vc=use_vc)


# (a0, a1, a3, a4) per case of the sand hardening study the reference's scenes draw on
MAST_CASES = ((35, 0, 0.2, 10), (35, 4, 0.29, 10), (35, 9, 0.3, 10), (35, 13, 0.27, 10), (35, 0, 0.2, 6.57),
              (35, 0, 0.2, 3.33), (35, 0, 0.2, 0), (38.33, 0, 0.2, 13.33), (41.67, 0, 0.2, 16.67), (45, 0, 0.2, 20))


def plastic_keys(pl) -> tuple:
    """Per-particle plastic state a dump / fixture carries for plasticity `pl`."""
    if pl is None:
        return ()
    if pl.kind == PLASTICITY_CLAMP:
        return ("Fp", "mu", "lam")
    return ("Fp", "pdef", "rho_F", "cohesion", "vc")


def plastic_params(pl) -> list:
    """The plasticity as the flat list the scene file and the fixtures hold (kind first)."""
    if pl.kind == PLASTICITY_CLAMP:
        return [pl.kind, pl.theta_c, pl.theta_s, pl.max_hardening, pl.hardening_factor]
    return [pl.kind, pl.a0, pl.a1, pl.a3, pl.a4, pl.cohesion, 1.0 if pl.use_vc else 0.0]


def plastic_from_params(p):
    p = [float(x) for x in p]
    if int(p[0]) == PLASTICITY_CLAMP:
        return Plasticity(int(p[0]), *p[1:5])
    return DruckerPrager(int(p[0]), *p[1:6], bool(p[6]))


@dataclasses.dataclass
class Implicit:
    """Backward-Euler force solve instead of symplectic Euler (the reference's default:
    `MPM_DRIVER::Apply_Forces`, `MPM_DRIVER.cpp:1024-1048`): Newton's method on
    `MPM_OBJECTIVE` with CG, tolerance `newton_tolerance * dt`, the Krylov tolerance
    relative (`MPM_EXAMPLE.h:119-122` defaults)."""
    newton_tolerance: float = 1.0
    newton_iterations: int = 100
    solver_tolerance: float = 0.5
    solver_iterations: int = 1000


@dataclasses.dataclass
class DtControl:
    """Adaptive substeps as MPM_DRIVER::Simulate_To_Frame takes them (`MPM_DRIVER.cpp:161-201`):
    dt = Compute_Dt (the affine CFL bound, `cfl`) clamped to [min_dt, max_dt] and fitted to
    the frame end, then Reduce_Dt after the forces (l.519-545): the strong CFL of
    Grid_To_Particle_Limit_Dt (`cfl_F` on the change of F, `cfl` on the displacement) and
    the sound-speed CFL (`cfl_sound`), each when switched on (`MPM_EXAMPLE.h:84-115`)."""
    frame_dt: float = 1.0 / 24
    cfl: float = 1.0
    min_dt: float = 0.0
    max_dt: float = 1.0 / 24
    strong_cfl: bool = False
    cfl_F: float = 0.5
    sound_cfl: bool = False
    cfl_sound: float = 0.9


BC_FREE, BC_SLIP, BC_NOSLIP, BC_SEP = 0, 1, 2, 3


@dataclasses.dataclass
class Reflection:
    """Reflection boundary conditions on the domain faces (MPM_EXAMPLE::reflection_bc,
    side_bc_type per side -x +x -y +y -z +z; `MPM_DRIVER.cpp:307-446`), as
    `STANDARD_TESTS_BASE::Add_Walls` sets them with -use_reflect (slip, separate or
    no-slip walls; `full` is -use_reflect_friction, with `friction`)."""
    side_type: Sequence[int] = (BC_SLIP, BC_SLIP, BC_NOSLIP, BC_FREE, BC_SLIP, BC_SLIP)
    friction: float = 0.0
    full: bool = False


@dataclasses.dataclass
class Penalty:
    """Penalty collision objects: one IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES per object, as
    `STANDARD_TESTS_BASE::Add_Penalty_Collision_Object` adds them with -use_penalty_collisions
    (`Projects/mpm/STANDARD_TESTS_BASE.cpp:555-563`).  A particle within `separation` of an
    object (phi <= separation, x = separation - phi) is pushed along the object's normal with
    the force 3 stiffness x^2; the implicit solve adds its energy stiffness x^3 and Hessian.
    Defaults as STANDARD_TESTS_BASE (stiffness 1e4, separation 1e-4).  The objects'
    `type` is not used; `friction` is the force's coefficient_of_friction, which the MPM
    substep does not apply."""
    objects: List[CollisionObject]
    stiffness: float = 1e4
    separation: float = 1e-4


@dataclasses.dataclass
class Scene:
    name: str
    dim: int
    counts: Sequence[int]
    domain_min: Sequence[float]
    domain_max: Sequence[float]
    model: int
    gravity: Sequence[float]
    dt: float
    nsteps: int
    objects: List[CollisionObject]
    X: np.ndarray
    V: np.ndarray
    F: np.ndarray
    B: np.ndarray
    mass: np.ndarray
    volume: np.ndarray
    mu: np.ndarray
    lam: np.ndarray
    plasticity: Optional[Plasticity] = None
    implicit: Optional[Implicit] = None
    dt_control: Optional[DtControl] = None     # set: nsteps counts frames of frame_dt
    reflection: Optional[Reflection] = None
    penalty: Optional[Penalty] = None
    models: Optional[np.ndarray] = None        # per-particle constitutive model (None: `model` for all)
    plastic_mask: Optional[np.ndarray] = None  # the particles the plasticity acts on (None: all)
    # a force the library does not model, added by the caller between P2G and the grid
    # update (mpm_add_grid_forces): this vector at every node with mass
    node_force: Optional[Sequence[float]] = None

    @property
    def n(self) -> int:
        return int(self.X.shape[0])

    @property
    def dx(self) -> float:
        return float((self.domain_max[0] - self.domain_min[0]) / self.counts[0])

    def copy(self) -> "Scene":
        return dataclasses.replace(
            self, X=self.X.copy(), V=self.V.copy(), F=self.F.copy(), B=self.B.copy(),
            mass=self.mass.copy(), volume=self.volume.copy(), mu=self.mu.copy(), lam=self.lam.copy(),
            objects=list(self.objects))

    def subset(self, idx) -> "Scene":
        return dataclasses.replace(
            self, X=self.X[idx].copy(), V=self.V[idx].copy(), F=self.F[idx].copy(),
            B=self.B[idx].copy(), mass=self.mass[idx].copy(), volume=self.volume[idx].copy(),
            mu=self.mu[idx].copy(), lam=self.lam[idx].copy(), objects=list(self.objects),
            models=None if self.models is None else self.models[idx].copy(),
            plastic_mask=None if self.plastic_mask is None else self.plastic_mask[idx].copy())


def lame(E, nu):
    """`STANDARD_TESTS_BASE::Set_Lame_On_Particles` (Projects/mpm/STANDARD_TESTS_BASE.cpp:567-586)."""
    E = np.asarray(E, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    return mu, lam


def walls(dim, counts, dmin, dmax, flags, type_, friction, inset):
    """RANGE walls as `STANDARD_TESTS_BASE::Add_Walls` builds them (STANDARD_TESTS_BASE.cpp:487-511).

    Bit ``2a+s`` of ``flags`` selects one wall; the reference puts bit ``2a+1``
    on the LOW side of axis ``a`` and bit ``2a`` on the high side.
    """
    dx = (np.asarray(dmax, float) - np.asarray(dmin, float)) / np.asarray(counts, float)
    lo = np.asarray(dmin, float) - dx * (GHOST * 2 + 1)
    hi = np.asarray(dmax, float) + dx * (GHOST * 2 + 1)
    out = []
    for a in range(dim):
        for s in range(2):
            if flags & (1 << (a * 2 + s)):
                wlo, whi = lo.copy(), hi.copy()
                if s:
                    whi[a] = dmin[a] + inset
                else:
                    wlo[a] = dmax[a] - inset
                out.append(CollisionObject(BOX, type_, friction, wlo.tolist(), whi.tolist()))
    return out


def _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc, inside):
    """Jitter ``ppc`` particles uniformly in every cell overlapping [lo, hi]; keep those ``inside``."""
    c0 = np.maximum(np.floor((np.asarray(lo) - dmin) / dx).astype(np.int64), 0)
    c1 = np.minimum(np.ceil((np.asarray(hi) - dmin) / dx).astype(np.int64), np.asarray(counts))
    axes = [np.arange(c0[a], c1[a]) for a in range(dim)]
    cells = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, dim)
    n = cells.shape[0] * ppc
    jitter = rng.random((n, dim))
    X = dmin + (np.repeat(cells, ppc, axis=0) + jitter) * dx
    return X[inside(X)]


def _finish(name, dim, counts, dmin, dmax, model, gravity, dt, nsteps, objects, X, V, E, nu, density, ppc):
    dx = (dmax[0] - dmin[0]) / counts[0]
    n = X.shape[0]
    vol = np.full(n, dx ** dim / ppc)
    mass = density * vol
    mu, lam = lame(np.broadcast_to(E, (n,)), np.broadcast_to(nu, (n,)))
    F = np.broadcast_to(np.eye(dim), (n, dim, dim)).copy()
    B = np.zeros((n, dim, dim))
    return Scene(name, dim, list(counts), list(map(float, dmin)), list(map(float, dmax)), model,
                 list(map(float, gravity)), float(dt), int(nsteps), objects,
                 np.ascontiguousarray(X, dtype=np.float64), np.ascontiguousarray(V, dtype=np.float64),
                 F, B, mass, vol, np.ascontiguousarray(mu), np.ascontiguousarray(lam))


def block_2d(seed=1234, G=64, ppc=4, E=1e4, nu=0.3, density=1000.0, dt=1e-4, nsteps=100):
    """2D elastic block: 0.25x0.25 centred (0.5, 0.6), sticky ground at y=0.05 (64^2, 4 ppc)."""
    rng = np.random.default_rng(seed)
    dim, counts = 2, [G, G]
    dmin, dmax = np.zeros(2), np.ones(2)
    dx = 1.0 / G
    lo, hi = np.array([0.375, 0.475]), np.array([0.625, 0.725])
    X = _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc,
                    lambda P: np.all((P >= lo) & (P < hi), axis=1))
    V = np.zeros_like(X)
    objects = walls(dim, counts, dmin, dmax, 1 << 3, STICK, 0.0, 0.05)
    return _finish("block2d", dim, counts, dmin, dmax, COROTATED, [0, -9.8], dt, nsteps, objects,
                   X, V, E, nu, density, ppc)


def spheres_3d(seed=1234, G=128, ppc=8, E=5e4, nu=0.35, density=1000.0, dt=5e-5, nsteps=200,
               radius=0.12, model=NEO_HOOKEAN):
    """Two colliding spheres (r=0.12 at x=0.35/0.65, v=+-2 m/s), slip walls, NEO_HOOKEAN (128^3, 8 ppc)."""
    rng = np.random.default_rng(seed)
    dim, counts = 3, [G, G, G]
    dmin, dmax = np.zeros(3), np.ones(3)
    dx = 1.0 / G
    Xs, Vs = [], []
    for c, v in (((0.35, 0.5, 0.5), 2.0), ((0.65, 0.5, 0.5), -2.0)):
        c = np.asarray(c)
        X = _seed_cells(rng, dim, counts, dmin, dx, c - radius, c + radius, ppc,
                        lambda P, c=c: np.sum((P - c) ** 2, axis=1) < radius * radius)
        Xs.append(X)
        V = np.zeros_like(X)
        V[:, 0] = v
        Vs.append(V)
    X, V = np.concatenate(Xs), np.concatenate(Vs)
    objects = walls(dim, counts, dmin, dmax, 63, SLIP, 0.0, 0.05)
    return _finish("spheres3d", dim, counts, dmin, dmax, model, [0, -9.8, 0], dt, nsteps, objects,
                   X, V, E, nu, density, ppc)


def dam_3d(seed=1234, G=256, ppc=8, E=2e5, nu=0.4, density=1000.0, dt=2e-5, nsteps=100, sigma=0.2):
    """Dam-break block [0.05,0.45]x[0.05,0.8]x[0.05,0.95], E log-normal (sigma 0.2), sticky floor, slip walls."""
    rng = np.random.default_rng(seed)
    dim, counts = 3, [G, G, G]
    dmin, dmax = np.zeros(3), np.ones(3)
    dx = 1.0 / G
    lo, hi = np.array([0.05, 0.05, 0.05]), np.array([0.45, 0.8, 0.95])
    X = _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc,
                    lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = E * np.exp(sigma * rng.standard_normal(X.shape[0]))
    V = np.zeros_like(X)
    objects = walls(dim, counts, dmin, dmax, 1 << 3, STICK, 0.0, 0.05)
    objects += walls(dim, counts, dmin, dmax, 63 & ~(1 << 3), SLIP, 0.0, 0.05)
    return _finish("dam3d", dim, counts, dmin, dmax, COROTATED, [0, -9.8, 0], dt, nsteps, objects,
                   X, V, Ep, nu, density, ppc)


def cube_3d(seed=1234, G=64, ppc=8, side=0.3, nu=0.3, density=1000.0, dt=1e-4, nsteps=64,
            v0=(1.0, 0.5, 0.0), E_range=(5e3, 5e4), model=COROTATED):
    """Differentiable cube: side 0.3 centred (0.5,0.5,0.5), E log-uniform, v0 = (1, .5, 0) (64^3, 8 ppc).

    Also returns the seeded target point in [0.3, 0.7]^3 as ``scene.target``.
    """
    rng = np.random.default_rng(seed)
    dim, counts = 3, [G, G, G]
    dmin, dmax = np.zeros(3), np.ones(3)
    dx = 1.0 / G
    c = np.array([0.5, 0.5, 0.5])
    lo, hi = c - side / 2, c + side / 2
    X = _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc,
                    lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = np.exp(rng.uniform(np.log(E_range[0]), np.log(E_range[1]), X.shape[0]))
    V = np.broadcast_to(np.asarray(v0, float), X.shape).copy()
    s = _finish("cube3d", dim, counts, dmin, dmax, model, [0, -9.8, 0], dt, nsteps, [],
                X, V, Ep, nu, density, ppc)
    s.target = rng.uniform(0.3, 0.7, 3)
    return s


def batch_scenes(seed=1234, count=256, ppc_range=(4, 8), nsteps=100, dt=1e-4):
    """Independent boxes: grid side from {32,48,64,96}, box side U[0.1,0.4], |v|<=2, per-scene model."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        G = int(rng.choice([32, 48, 64, 96]))
        ppc = int(rng.integers(ppc_range[0], ppc_range[1] + 1))
        size = rng.uniform(0.1, 0.4, 3)
        lo = rng.uniform(0.1, 0.9 - size)
        hi = lo + size
        v = rng.normal(size=3)
        v *= rng.uniform(0, 2.0) / max(np.linalg.norm(v), 1e-12)
        E = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        nu = float(rng.uniform(0.2, 0.45))
        model = int(rng.integers(0, 2))
        srng = np.random.default_rng([seed, s])
        dmin = np.zeros(3)
        X = _seed_cells(srng, 3, [G] * 3, dmin, 1.0 / G, lo, hi, ppc,
                        lambda P, lo=lo, hi=hi: np.all((P >= lo) & (P < hi), axis=1))
        V = np.broadcast_to(v, X.shape).copy()
        out.append(_finish("batch%d" % s, 3, [G] * 3, dmin, np.ones(3), model, [0, -9.8, 0], dt, nsteps,
                           [], X, V, E, nu, 1000.0, ppc))
    return out


def small_3d(seed=7, G=16, ppc=8, model=COROTATED, nsteps=20, dt=1e-4, E=(2e4, 8e4), nu=0.3,
             v=(1.5, -0.5, 0.75), with_walls=True, friction=0.0):
    """A small 3D scene for golden fixtures: a box with a rotating velocity field, walls, per-particle E."""
    rng = np.random.default_rng(seed)
    dim, counts = 3, [G, G, G]
    dmin, dmax = np.zeros(3), np.ones(3)
    dx = 1.0 / G
    lo, hi = np.array([0.2, 0.12, 0.3]), np.array([0.6, 0.5, 0.7])
    X = _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc,
                    lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = np.exp(rng.uniform(np.log(E[0]), np.log(E[1]), X.shape[0]))
    c = (lo + hi) / 2
    V = np.asarray(v, float) + 4.0 * np.cross(np.array([0.3, 1.0, -0.2]), X - c)
    objects = []
    if with_walls:
        objects = walls(dim, counts, dmin, dmax, 1 << 3, STICK, 0.0, 0.15)
        objects += walls(dim, counts, dmin, dmax, 63 & ~(1 << 3), SLIP, friction, 0.2)
    s = _finish("small3d", dim, counts, dmin, dmax, model, [0, -9.8, 0], dt, nsteps, objects,
                X, V, Ep, nu, 1000.0, ppc)
    # start from a deformed, slightly sheared state so the stress is non-trivial on step 0
    A = np.eye(3) + 0.08 * rng.standard_normal((3, 3))
    s.F = np.broadcast_to(A, s.F.shape).copy()
    s.B = 0.5 * rng.standard_normal(s.B.shape) * dx
    return s


def small_2d(seed=11, G=16, ppc=4, model=COROTATED, nsteps=20, dt=1e-4, friction=0.3):
    """A small 2D scene for golden fixtures: block falling onto a sticky floor with slip side walls."""
    rng = np.random.default_rng(seed)
    dim, counts = 2, [G, G]
    dmin, dmax = np.zeros(2), np.ones(2)
    dx = 1.0 / G
    lo, hi = np.array([0.25, 0.2]), np.array([0.7, 0.55])
    X = _seed_cells(rng, dim, counts, dmin, dx, lo, hi, ppc,
                    lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = np.exp(rng.uniform(np.log(1e4), np.log(5e4), X.shape[0]))
    V = np.column_stack([np.full(X.shape[0], 1.0), -2.0 + 3.0 * (X[:, 0] - 0.5)])
    objects = walls(dim, counts, dmin, dmax, 1 << 3, STICK, 0.0, 0.2)
    objects += walls(dim, counts, dmin, dmax, 3, SLIP, friction, 0.2)
    s = _finish("small2d", dim, counts, dmin, dmax, model, [0, -9.8], dt, nsteps, objects,
                X, V, Ep, 0.3, 1000.0, ppc)
    A = np.eye(2) + 0.1 * rng.standard_normal((2, 2))
    s.F = np.broadcast_to(A, s.F.shape).copy()
    s.B = 0.5 * rng.standard_normal(s.B.shape) * dx
    return s


def small_snow_3d(seed=21, G=16, nsteps=20, dt=1e-4, model=COROTATED):
    """A small snow block thrown against a sticky floor: small_3d with clamped plasticity
    (the initial shear already pushes singular values past the clamp)."""
    s = small_3d(seed=seed, G=G, model=model, nsteps=nsteps, dt=dt, E=(1e4, 4e4), v=(0.5, -3.0, 0.25))
    s.name = "smallsnow3d"
    s.plasticity = Plasticity()
    return s


def small_snow_2d(seed=23, G=16, nsteps=20, dt=1e-4):
    s = small_2d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.name = "smallsnow2d"
    s.plasticity = Plasticity(theta_c=2e-2, theta_s=6e-3, max_hardening=4.0, hardening_factor=8.0)
    return s


def small_3d_implicit(seed=41, G=16, nsteps=10, dt=1e-3):
    """small_3d with the backward-Euler Newton solve at a step 10x the explicit one
    (stick floor, slip walls with friction 0.3, corotated)."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt, friction=0.3)
    s.name = "small3dimplicit"
    s.implicit = Implicit()
    return s


def small_2d_implicit(seed=43, G=16, nsteps=10, dt=1e-3):
    """small_2d, neo-Hookean, with the backward-Euler Newton solve."""
    s = small_2d(seed=seed, G=G, nsteps=nsteps, dt=dt, model=NEO_HOOKEAN)
    s.name = "small2dimplicit"
    s.implicit = Implicit()
    return s


def small_3d_sphere(seed=71, G=16, nsteps=20, dt=1e-4, implicit=False):
    """small_3d thrown at a spherical obstacle (separate, friction 0.3) as well as the walls."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt, friction=0.2, v=(3.0, -1.0, 1.5))
    s.name = "small3dsphere"
    s.objects = s.objects + [CollisionObject(SPHERE, SEPARATE, 0.3, [0.62, 0.3, 0.55], [0.12, 0, 0])]
    if implicit:
        s.name = "small3dsphereimplicit"
        s.dt = 1e-3
        s.nsteps = 8
        s.implicit = Implicit()
    return s


def small_2d_sphere(seed=73, G=16, nsteps=20, dt=1e-4):
    """small_2d with a sticky circle inside the block (its nodes are held at rest)."""
    s = small_2d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.name = "small2dsphere"
    s.objects = s.objects + [CollisionObject(SPHERE, STICK, 0.0, [0.45, 0.3], [0.08, 0])]
    return s


def small_3d_penalty(seed=81, G=16, nsteps=20, dt=1e-4, implicit=False):
    """small_3d with penalty collision objects overlapping the block: a ball on its +x side,
    a slab under its floor and a plane through its -z side (the walls stay as ordinary
    collision objects).  Particles start up to 7 cm deep in the ball, so the penalty forces,
    and in the implicit solve their Hessians with the ball's curvature, are far from zero."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt, friction=0.2, v=(1.0, -1.5, 0.5))
    s.name = "small3dpenalty"
    s.penalty = Penalty([CollisionObject(SPHERE, SLIP, 0.3, [0.62, 0.33, 0.52], [0.09, 0, 0]),
                         CollisionObject(BOX, SLIP, 0.0, [-1.0, -1.0, -1.0], [2.0, 0.135, 2.0]),
                         CollisionObject(PLANE, SLIP, 0.0, [0.0, 0.0, 1.0], [0.0, 0.0, 0.31])])
    if implicit:
        s.name = "small3dpenaltyimplicit"
        s.dt = 1e-3
        s.nsteps = 8
        s.implicit = Implicit()
    return s


def small_2d_penalty(seed=83, G=16, nsteps=20, dt=1e-4):
    """small_2d with a penalty circle on the block's +x side and a penalty slab under it,
    with stiffness 2e4 and a wider separation (5e-3)."""
    s = small_2d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.name = "small2dpenalty"
    s.penalty = Penalty([CollisionObject(SPHERE, SLIP, 0.0, [0.7, 0.4], [0.1, 0]),
                         CollisionObject(BOX, SLIP, 0.0, [-1.0, -1.0], [2.0, 0.215])], stiffness=2e4, separation=5e-3)
    return s


def small_3d_node_force(seed=121, G=16, nsteps=20, dt=1e-4, force=(0.05, 0.1, -0.025)):
    """The small 3D scene with a constant extra force at every node with mass (a force the
    library does not model, handed in through mpm_add_grid_forces)."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.node_force = list(force)
    return s


def small_3d_moving(seed=91, G=16, nsteps=20, dt=1e-4, implicit=False):
    """small_3d with two moving collision objects: a sticky paddle (a box in its own frame)
    that starts inside the block's +x face and turns about y while it pushes in, and a
    separating ball that comes down on the block's top (the walls stay static)."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt, friction=0.2, v=(0.5, -0.5, 0.25))
    s.name = "small3dmoving"
    s.objects = s.objects + [
        CollisionObject(BOX, STICK, 0.0, [-0.04, -0.1, -0.12], [0.04, 0.1, 0.12],
                        motion=Motion([0.62, 0.31, 0.5], [-4.0, 0.5, 0.0], [0.0, 6.0, 1.0])),
        CollisionObject(SPHERE, SEPARATE, 0.3, [0.0, 0.0, 0.0], [0.08, 0, 0],
                        motion=Motion([0.35, 0.56, 0.45], [0.5, -5.0, 0.0], [0.0, 0.0, 0.0]))]
    if implicit:
        s.name = "small3dmovingimplicit"
        s.dt = 1e-3
        s.nsteps = 8
        s.implicit = Implicit()
    return s


def small_2d_moving(seed=93, G=16, nsteps=20, dt=1e-4):
    """small_2d with a spinning sticky paddle inside the block's +x side and a slip box
    sliding along its top with friction."""
    s = small_2d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.name = "small2dmoving"
    s.objects = s.objects + [
        CollisionObject(BOX, STICK, 0.0, [-0.03, -0.1], [0.03, 0.1], motion=Motion([0.68, 0.38], [-3.0, 0.0], [8.0])),
        CollisionObject(BOX, SLIP, 0.5, [-0.1, -0.03], [0.1, 0.03], motion=Motion([0.45, 0.57], [4.0, -2.0], [0.0]))]
    return s


def small_3d_mixed(seed=101, G=16, nsteps=20, dt=1e-4, implicit=False):
    """small_3d with two materials: COROTATED_FIXED for x < 0.4, NEO_HOOKEAN beyond (the
    reference's several MPM_FINITE_ELEMENTS forces over particle subsets)."""
    s = small_3d(seed=seed, G=G, nsteps=nsteps, dt=dt, friction=0.2, E=(2e4, 2e5))
    s.name = "small3dmixed"
    s.models = np.where(s.X[:, 0] < 0.4, COROTATED, NEO_HOOKEAN).astype(np.uint8)
    if implicit:
        s.name = "small3dmixedimplicit"
        s.dt = 1e-3
        s.nsteps = 8
        s.implicit = Implicit()
    return s


def small_sand_water_3d(seed=111, G=16, nsteps=20, dt=1e-4):
    """A sand block (Hencky + Drucker-Prager, x >= 0.4) beside an elastic one (COROTATED_FIXED,
    no plasticity): two MPM_FINITE_ELEMENTS forces over particle subsets and the plasticity over
    the sand alone, the structure of the reference's sand-and-water scenes."""
    s = small_sand_3d(seed=seed, G=G, nsteps=nsteps, dt=dt)
    s.name = "smallsandwater3d"
    sand = s.X[:, 0] >= 0.4
    s.models = np.where(sand, HENCKY, COROTATED).astype(np.uint8)
    s.plastic_mask = sand.astype(np.uint8)
    return s


def small_3d_adaptive(seed=51, G=16, nframes=3):
    """A stiff small_3d (E 2e6..8e6) run frame by frame as Simulate_To_Frame does,
    with the strong and the sound-speed CFL on: the sound speed shortens most steps."""
    s = small_3d(seed=seed, G=G, nsteps=nframes, E=(2e6, 8e6))
    s.name = "small3dadaptive"
    s.dt_control = DtControl(frame_dt=1e-3, cfl=0.5, min_dt=1e-7, max_dt=5e-4, strong_cfl=True, cfl_F=0.01,
                             sound_cfl=True, cfl_sound=0.5)
    return s


def small_2d_adaptive(seed=53, G=16, nframes=3):
    """small_2d run frame by frame with the strong CFL only (a tight cfl_F)."""
    s = small_2d(seed=seed, G=G, nsteps=nframes)
    s.name = "small2dadaptive"
    s.dt_control = DtControl(frame_dt=2e-3, cfl=0.5, min_dt=1e-7, max_dt=1e-3, strong_cfl=True, cfl_F=0.002)
    return s


def small_3d_reflect(seed=61, G=16, nsteps=20, dt=1e-4):
    """A block in the domain's low corner thrown at the faces, with reflection
    boundary conditions instead of wall objects: slip on x, no-slip floor, a free
    top, separate on -z and slip on +z; particles cross the faces and are mirrored."""
    rng = np.random.default_rng(seed)
    dim, counts = 3, [G, G, G]
    dmin, dmax = np.zeros(3), np.ones(3)
    lo, hi = np.array([0.001, 0.002, 0.0015]), np.array([0.3, 0.3, 0.28])
    X = _seed_cells(rng, dim, counts, dmin, 1.0 / G, lo, hi, 8, lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = np.exp(rng.uniform(np.log(2e4), np.log(8e4), X.shape[0]))
    V = np.tile(np.array([-8.0, -10.0, -6.0]), (X.shape[0], 1)) + 2.0 * np.cross(np.array([0.2, 1.0, 0.3]), X - 0.15)
    s = _finish("small3dreflect", dim, counts, dmin, dmax, COROTATED, [0, -9.8, 0], dt, nsteps, [], X, V, Ep, 0.3,
                1000.0, 8)
    s.F = np.eye(3) + 0.05 * rng.standard_normal((s.n, 3, 3))
    s.B = 0.3 * rng.standard_normal(s.B.shape) / G
    s.reflection = Reflection(side_type=(BC_SLIP, BC_SLIP, BC_NOSLIP, BC_FREE, BC_SEP, BC_SLIP))
    return s


def small_2d_reflect(seed=63, G=16, nsteps=20, dt=1e-4, full=True):
    """A 2D block against the low corner with frictional reflection (separate walls,
    friction 0.4, -use_reflect_friction)."""
    rng = np.random.default_rng(seed)
    dim, counts = 2, [G, G]
    dmin, dmax = np.zeros(2), np.ones(2)
    lo, hi = np.array([0.001, 0.0015]), np.array([0.35, 0.3])
    X = _seed_cells(rng, dim, counts, dmin, 1.0 / G, lo, hi, 4, lambda P: np.all((P >= lo) & (P < hi), axis=1))
    Ep = np.exp(rng.uniform(np.log(1e4), np.log(5e4), X.shape[0]))
    V = np.column_stack([np.full(X.shape[0], -8.0), -10.0 + 2.0 * (X[:, 0] - 0.2)])
    s = _finish("small2dreflect", dim, counts, dmin, dmax, NEO_HOOKEAN, [0, -9.8], dt, nsteps, [], X, V, Ep, 0.3,
                1000.0, 4)
    s.F = np.eye(2) + 0.05 * rng.standard_normal((s.n, 2, 2))
    s.reflection = Reflection(side_type=(BC_SEP, BC_SLIP, BC_SEP, BC_FREE), friction=0.4, full=full)
    return s


def small_sand_3d(seed=31, G=16, nsteps=20, dt=1e-4):
    """A small sand block (St. Venant-Kirchhoff Hencky + Drucker-Prager with Mast hardening)
    thrown against a sticky floor; a random initial F per particle, compressed by 3 % for
    x > 0.4, starts particles in every branch of the return mapping (elastic, cone, tip)."""
    s = small_3d(seed=seed, G=G, model=HENCKY, nsteps=nsteps, dt=dt, E=(1e5, 3e5), v=(0.5, -3.0, 0.25))
    s.name = "smallsand3d"
    rng = np.random.default_rng(seed + 1)
    s.F = np.eye(3) + 0.04 * rng.standard_normal((s.n, 3, 3))
    s.F[s.X[:, 0] > 0.4] *= 0.97
    s.plasticity = DruckerPrager(a0=35.0, a1=9.0, a3=0.3, a4=10.0)
    return s


def small_sand_2d(seed=33, G=16, nsteps=20, dt=1e-4):
    """The 2D sand block, with cohesion (sigma_Y = 100 Pa) and no volume correction."""
    s = small_2d(seed=seed, G=G, model=HENCKY, nsteps=nsteps, dt=dt)
    s.name = "smallsand2d"
    s.mu *= 5.0
    s.lam *= 5.0
    rng = np.random.default_rng(seed + 1)
    s.F = np.eye(2) + 0.04 * rng.standard_normal((s.n, 2, 2))
    s.F[s.X[:, 0] > 0.5] *= 0.97
    s.plasticity = DruckerPrager(cohesion=100.0, use_vc=False)
    return s


def sand_3d(seed=1234, G=128, ppc=8, E=3.537e5, nu=0.3, density=2200.0, dt=5e-5, nsteps=200):
    """Two balls of sand colliding on the 128^3 grid (the spheres_3d geometry): St. Venant-Kirchhoff
    Hencky with Drucker-Prager (Mast et al. case 2 hardening: 35, 9, 0.3, 10)."""
    s = spheres_3d(seed=seed, G=G, ppc=ppc, E=E, nu=nu, density=density, dt=dt, nsteps=nsteps, model=HENCKY)
    s.name = "sand3d"
    s.plasticity = DruckerPrager.mast_case(2)
    return s


def snowballs_3d(seed=1234, G=128, ppc=8, E=1.4e5, nu=0.2, density=400.0, dt=5e-5, nsteps=200):
    """Two snowballs (r = 0.12) colliding in a 128^3 box, the spheres_3d geometry with the
    Stomakhin et al. 2013 snow parameters (theta_c 2.5e-2, theta_s 7.5e-3, hardening 10)."""
    s = spheres_3d(seed=seed, G=G, ppc=ppc, E=E, nu=nu, density=density, dt=dt, nsteps=nsteps, model=COROTATED)
    s.name = "snowballs3d"
    s.plasticity = Plasticity(max_hardening=10.0)
    return s


# --------------------------------------------------------------------------------------------
# Scene file: read by the reference runner (oracle/ref_scene.cpp) and by the C oracle harness.
# --------------------------------------------------------------------------------------------
MAGIC = b"MPMSCN08"


def write_scene(path, s: Scene, dumps: Optional[Sequence[int]] = None):
    dumps = list(dumps if dumps is not None else [s.nsteps - 1])
    d = s.dim
    pad3 = lambda v: list(v) + [0.0] * (3 - len(v))
    with open(path, "wb") as f:
        f.write(MAGIC)
        counts = list(s.counts) + [1] * (3 - d)
        pl = s.plasticity
        im, dc, rf, pn = s.implicit, s.dt_control, s.reflection, s.penalty
        moving = [(j, o.motion) for j, o in enumerate(s.objects) if o.motion is not None]
        f.write(struct.pack("<16i", d, *counts, s.model, s.nsteps, len(s.objects), len(dumps), pl.kind if pl else 0,
                            1 if im else 0, 1 if dc else 0, 1 if rf else 0, len(pn.objects) if pn else 0, len(moving),
                            1 if s.models is not None else 0, 1 if s.plastic_mask is not None else 0))
        f.write(struct.pack("<11d", *pad3(s.domain_min), *pad3(s.domain_max), *pad3(s.gravity), s.dt, 0.0))
        f.write(struct.pack("<%di" % len(dumps), *dumps))
        for o in s.objects:
            f.write(struct.pack("<2i7d", o.kind, o.type, o.friction, *pad3(o.a), *pad3(o.b)))
        if pl:
            prm = plastic_params(pl)[1:]
            f.write(struct.pack("<%dd" % len(prm), *prm))
        if im:
            f.write(struct.pack("<4d", im.newton_tolerance, im.newton_iterations, im.solver_tolerance,
                                im.solver_iterations))
        if dc:
            f.write(struct.pack("<8d", dc.frame_dt, dc.cfl, dc.min_dt, dc.max_dt, 1.0 if dc.strong_cfl else 0.0,
                                dc.cfl_F, 1.0 if dc.sound_cfl else 0.0, dc.cfl_sound))
        if rf:
            sides = list(rf.side_type) + [BC_FREE] * (6 - len(rf.side_type))
            f.write(struct.pack("<8d", *[float(x) for x in sides], rf.friction, 1.0 if rf.full else 0.0))
        if pn and pn.objects:
            f.write(struct.pack("<2d", pn.stiffness, pn.separation))
            for o in pn.objects:
                f.write(struct.pack("<2i7d", o.kind, o.type, o.friction, *pad3(o.a), *pad3(o.b)))
        for j, m in moving:   # object index, center, linear, angular (2D: the spin first)
            f.write(struct.pack("<i9d", j, *pad3(m.center), *pad3(m.linear), *pad3(m.angular)))
        f.write(struct.pack("<q", s.n))
        f.write(np.ascontiguousarray(s.X, np.float64).tobytes())
        f.write(np.ascontiguousarray(s.V, np.float64).tobytes())
        # column-major per particle, as MATRIX<T,d> stores it
        f.write(np.ascontiguousarray(np.swapaxes(s.F, 1, 2), np.float64).tobytes())
        f.write(np.ascontiguousarray(np.swapaxes(s.B, 1, 2), np.float64).tobytes())
        for a in (s.mass, s.volume, s.mu, s.lam):
            f.write(np.ascontiguousarray(a, np.float64).tobytes())
        if s.models is not None:
            f.write(np.ascontiguousarray(s.models, np.uint8).tobytes())
        if s.plastic_mask is not None:
            f.write(np.ascontiguousarray(s.plastic_mask, np.uint8).tobytes())
        if s.node_force is not None:   # optional trailer: a constant force at every node with mass
            f.write(b"XNF1")
            f.write(struct.pack("<3d", *pad3(s.node_force)))


def read_dump(path, dim, n, counts, plastic=()):
    """Read the per-substep dumps written by the reference runner / C oracle.

    Record: int32 step; X (n,d); V (n,d); F (n,d,d col-major); B (same); valid u8[n];
    grid mass after P2G; grid velocity after P2G (``v = mv/m``, d per node); grid
    velocity after forces; grid friction velocity after forces; then the plastic
    state named by `plastic` (`plastic_keys`): Fp (n,d,d col-major) and n scalars
    per other key.  Grids cover the ghosted domain
    (G+6)^d, last index fastest (`Core/Math_Tools/RANGE_ITERATOR.h`).
    """
    gshape = tuple(c + 2 * GHOST for c in counts[:dim])
    gn = int(np.prod(gshape))
    out = {}
    with open(path, "rb") as f:
        while True:
            hdr = f.read(4)
            if len(hdr) < 4:
                break
            step = struct.unpack("<i", hdr)[0]
            rec = {}
            rec["X"] = np.frombuffer(f.read(8 * n * dim), np.float64).reshape(n, dim)
            rec["V"] = np.frombuffer(f.read(8 * n * dim), np.float64).reshape(n, dim)
            rec["F"] = np.swapaxes(np.frombuffer(f.read(8 * n * dim * dim), np.float64).reshape(n, dim, dim), 1, 2)
            rec["B"] = np.swapaxes(np.frombuffer(f.read(8 * n * dim * dim), np.float64).reshape(n, dim, dim), 1, 2)
            rec["valid"] = np.frombuffer(f.read(n), np.uint8).astype(bool)
            rec["grid_m"] = np.frombuffer(f.read(8 * gn), np.float64).reshape(gshape)
            rec["grid_v0"] = np.frombuffer(f.read(8 * gn * dim), np.float64).reshape(gshape + (dim,))
            rec["grid_v"] = np.frombuffer(f.read(8 * gn * dim), np.float64).reshape(gshape + (dim,))
            rec["grid_vf"] = np.frombuffer(f.read(8 * gn * dim), np.float64).reshape(gshape + (dim,))
            for k in plastic:
                if k == "Fp":
                    rec[k] = np.swapaxes(np.frombuffer(f.read(8 * n * dim * dim), np.float64).reshape(n, dim, dim), 1, 2)
                else:
                    rec[k] = np.frombuffer(f.read(8 * n), np.float64).copy()
            out[step] = rec
    return out


CONFIGS = {
    "block2d": block_2d,
    "spheres3d": spheres_3d,
    "dam3d": dam_3d,
    "cube3d": cube_3d,
    "small3d": small_3d,
    "small2d": small_2d,
    "smallsnow3d": small_snow_3d,
    "smallsnow2d": small_snow_2d,
    "snowballs3d": snowballs_3d,
}
