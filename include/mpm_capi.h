/*
 * mpm_capi.h -- C ABI of the B200 explicit MPM substep (libphysbam_mpm.so).
 *
 * Drop-in for the explicit (symplectic Euler) APIC substep of PhysBAM's
 * Hybrid_Methods MPM driver.  Every entry point is extern "C", takes plain
 * pointers and sizes, returns an int status (0 = MPM_OK) and never throws.
 * One handle owns one simulation on one CUDA device and one stream; a handle
 * is not re-entrant (the reference driver is called from one host thread too,
 * Projects/mpm/STANDARD_TESTS_BASE.cpp:171-183).
 *
 * Particle arrays use the reference's MPM_PARTICLES layout
 * (Hybrid_Methods/Examples_And_Drivers/MPM_PARTICLES.h:18-44):
 *   X, V      n * d scalars, one d-vector per particle (ARRAY_VIEW<TV>)
 *   F, B      n * d * d scalars, column-major per particle (MATRIX<T,d>,
 *             Core/Matrices/MATRIX_3X3.h:115-119)
 *   mass, volume, mu, lambda   n scalars
 *   valid     n bytes (ARRAY_VIEW<bool>)
 * with scalar type float or double (the reference's T).
 *
 * Grid arrays returned by mpm_get_grid cover the ghosted domain
 * GRID::Domain_Indices(3) = [-3, G+3)^d with the last index fastest, the
 * layout of ARRAY<T,TV_INT> (MPM_DRIVER.cpp:102-108).
 */
#ifndef MPM_CAPI_H
#define MPM_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; PHYSBAM_FATAL_ERROR / PHYSBAM_ASSERT throw std::runtime_error in
 * the reference (Core/Log/DEBUG_UTILITIES.cpp:95-103); here they become codes. */
enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_ARG = 1,        /* bad argument, size or layout */
    MPM_ERR_CUDA = 2,       /* a CUDA call failed; see mpm_last_error */
    MPM_ERR_NAN = 3,        /* a non-finite value appeared in the particle state */
    MPM_ERR_DOMAIN = 4,     /* a particle stencil left the ghosted grid */
    MPM_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
    MPM_ERR_NOMEM = 6,      /* device allocation failed */
    MPM_ERR_STATE = 7,      /* call out of order (e.g. substep before particles) */
    MPM_ERR_NOT_CONVERGED = 8 /* a bounded SVD iteration did not converge */
};

enum mpm_precision { MPM_FP32 = 0, MPM_FP64 = 1 };

/* COROTATED_FIXED (Deformables/Constitutive_Models/COROTATED_FIXED.cpp:59-65),
 * NEO_HOOKEAN with failure threshold .25 (NEO_HOOKEAN.cpp:42-82),
 * ST_VENANT_KIRCHHOFF_HENCKY_STRAIN (ST_VENANT_KIRCHHOFF_HENCKY_STRAIN.cpp:67-78,
 * the elastic model of the reference's sand scenes). */
enum mpm_model { MPM_COROTATED_FIXED = 0, MPM_NEO_HOOKEAN = 1, MPM_STVK_HENCKY = 2 };

/* MPM_COLLISION_OBJECT::COLLISION_TYPE (Hybrid_Methods/Collisions/MPM_COLLISION_OBJECT.h:21) */
enum mpm_collision_type { MPM_STICK = 0, MPM_SLIP = 1, MPM_SEPARATE = 2 };

/* implicit object behind a collision object: RANGE box, PLANE half-space or SPHERE */
enum mpm_object_kind { MPM_BOX = 0, MPM_PLANE = 1, MPM_SPHERE = 2 };

/* which kernels run the substep */
enum mpm_path {
    MPM_PATH_FAST = 0,   /* cell-sorted particles, shared-memory tiles, fused stress (FP32) */
    MPM_PATH_PLAIN = 1   /* one thread per particle, global atomics, reference data layout */
};

#define MPM_MAX_OBJECTS 8

typedef struct mpm_handle mpm_handle;

/* GRID<TV> (Grid_Tools/Grids/GRID.h) as MPM_EXAMPLE uses it: a MAC grid of
 * counts[a] cells over [domain_min, domain_max], ghost = 3 (MPM_EXAMPLE.h:86). */
typedef struct {
    int dim;                 /* 2 or 3 */
    int counts[3];
    double domain_min[3];
    double domain_max[3];
    int ghost;               /* must be 3 */
} mpm_grid_desc;

/* The forces of MPM_EXAMPLE::forces for the explicit path: one
 * MPM_FINITE_ELEMENTS force (per-particle Lame arrays) and MPM_GRAVITY. */
typedef struct {
    int model;               /* mpm_model */
    int precision;           /* mpm_precision: arithmetic of the device path */
    int path;                /* mpm_path */
    double gravity[3];
} mpm_model_desc;

/* MPM_EXAMPLE::Add_Collision_Object(io, type, friction) for a static object.
 * MPM_BOX:    a = min corner, b = max corner (RANGE<TV>).
 * MPM_PLANE:  a = unit normal, b = a point on the plane (PLANE<T>).
 * MPM_SPHERE: a = center, b[0] = radius (SPHERE<TV>; a circle in 2D). */
typedef struct {
    int kind;
    int type;
    double friction;
    double a[3];
    double b[3];
} mpm_collision_object;

/* A view of MPM_PARTICLES attribute arrays.  dtype is the element type of
 * every floating-point array (mpm_precision).  on_device = 1 means the
 * pointers are CUDA device pointers on the handle's device. */
typedef struct {
    int64_t n;
    int dtype;
    int on_device;
    void* X;
    void* V;
    void* F;
    void* B;
    void* mass;
    void* volume;
    void* mu;
    void* lambda;
    uint8_t* valid;
} mpm_particles_view;

/* ---- lifetime ----------------------------------------------------------- */

/* Replaces MPM_DRIVER<TV>::MPM_DRIVER(example) + MPM_DRIVER::Initialize's grid
 * set-up (Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.cpp:47-55,81-137).
 * Binds the handle to the current CUDA device. */
int mpm_create(const mpm_grid_desc* grid, const mpm_model_desc* model, mpm_handle** out);

/* Replaces MPM_DRIVER::~MPM_DRIVER (MPM_DRIVER.cpp:59-67). */
int mpm_destroy(mpm_handle* h);

/* Run on this CUDA stream (cudaStream_t) instead of the handle's own. */
int mpm_set_stream(mpm_handle* h, void* stream);

/* ---- scene --------------------------------------------------------------- */

/* Replaces MPM_EXAMPLE::Add_Collision_Object for the whole list
 * (Hybrid_Methods/Examples_And_Drivers/MPM_EXAMPLE.cpp:331-338).  At most
 * MPM_MAX_OBJECTS objects. */
int mpm_set_collision_objects(mpm_handle* h, const mpm_collision_object* objs, int count);

/* Copies the particles in (the caller keeps ownership).  Replaces filling
 * MPM_EXAMPLE::particles in a scene's Initialize (MPM_PARTICLES.cpp:10-22,76-88). */
int mpm_set_particles(mpm_handle* h, const mpm_particles_view* view);

/* Copies X, V, F, B and valid out in the caller's particle order (mass,
 * volume, mu, lambda are read-only and left untouched). */
int mpm_get_particles(mpm_handle* h, mpm_particles_view* view);

/* ---- the substep ------------------------------------------------------- */

/* One explicit substep: MPM_DRIVER::Advance_One_Time_Step (MPM_DRIVER.cpp:141-157)
 * with use_symplectic_euler, use_affine, flip = 0 and quadratic weights:
 * Update_Simulated_Particles, Update_Particle_Weights, Particle_To_Grid,
 * Apply_Forces (incl. MPM_OBJECTIVE::Adjust_For_Collision and Apply_Friction),
 * Grid_To_Particle.  Asynchronous on the handle's stream. */
int mpm_substep(mpm_handle* h, double dt, double time);

/* nsteps substeps at fixed dt (the fixed-dt frame loop of
 * MPM_DRIVER::Simulate_To_Frame with min_dt = max_dt, MPM_DRIVER.cpp:161-201),
 * replayed from a captured CUDA graph. */
int mpm_advance(mpm_handle* h, double dt, double time, int nsteps);

/* The three phases of the substep, for callers that hook between them like
 * the reference's named Step callbacks "p2g", "forces", "g2p"
 * (MPM_DRIVER.cpp:1380-1393).  On the fast path the stress scatter of
 * Apply_Forces is fused into the P2G kernel; mpm_apply_forces then runs the
 * grid update alone. */
int mpm_particle_to_grid(mpm_handle* h, double dt, double time);  /* MPM_DRIVER::Particle_To_Grid, l.245-306 */
int mpm_apply_forces(mpm_handle* h, double dt, double time);      /* MPM_DRIVER::Apply_Forces, l.959-1060 */
int mpm_grid_to_particle(mpm_handle* h, double dt, double time);  /* MPM_DRIVER::Grid_To_Particle, l.450-515 */

/* Waits for the handle's stream and reports device-side error flags
 * (NaN, domain, non-convergence). */
int mpm_synchronize(mpm_handle* h);

/* ---- plasticity ----------------------------------------------------------- */

/* Plasticity, applied after each G2P to every particle simulated in the
 * substep (valid at its start, including one that left the domain in that
 * G2P) as MPM_DRIVER::Update_Plasticity_And_Hardening (MPM_DRIVER.cpp:156,
 * 922-928) through MPM_PLASTICITY_MODEL::Update_Particles
 * (MPM_PLASTICITY_MODEL.cpp:35-49).  The fast path runs it in FP32 inside G2P.
 *   MPM_PLASTICITY_CLAMP (snow; Hybrid_Methods/Forces/MPM_PLASTICITY_CLAMP.cpp:28-45)
 *   MPM_PLASTICITY_DRUCKER_PRAGER (sand; MPM_DRUCKER_PRAGER.cpp:42-125, explicit) */
enum mpm_plasticity_kind { MPM_PLASTICITY_NONE = 0, MPM_PLASTICITY_CLAMP = 1, MPM_PLASTICITY_DRUCKER_PRAGER = 2 };
typedef struct {
    int kind;
    /* clamp */
    double theta_c;            /* singular values are clamped to [1 - theta_c, 1 + theta_s] */
    double theta_s;
    double max_hardening;      /* hardening = exp(min(max_hardening, hardening_factor (1 - det Fp))) */
    double hardening_factor;
    /* Drucker-Prager: friction angle (degrees) a0 + (a1 q - a4) exp(-a3 q) of the
     * accumulated plastic deformation q; cohesion = the initial sigma_Y; use_vc
     * keeps the volume-correction term (MPM_DRUCKER_PRAGER::use_vc) */
    double dp_a0;
    double dp_a1;
    double dp_a3;
    double dp_a4;
    double cohesion;
    int use_vc;
} mpm_plasticity_desc;

/* Turn plasticity on or off (before or after mpm_set_particles).  Particles
 * then start unplastic, as the reference's scenes seed them: Fp = I; for the
 * clamp mu0 = mu, lambda0 = lambda (Projects/mpm/STANDARD_TESTS_BASE.cpp:299,
 * 568-586); for Drucker-Prager plastic_def = vc = 0, sigma_Y = cohesion and
 * rho_F from the friction angle at q = 0 (MPM_DRUCKER_PRAGER::Initialize_Particles).
 * The Drucker-Prager scenes pair it with MPM_STVK_HENCKY. */
int mpm_set_plasticity(mpm_handle* h, const mpm_plasticity_desc* p);

/* The plastic state of MPM_PARTICLES: Fp (n*d*d column-major) and n scalars
 * per other array; the clamp's (mu0, lambda0 and the hardened mu, lambda) or
 * Drucker-Prager's (plastic_def, rho_F, sigma_Y = cohesion, vc).  Any pointer
 * may be NULL (not copied); the other kind's arrays must be NULL. */
typedef struct {
    int64_t n;
    int dtype;
    int on_device;
    void* Fp;
    void* mu;
    void* lambda;
    void* mu0;
    void* lambda0;
    void* plastic_def;
    void* rho_F;
    void* cohesion;
    void* vc;
} mpm_plastic_view;
int mpm_get_plastic_state(mpm_handle* h, mpm_plastic_view* view);
int mpm_set_plastic_state(mpm_handle* h, const mpm_plastic_view* view);

/* Backward-Euler force solve instead of symplectic Euler: the reference's
 * default Apply_Forces (MPM_DRIVER.cpp:1024-1048), Newton's method on
 * MPM_OBJECTIVE with conjugate gradients and a strong-Wolfe line search, stopping
 * once the mass-weighted gradient norm is below newton_tolerance * dt; the CG
 * tolerance is relative, min(.5, solver_tolerance sqrt(max(residual,
 * tolerance))).  Defaults as MPM_EXAMPLE.h:119-122: 1, 100, .5, 1000.
 * Plain path only (FP64 or FP32, 2D or 3D); substeps then run eagerly, not
 * from CUDA graphs, since the host steers the iteration. */
typedef struct {
    int enabled;
    double newton_tolerance;
    int newton_iterations;
    double solver_tolerance;
    int solver_iterations;
} mpm_implicit_desc;
int mpm_set_implicit(mpm_handle* h, const mpm_implicit_desc* d);

/* Iterations of the last implicit solve (NEWTONS_METHOD::iterations_used and
 * the CG iterations summed over it) and its last gradient norm. */
typedef struct {
    int newton_iterations;
    int krylov_iterations;
    int converged;
    double residual;
} mpm_implicit_stats;
int mpm_get_implicit_stats(mpm_handle* h, mpm_implicit_stats* s);

/* Adaptive substeps: MPM_DRIVER::Simulate_To_Frame (MPM_DRIVER.cpp:161-201)
 * and Reduce_Dt (l.519-545).  Each substep takes Compute_Dt (the affine CFL
 * bound with `cfl`) clamped to [min_dt, max_dt] and fitted to the frame end;
 * after the forces, with strong_cfl, Grid_To_Particle_Limit_Dt limits the change
 * of F (cfl_F) and the displacement (cfl) of the coming G2P, and with
 * sound_cfl the largest sound speed limits dt to cfl_sound dx / c; a step so
 * shortened scales the grid velocity increments and ends early, and the frame
 * takes more substeps.  Defaults as MPM_EXAMPLE.h:84-115.  The reductions
 * of dt run on the plain path (they need the velocity after P2G and the stress
 * derivative); the fast path takes Compute_Dt steps without them. */
typedef struct {
    double cfl;
    double min_dt;
    double max_dt;
    int strong_cfl;
    double cfl_F;
    int sound_cfl;
    double cfl_sound;
} mpm_dt_control;
int mpm_set_dt_control(mpm_handle* h, const mpm_dt_control* c);

/* One frame of adaptive substeps from `time` to time + frame_dt; returns the
 * time reached (the frame end) and the number of substeps taken.  Each step is
 * one mpm_substep; mpm_last_dt gives the step the last substep took. */
int mpm_simulate_frame(mpm_handle* h, double time, double frame_dt, double* time_out, int* substeps);
int mpm_last_dt(mpm_handle* h, double* dt);

/* Reflection boundary conditions on the faces of the grid domain (MPM_EXAMPLE::
 * reflection_bc, side_bc_type; MPM_DRIVER.cpp:307-446, 1219-1239): the ghost
 * layer mirrors the interior.  Per side (-x, +x, -y, +y, -z, +z) free, slip,
 * no-slip or separating.  Without full_reflection, mass and momentum are
 * folded across each face after P2G, forces after the force computation and
 * velocities after the grid update; with full_reflection the velocities are
 * reflected once with Coulomb friction (`friction`) instead (scenes without
 * collision objects).  A particle that crosses a non-free face is mirrored
 * back (position and velocity) instead of being invalidated.  Plain path. */
enum mpm_bc_type { MPM_BC_FREE = 0, MPM_BC_SLIP = 1, MPM_BC_NOSLIP = 2, MPM_BC_SEP = 3 };
typedef struct {
    int enabled;
    int side_type[6];
    double friction;
    int full_reflection;
} mpm_reflection_desc;
int mpm_set_reflection(mpm_handle* h, const mpm_reflection_desc* r);

/* Penalty collision objects: one IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES per
 * object (Deformables/Collisions_And_Interactions/
 * IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES.cpp), added to the example's
 * Lagrangian forces as STANDARD_TESTS_BASE::Add_Penalty_Collision_Object does
 * (Projects/mpm/STANDARD_TESTS_BASE.cpp:555-563).  A particle whose signed
 * distance phi to an object is at most `separation` (x = separation - phi)
 * gets the force 3 stiffness x^2 n (n the object's normal at the particle;
 * l.49-60, 82-85), scattered to the grid with its weights
 * (MPM_DRIVER::Apply_Particle_Forces, MPM_DRIVER.cpp:933-945).  The implicit
 * solve adds the energy stiffness x^3 at the particle's moved position and the
 * Hessian 6 stiffness x n n^T - 3 stiffness x^2 Hess(phi)
 * (MPM_EXAMPLE::Add_Forces / Add_Hessian_Times, MPM_EXAMPLE.cpp:139-177).
 * Objects take mpm_collision_object's kind, a and b; `type` is not used and
 * `friction` is the force's coefficient_of_friction, which the MPM substep does
 * not apply.  The reference's scenes use stiffness 1e4 and separation 1e-4
 * (STANDARD_TESTS_BASE.cpp:47-49).  count = 0 removes them.  Both paths (on
 * the fast path as an impulse dt f added to the particle momentum in P2G); a
 * batch takes none. */
int mpm_set_penalty_objects(mpm_handle* h, const mpm_collision_object* objs, int count, double stiffness,
                            double separation);

/* A moving collision object: MPM_COLLISION_OBJECT's func_frame and func_twist
 * (Hybrid_Methods/Collisions/MPM_COLLISION_OBJECT.cpp:23-71).  The object's
 * geometry (mpm_collision_object's a, b) is then given in its own frame: at a
 * time its points Z sit at R Z + translation, R the rotation of the unit
 * quaternion `rotation` (w, x, y, z) (ROTATION<VECTOR<T,3> >; in 2D
 * (cos theta, sin theta, 0, 0), ROTATION<VECTOR<T,2> >), and a point X of the
 * object moves with linear + angular x (X - translation) (TWIST; in 2D
 * angular[0] is the spin).  The callback fills the state at `time` and returns
 * 0 (non-zero: the substep fails with MPM_ERR_ARG).  Each substep from t to
 * t + dt calls it at t and t + dt: MPM_OBJECTIVE::Test_Add_Collision
 * (MPM_OBJECTIVE.cpp:150-181) tests a node's start against the frame at t,
 * projects its end at t + dt, and holds a sticky node at the object's velocity
 * there.  fn = NULL makes the object static again.  mpm_substep with moving
 * objects runs eagerly; mpm_advance over several substeps evaluates every
 * substep's frames first and replays its CUDA graph, whose first kernel takes
 * the next substep's frames.  Both paths and the implicit solve; a batch takes
 * none. */
typedef struct {
    double translation[3];
    double rotation[4];
    double linear[3];
    double angular[3];
} mpm_object_state;
typedef int (*mpm_motion_fn)(void* user, int object, double time, mpm_object_state* state);
int mpm_set_object_motion(mpm_handle* h, int object, mpm_motion_fn fn, void* user);

/* A constitutive model per particle (mpm_model values, n bytes in the caller's
 * particle order): the reference's several MPM_FINITE_ELEMENTS forces, each
 * over its affected_particles with its own model (MPM_FINITE_ELEMENTS.cpp:
 * 47-132; Projects/mpm/STANDARD_TESTS_BASE.cpp:373-404).  models = NULL: every
 * particle takes the handle's model again.  Call after mpm_set_particles; a
 * new particle count drops the per-particle models.  Both paths (the implicit
 * solve included); a batch takes one model per scene. */
int mpm_set_particle_models(mpm_handle* h, const uint8_t* models, int64_t n);

/* The particles the plasticity model acts on (n bytes, non-zero: plastic), the
 * model's affected_particles (MPM_PLASTICITY_MODEL::Update_Particles over its
 * gather_scatter's particles, MPM_PLASTICITY_MODEL.cpp:35-49; Initialize_
 * Particles over the same, MPM_DRUCKER_PRAGER.cpp:43-60), e.g. the sand of a
 * sand-and-water scene.  The others keep Fp = I and a zero Drucker-Prager state.
 * mask = NULL: every particle.  Call after mpm_set_particles; it restarts the
 * plastic state.  Both paths; a batch takes one plasticity for all. */
int mpm_set_plastic_particles(mpm_handle* h, const uint8_t* mask, int64_t n);

/* ---- inspection ---------------------------------------------------------- */

/* Grids of the last substep as doubles on the host, each (G+6)^d nodes (times
 * d for vectors): mass after P2G (MPM_EXAMPLE::mass), velocity after P2G
 * (velocity_save; NULL-able, FP64/plain path only), velocity after the forces
 * (MPM_EXAMPLE::velocity) and friction velocity (velocity_friction_save).
 * Any pointer may be NULL. */
int mpm_get_grid(mpm_handle* h, double* mass, double* v0, double* v, double* vfric);

/* Extra node forces for the next grid update: the Add_Forces of a force this
 * library does not model (PARTICLE_GRID_FORCES::Add_Forces,
 * Hybrid_Methods/Forces/PARTICLE_GRID_FORCES.h:17-36; MPM_EXAMPLE::Add_Forces
 * sums every force's, MPM_EXAMPLE.cpp:115-153), evaluated by the caller.
 * `force` holds d values per node of the ghosted grid ((G+6)^d nodes, last
 * index fastest: the layout of MPM_EXAMPLE's ARRAY<TV,TV_INT>), float or
 * double (dtype), host or device pointer (on_device).  Call between
 * mpm_particle_to_grid and mpm_apply_forces; that grid update adds the force
 * at every node with mass (dv = dt f / m), dt being the step it takes.  Calls
 * add up.  Single-scene handles, explicit substep. */
int mpm_add_grid_forces(mpm_handle* h, double dt, const void* force, int dtype, int on_device);

/* Number of valid particles (MPM_EXAMPLE::simulated_particles.m). */
int mpm_count_valid(mpm_handle* h, int64_t* count);

/* Conservation and CFL diagnostics, reduced on the GPU in FP64. */
typedef struct {
    double mass;
    double momentum[3];
    double angular_momentum[3];   /* 2D: the one component is [0] */
    double kinetic_energy;
    double max_speed;             /* particles only */
    double max_affine_speed;      /* particles only: |V| + |B|_F 6 sqrt(d) / dx */
    int64_t count;                /* valid particles / grid nodes with mass */
} mpm_totals;

/* Over the valid particles: MPM_EXAMPLE::Total_Particle_Linear_Momentum,
 * Total_Particle_Angular_Momentum (incl. the APIC B term) and
 * Total_Particle_Kinetic_Energy (MPM_EXAMPLE.cpp:209-327), with
 * MPM_DRIVER::Max_Particle_Speed and Grid_V_Upper_Bound (MPM_DRIVER.cpp:1112-1138). */
int mpm_particle_totals(mpm_handle* h, mpm_totals* out);

/* Over the grid of the last substep, velocity after the forces:
 * Total_Grid_Linear_Momentum / Angular_Momentum / Kinetic_Energy. */
int mpm_grid_totals(mpm_handle* h, mpm_totals* out);

/* MPM_DRIVER::Compute_Dt (MPM_DRIVER.cpp:1098-1105) with the affine CFL bound
 * (use_affine_cfl): cfl * dx_min / v, or max_dt when v is below
 * cfl * dx_min / max_dt.  For a batch, dx_min is the smallest cell of any
 * scene and v the largest bound of any scene: a step every scene can take. */
int mpm_compute_dt(mpm_handle* h, double cfl, double max_dt, double* dt);

/* Per-kernel device time: enable (1) / disable (0) CUDA-event timing, then read
 * totals.  names gets a comma-separated list, ms and launches one entry each. */
int mpm_set_timing(mpm_handle* h, int enable);
int mpm_get_timing(mpm_handle* h, char* names, int names_len, double* ms, int64_t* launches, int max_entries, int* count);

/* ---- many independent scenes in one handle --------------------------------- */

/* One scene of a batch.  Its particles are particle_count consecutive entries
 * of the arrays given to mpm_set_particles, scenes in order; its collision
 * objects are objects[first_object, first_object + object_count) of
 * mpm_batch_create. */
typedef struct {
    mpm_grid_desc grid;      /* dim must be 3, ghost 3 */
    int model;               /* mpm_model */
    double gravity[3];
    int64_t particle_count;
    int first_object;
    int object_count;        /* <= MPM_MAX_OBJECTS */
} mpm_scene_desc;

/* A handle that advances `count` independent scenes (different grid sizes,
 * domains, models, objects) together: every phase of the substep is one
 * persistent launch over the blocks of all scenes, and mpm_advance replays it
 * from a CUDA graph.  FP32 fast path.  The reference runs one MPM_EXAMPLE per
 * process; there is no counterpart call. */
int mpm_batch_create(const mpm_scene_desc* scenes, int count, const mpm_collision_object* objects, int object_count,
                     mpm_handle** out);

/* mpm_get_grid for scene `scene` of a batch (or scene 0 of any fast-path
 * handle): the scene's ghosted grid, (G+6)^3 nodes, of the last substep, as
 * that scene's MPM_EXAMPLE would hold it (mass, velocity after the forces,
 * friction velocity; any pointer may be NULL). */
int mpm_batch_get_grid(mpm_handle* h, int scene, double* mass, double* v, double* vfric);

/* Time the fast path's launch shapes (P2G work split, G2P block size, number of
 * persistent CTAs) for `substeps` substeps each on the handle's own particles
 * and keep the fastest; the particle state is left unchanged.  `report` (may be
 * NULL) receives the timings. */
int mpm_autotune(mpm_handle* h, double dt, int substeps, char* report, int report_len);

/* mpm_autotune with flags.  MPM_AUTOTUNE_COLD_L2: write a buffer of twice the
 * L2 size before each timed substep (untimed), so the choice holds for a
 * caller whose substeps do not find the particles in L2 (substeps up to 64). */
#define MPM_AUTOTUNE_COLD_L2 1
int mpm_autotune_ex(mpm_handle* h, double dt, int substeps, int flags, char* report, int report_len);

/* The fast path's launch shape, as mpm_autotune chooses it (no reference
 * counterpart: the reference's OpenMP loops have no launch configuration).
 * p2g_variant: MPM_P2G_GROUPS128 / MPM_P2G_GROUPS256 (groups of 4 lanes
 * accumulating a cell's node values in registers, 128 or 256 threads, work
 * items of up to 512 / 1024 particles of a block), MPM_P2G_FIXED128 /
 * MPM_P2G_FIXED256 (one thread per particle into a fixed-point shared tile,
 * work items of up to 128 / 256 particles); G2P takes the same work items;
 * g2p_threads: 64, 128 or 256 per CTA; cta_mult: 1 or 2 times the resident
 * CTAs per SM.  A new handle starts with MPM_P2G_FIXED256, 128, 1. */
enum { MPM_P2G_GROUPS128 = 0, MPM_P2G_GROUPS256 = 1, MPM_P2G_FIXED128 = 2, MPM_P2G_FIXED256 = 3 };
int mpm_set_launch_shape(mpm_handle* h, int p2g_variant, int g2p_threads, int cta_mult);
int mpm_get_launch_shape(mpm_handle* h, int* p2g_variant, int* g2p_threads, int* cta_mult);

/* ---- differentiation ------------------------------------------------------ */

/* Records a differentiable rollout: nsteps explicit substeps from the current
 * particles, keeping the particle state every checkpoint_every substeps, and,
 * when the tape budget allows (mpm_set_diff_tape_budget), every substep's
 * intermediates.  MPM_PATH_PLAIN, 3D, static frictionless boxes, planes and
 * spheres, one constitutive model.  The reference has no reverse
 * mode; this is the forward whose transposed linearisation mpm_diff_backward
 * applies (the reference's linearisations of the same maps are
 * MPM_FINITE_ELEMENTS::Add_Hessian_Times, Hybrid_Methods/Forces/
 * MPM_FINITE_ELEMENTS.cpp:103-132, and MPM_OBJECTIVE::Update_F,
 * Hybrid_Methods/System/MPM_OBJECTIVE.cpp:95-134).  The handle ends at the
 * final state. */
int mpm_diff_forward(mpm_handle* h, double dt, int nsteps, int checkpoint_every);

/* Reverse pass of the last mpm_diff_forward: given dL/d(final X, V, F, B) in
 * grad_final, writes dL/d(initial X, V, F, B) to grad_initial and dL/dmu,
 * dL/dlambda (n each) to grad_mu / grad_lambda.  Segments between checkpoints
 * are recomputed unless the forward kept every substep.  Views carry only X,
 * V, F, B; dtype must equal the path's precision; on_device selects device or
 * host pointers. */
int mpm_diff_backward(mpm_handle* h, const mpm_particles_view* grad_final, mpm_particles_view* grad_initial,
                      void* grad_mu, void* grad_lambda);

/* Device memory the next mpm_diff_forward may spend on keeping every substep's
 * intermediates (state, node masses and velocities, the grid update's map,
 * P F^T), so that the backward recomputes nothing: bytes < 0 (the default)
 * allows up to a quarter of the free device memory, 0 keeps checkpoints only
 * (every segment recomputed by the backward, memory bounded by the checkpoint
 * interval), bytes > 0 caps it.  No reference counterpart (the reference has
 * no reverse mode). */
int mpm_set_diff_tape_budget(mpm_handle* h, int64_t bytes);

/* ---- sorting ------------------------------------------------------------- */

/* Stable LSD radix sort of n 32-bit keys by their low `bits` bits (1..32) on
 * the current device, host arrays in and out: the kernels the fast path sorts
 * particle cell keys with, which replace the reference's x-slab binning
 * GATHER_SCATTER::Prepare_Scatter (Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:33-87).
 * perm[i] = index of the i-th smallest key (ties keep input order). */
int mpm_radix_sort_u32(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys, uint32_t* perm);

/* The same sort for callers that cannot allocate device memory at the time
 * they sort: hosts that give the library a fixed memory budget up front and
 * forbid growth afterwards, and loops that cannot absorb cudaMalloc/cudaFree
 * and the device-wide synchronisation cudaFree brings.
 * There is no counterpart in the reference (it sorts on the CPU).
 * keys, sorted_keys and perm are DEVICE arrays of n entries on the current
 * device; keys must not alias an output and the two outputs must not alias
 * each other (MPM_ERR_ARG).  The work runs on `stream` (cudaStream_t, NULL =
 * legacy default stream) and the call blocks until it is done: it reads back
 * the sort's timeout flag and returns MPM_ERR_TIMEOUT if a bounded wait gave up.
 * It allocates nothing: its temporaries live in one fixed array compiled into
 * the library (about 2.6 MB, held on every device that loads the library until
 * exit), so n is limited to MPM_NOALLOC_MAX_KEYS; larger n returns MPM_ERR_ARG
 * (use mpm_radix_sort_u32).  The first call on a device looks up that array's
 * address and zeroes it (a synchronous cudaMemset): make that first call before
 * any stream capture.  All calls on a device share the array, so calls that
 * overlap on the GPU race; serialise them. */
#define MPM_NOALLOC_MAX_KEYS 262144
int mpm_radix_sort_u32_noalloc(const uint32_t* keys, int64_t n, int bits, uint32_t* sorted_keys, uint32_t* perm,
                               void* stream);

/* Fast path only: cell keys of the current particle slots, and the sorted keys
 * and slot permutation of the last sort (host arrays of n entries, NULL-able).
 * Key = (particle block << 6) | cell in block; 0xffffffff = invalid particle. */
int mpm_debug_sort_state(mpm_handle* h, uint32_t* slot_keys, uint32_t* sorted_keys, uint32_t* perm);

/* Test hooks for the device-side failure paths (no reference counterpart; the
 * reference's asserts throw, Core/Log/DEBUG_UTILITIES.cpp:95-103):
 * mpm_debug_sort_stall runs one radix pass over the host keys whose first tile
 * never runs, so the other tiles' bounded look-back gives up after spin_limit
 * polls (<= 2^22); returns MPM_ERR_TIMEOUT when it did (2 to 2^21/1024 tiles of
 * 1024 keys).  mpm_debug_set_sort_epoch seeds the epoch word of a fast-path
 * handle's sort scratch (sorts across the wrap of its 30-bit field).
 * mpm_debug_set_svd_iterations bounds the FP64 3x3 SVD's QR sweeps on the
 * current device (default 64); a particle whose SVD does not converge within
 * the bound sets MPM_ERR_NOT_CONVERGED. */
int mpm_debug_sort_stall(const uint32_t* keys, int64_t n, int bits, uint32_t spin_limit);
int mpm_debug_set_sort_epoch(mpm_handle* h, uint32_t epoch);
int mpm_debug_set_svd_iterations(int max_it);

/* Human-readable text of the last error on this handle / of a status code. */
int mpm_last_error(mpm_handle* h, char* buf, int len);
const char* mpm_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif
