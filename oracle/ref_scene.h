// Scene files of physbam_b200/scenes.py read into the reference's own
// MPM_EXAMPLE (test infrastructure, shared by the runners ref_scene.cpp and
// ref_b200.cpp under oracle/; built by oracle/ref.mk against the reference's
// sources).
//
// The scene is set up through the reference's public API exactly as
// Projects/mpm/STANDARD_TESTS_BASE.cpp does it: quadratic weights
// (MPM_EXAMPLE.cpp:197-205), MPM_FINITE_ELEMENTS + COROTATED_FIXED,
// NEO_HOOKEAN or ST_VENANT_KIRCHHOFF_HENCKY_STRAIN with per-particle Lame
// arrays (STANDARD_TESTS_BASE.cpp:372-404), MPM_PLASTICITY_CLAMP or
// MPM_DRUCKER_PRAGER after G2P (l.409-486),
// MPM_GRAVITY (l.354-358), collision objects through Add_Collision_Object,
// penalty collision objects (IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES, l.555-563),
// moving collision objects (func_frame, func_twist of a constant twist),
// symplectic Euler or (scene flag) the backward-Euler Newton solve, APIC
// (use_affine), flip=0, fixed dt.
#pragma once
#include <Core/Log/LOG.h>
#include <Core/Math_Tools/RANGE.h>
#include <Core/Matrices/FRAME.h>
#include <Core/Matrices/MATRIX.h>
#include <Core/Vectors/TWIST.h>
#include <Core/Vectors/VECTOR.h>
#include <Geometry/Basic_Geometry/PLANE.h>
#include <Geometry/Basic_Geometry/SPHERE.h>
#include <Geometry/Implicit_Objects/ANALYTIC_IMPLICIT_OBJECT.h>
#include <Deformables/Collisions_And_Interactions/IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES.h>
#include <Deformables/Constitutive_Models/COROTATED_FIXED.h>
#include <Deformables/Constitutive_Models/NEO_HOOKEAN.h>
#include <Deformables/Constitutive_Models/ST_VENANT_KIRCHHOFF_HENCKY_STRAIN.h>
#include <Hybrid_Methods/Examples_And_Drivers/MPM_DRIVER.h>
#include <Hybrid_Methods/Examples_And_Drivers/MPM_EXAMPLE.h>
#include <Hybrid_Methods/Examples_And_Drivers/MPM_PARTICLES.h>
#include <Hybrid_Methods/Forces/MPM_FINITE_ELEMENTS.h>
#include <Hybrid_Methods/Forces/MPM_GRAVITY.h>
#include <Hybrid_Methods/Forces/PARTICLE_GRID_FORCES.h>
#include <Hybrid_Methods/Forces/MPM_PLASTICITY_CLAMP.h>
#include <Hybrid_Methods/Forces/MPM_DRUCKER_PRAGER.h>
#include <Hybrid_Methods/Forces/MPM_FORCE_HELPER.h>
#include <Hybrid_Methods/Iterators/GATHER_SCATTER.h>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef USE_OPENMP
#include <omp.h>
#endif
using namespace PhysBAM;

namespace {
struct OBJ { int kind, type; double friction, a[3], b[3]; int moving = 0; double c[3], v[3], w[3]; };
struct SCENE_FILE
{
    int dim, counts[3], model, nsteps, nobj, ndump, plasticity, implicit, dt_control, reflection, npen;
    double pen_prm[2];   // penalty stiffness, separation
    double refl[8];   // side types (6), friction, full
    // frame_dt, cfl, min_dt, max_dt, strong_cfl, cfl_F, sound_cfl, cfl_sound
    double dtc[8];
    double implicit_prm[4];   // newton_tolerance, newton_iterations, solver_tolerance, solver_iterations
    // clamp (1): theta_c, theta_s, max_hardening, hardening_factor;
    // Drucker-Prager (2): a0, a1, a3, a4, sigma_Y0, use_vc
    double plastic[6];
    double dmin[3], dmax[3], gravity[3], dt, t0;
    std::vector<int> dumps;
    std::vector<OBJ> objs, pen;
    long long n;
    std::vector<double> X, V, F, B, mass, volume, mu, lambda;
    std::vector<unsigned char> models;   // per-particle constitutive model (empty: `model` for all)
    std::vector<unsigned char> plastic_mask;   // the plasticity's particles (empty: all)
    bool node_force = false;                    // trailer: a constant force at every node with mass
    double node_f[3] = {0, 0, 0};
};

template<class T> void rd(FILE* f, T* p, size_t n)
{
    if(fread(p, sizeof(T), n, f) != n) throw std::runtime_error("short scene file");
}

SCENE_FILE Read_Scene(const char* path)
{
    FILE* f = fopen(path, "rb");
    if(!f) throw std::runtime_error("cannot open scene");
    char magic[8];
    rd(f, magic, 8);
    if(memcmp(magic, "MPMSCN08", 8)) throw std::runtime_error("bad scene magic");
    SCENE_FILE s;
    int hdr[16];
    rd(f, hdr, 16);
    s.npen = hdr[12];
    const int nmoving = hdr[13];
    s.reflection = hdr[11];
    s.implicit = hdr[9];
    s.dt_control = hdr[10];
    s.dim = hdr[0]; s.counts[0] = hdr[1]; s.counts[1] = hdr[2]; s.counts[2] = hdr[3];
    s.model = hdr[4]; s.nsteps = hdr[5]; s.nobj = hdr[6]; s.ndump = hdr[7]; s.plasticity = hdr[8];
    double dh[11];
    rd(f, dh, 11);
    for(int i = 0; i < 3; i++) { s.dmin[i] = dh[i]; s.dmax[i] = dh[3 + i]; s.gravity[i] = dh[6 + i]; }
    s.dt = dh[9]; s.t0 = dh[10];
    s.dumps.resize(s.ndump);
    if(s.ndump) rd(f, s.dumps.data(), s.ndump);
    for(int i = 0; i < s.nobj; i++) {
        OBJ o;
        rd(f, &o.kind, 1); rd(f, &o.type, 1); rd(f, &o.friction, 1); rd(f, o.a, 3); rd(f, o.b, 3);
        s.objs.push_back(o);
    }
    if(s.plasticity == 1) rd(f, s.plastic, 4);
    else if(s.plasticity == 2) rd(f, s.plastic, 6);
    else if(s.plasticity) throw std::runtime_error("unknown plasticity");
    if(s.implicit) rd(f, s.implicit_prm, 4);
    if(s.dt_control) rd(f, s.dtc, 8);
    if(s.reflection) rd(f, s.refl, 8);
    if(s.npen) {
        rd(f, s.pen_prm, 2);
        for(int i = 0; i < s.npen; i++) {
            OBJ o;
            rd(f, &o.kind, 1); rd(f, &o.type, 1); rd(f, &o.friction, 1); rd(f, o.a, 3); rd(f, o.b, 3);
            s.pen.push_back(o);
        }
    }
    for(int i = 0; i < nmoving; i++) {   // object index, then its constant twist: center, linear, angular
        int j;
        rd(f, &j, 1);
        if(j < 0 || j >= s.nobj) throw std::runtime_error("moving object index");
        OBJ& o = s.objs[j];
        o.moving = 1;
        rd(f, o.c, 3); rd(f, o.v, 3); rd(f, o.w, 3);
    }
    rd(f, &s.n, 1);
    size_t n = s.n, d = s.dim;
    s.X.resize(n * d); s.V.resize(n * d); s.F.resize(n * d * d); s.B.resize(n * d * d);
    s.mass.resize(n); s.volume.resize(n); s.mu.resize(n); s.lambda.resize(n);
    rd(f, s.X.data(), n * d); rd(f, s.V.data(), n * d);
    rd(f, s.F.data(), n * d * d); rd(f, s.B.data(), n * d * d);
    rd(f, s.mass.data(), n); rd(f, s.volume.data(), n); rd(f, s.mu.data(), n); rd(f, s.lambda.data(), n);
    if(hdr[14]) { s.models.resize(n); rd(f, s.models.data(), n); }
    if(hdr[15]) { s.plastic_mask.resize(n); rd(f, s.plastic_mask.data(), n); }
    char tag[4];
    if(fread(tag, 1, 4, f) == 4 && !memcmp(tag, "XNF1", 4)) { rd(f, s.node_f, 3); s.node_force = true; }
    fclose(f);
    return s;
}

// A force the GPU library does not model, for the parity test of its
// extra-force entry point: the same vector at every node with mass
// (PARTICLE_GRID_FORCES, Hybrid_Methods/Forces/PARTICLE_GRID_FORCES.h:17-36;
// explicit substep only).
template<class TV> struct NODE_FORCE_CONSTANT: public PARTICLE_GRID_FORCES<TV>
{
    typedef typename TV::SCALAR T;
    typedef VECTOR<int, TV::m> TV_INT;
    const MPM_EXAMPLE<TV>& ex;
    TV f0;
    NODE_FORCE_CONSTANT(const MPM_EXAMPLE<TV>& ex, const TV& f0): PARTICLE_GRID_FORCES<TV>(ex.force_helper), ex(ex), f0(f0) {}
    void Precompute(const T, const T, bool, bool) override {}
    T Potential_Energy(const T) const override { return 0; }
    void Add_Forces(ARRAY<TV, TV_INT>& F, const T) const override
    {
        for(int k = 0; k < ex.valid_grid_indices.m; k++) F.array(ex.valid_grid_indices(k)) += f0;
    }
    void Add_Hessian_Times(ARRAY<TV, TV_INT>&, const ARRAY<TV, TV_INT>&, const T) const override {}
};

template<class TV> struct FILE_SCENE: public MPM_EXAMPLE<TV>
{
    typedef typename TV::SCALAR T;
    typedef VECTOR<int, TV::m> TV_INT;
    typedef MPM_EXAMPLE<TV> BASE;
    typedef typename BASE::COLLISION_TYPE COLLISION_TYPE;
    using BASE::grid; using BASE::particles; using BASE::gather_scatter; using BASE::force_helper;
    const SCENE_FILE& s;
    MPM_DRUCKER_PRAGER<TV>* dp = 0;

    FILE_SCENE(const SCENE_FILE& s_, int threads)
        : BASE(STREAM_TYPE(T())), s(s_)
    {
        this->threads = threads;
        gather_scatter.threads = threads;
        this->use_symplectic_euler = !s.implicit;
        if(s.implicit) {   // MPM_EXAMPLE's Newton / Krylov controls (MPM_EXAMPLE.h:119-122)
            this->newton_tolerance = (T)s.implicit_prm[0];
            this->newton_iterations = (int)s.implicit_prm[1];
            this->solver_tolerance = (T)s.implicit_prm[2];
            this->solver_iterations = (int)s.implicit_prm[3];
        }
        this->use_affine = true;
        this->flip = 0;
        this->min_dt = this->max_dt = (T)s.dt;
        if(s.reflection) {   // as Add_Walls sets them with -use_reflect (STANDARD_TESTS_BASE.cpp:487-511)
            this->reflection_bc = true;
            for(int k = 0; k < 2 * TV::m; k++) this->side_bc_type(k) = (typename BASE::BC_TYPE)(int)s.refl[k];
            this->reflection_bc_friction = (T)s.refl[6];
            this->use_full_reflection = s.refl[7] != 0;
        }
        if(s.dt_control) {   // Simulate_To_Frame with MPM_EXAMPLE's step controls
            this->frame_dt = (T)s.dtc[0];
            this->cfl = (T)s.dtc[1];
            this->min_dt = (T)s.dtc[2];
            this->max_dt = (T)s.dtc[3];
            this->use_strong_cfl = s.dtc[4] != 0;
            this->cfl_F = (T)s.dtc[5];
            this->use_sound_speed_cfl = s.dtc[6] != 0;
            this->cfl_sound = (T)s.dtc[7];
        }
        particles.Store_B(true);
    }

    void Initialize() override
    {
        const int d = TV::m;
        TV_INT counts; TV lo, hi;
        for(int a = 0; a < d; a++) { counts(a) = s.counts[a]; lo(a) = (T)s.dmin[a]; hi(a) = (T)s.dmax[a]; }
        grid.Initialize(counts, RANGE<TV>(lo, hi), true);
        this->Set_Weights(2);
        particles.Store_Lame(true);
        if(s.plasticity) particles.Store_Fp(true);   // also stores mu0, lambda0
        particles.Add_Elements((int)s.n);
        for(int p = 0; p < s.n; p++) {
            for(int a = 0; a < d; a++) {
                particles.X(p)(a) = (T)s.X[p * d + a];
                particles.V(p)(a) = (T)s.V[p * d + a];
            }
            for(int k = 0; k < d * d; k++) {
                particles.F(p).x[k] = (T)s.F[p * d * d + k];
                particles.B(p).x[k] = (T)s.B[p * d * d + k];
            }
            particles.mass(p) = (T)s.mass[p];
            particles.volume(p) = (T)s.volume[p];
            particles.mu(p) = (T)s.mu[p];
            particles.lambda(p) = (T)s.lambda[p];
            particles.valid(p) = true;
            if(s.plasticity) {   // as STANDARD_TESTS_BASE seeds and Set_Lame_On_Particles
                particles.Fp(p).Set_Identity_Matrix();
                particles.mu0(p) = particles.mu(p);
                particles.lambda0(p) = particles.lambda(p);
            }
        }
        // a plasticity over a particle subset runs on its own gather_scatter of those particles, as
        // Add_Drucker_Prager hands it the subset force's (STANDARD_TESTS_BASE.cpp:409-433)
        GATHER_SCATTER<TV>* pgs = &gather_scatter;
        ARRAY<int> plastic;
        if(!s.plastic_mask.empty()) {
            for(int p = 0; p < (int)s.plastic_mask.size(); p++) if(s.plastic_mask[p]) plastic.Append(p);
            pgs = new GATHER_SCATTER<TV>(grid, *new ARRAY<int>(plastic));
            pgs->weights = gather_scatter.weights;
            pgs->threads = gather_scatter.threads;
            pgs->Prepare_Scatter(particles);
        }
        if(s.plasticity == 1)
            this->plasticity_models.Append(new MPM_PLASTICITY_CLAMP<TV>(particles, pgs, (T)s.plastic[0],
                (T)s.plastic[1], (T)s.plastic[2], (T)s.plastic[3]));
        if(s.plasticity == 2) {   // as STANDARD_TESTS_BASE::Add_Drucker_Prager (explicit)
            dp = new MPM_DRUCKER_PRAGER<TV>(particles, pgs, (T)s.plastic[0], (T)s.plastic[1],
                (T)s.plastic[2], (T)s.plastic[3]);
            dp->use_vc = s.plastic[5] != 0;
            dp->Initialize_Particles(s.plastic_mask.empty() ? 0 : &plastic, (T)s.plastic[4]);
            this->plasticity_models.Append(dp);
        }
        auto make_model = [](int m) -> ISOTROPIC_CONSTITUTIVE_MODEL<T, TV::m>* {
            if(m == 0) return new COROTATED_FIXED<T, TV::m>((T)1, (T).3);
            if(m == 1) return new NEO_HOOKEAN<T, TV::m>((T)1, (T).3);
            return new ST_VENANT_KIRCHHOFF_HENCKY_STRAIN<T, TV::m>((T)1, (T).3);};
        if(s.models.empty()) this->Add_Force(*new MPM_FINITE_ELEMENTS<TV>(force_helper, *make_model(s.model), gather_scatter, 0));
        else   // one force per model over its particles, as the scenes pass affected_particles
            for(int m = 0; m < 3; m++) {
                ARRAY<int> affected;
                for(int p = 0; p < (int)s.models.size(); p++) if(s.models[p] == m) affected.Append(p);
                if(affected.m) this->Add_Force(*new MPM_FINITE_ELEMENTS<TV>(force_helper, *make_model(m), gather_scatter, &affected));
            }
        TV g;
        for(int a = 0; a < d; a++) g(a) = (T)s.gravity[a];
        this->Add_Force(*new MPM_GRAVITY<TV>(force_helper, g, gather_scatter, 0));
        if(s.node_force) {
            TV f0;
            for(int a = 0; a < d; a++) f0(a) = (T)s.node_f[a];
            this->Add_Force(*new NODE_FORCE_CONSTANT<TV>(*this, f0));
        }
        for(const OBJ& o: s.objs) {
            COLLISION_TYPE type = o.type == 0 ? COLLISION_TYPE::stick : o.type == 1 ? COLLISION_TYPE::slip : COLLISION_TYPE::separate;
            TV a, b;
            for(int k = 0; k < d; k++) { a(k) = (T)o.a[k]; b(k) = (T)o.b[k]; }
            std::function<FRAME<TV>(T)> frame;
            std::function<TWIST<TV>(T)> twist;
            if(o.moving) {   // func_frame / func_twist of a constant twist, as the rotating scenes write them
                TV c, v;
                typename TV::SPIN w;
                for(int k = 0; k < d; k++) { c(k) = (T)o.c[k]; v(k) = (T)o.v[k]; }
                for(int k = 0; k < w.m; k++) w(k) = (T)o.w[k];
                frame = [=](T time){return FRAME<TV>(c + v * time, ROTATION<TV>::From_Rotation_Vector(w * time));};
                twist = [=](T){return TWIST<TV>(v, w);};
            }
            if(o.kind == 0) this->Add_Collision_Object(RANGE<TV>(a, b), type, (T)o.friction, frame, twist);
            else if(o.kind == 2) this->Add_Collision_Object(SPHERE<TV>(a, (T)o.b[0]), type, (T)o.friction, frame, twist);
            else Add_Plane(a, b, type, (T)o.friction, frame, twist);
        }
        // penalty collision objects as STANDARD_TESTS_BASE::Add_Penalty_Collision_Object
        // adds them (Projects/mpm/STANDARD_TESTS_BASE.cpp:557-563): one force per object
        for(const OBJ& o: s.pen) {
            TV a, b;
            for(int k = 0; k < d; k++) { a(k) = (T)o.a[k]; b(k) = (T)o.b[k]; }
            IMPLICIT_OBJECT<TV>* io;
            if(o.kind == 0) io = new ANALYTIC_IMPLICIT_OBJECT<RANGE<TV> >(RANGE<TV>(a, b));
            else if(o.kind == 2) io = new ANALYTIC_IMPLICIT_OBJECT<SPHERE<TV> >(SPHERE<TV>(a, (T)o.b[0]));
            else io = Plane_Object(a, b);
            auto* pf = new IMPLICIT_OBJECT_COLLISION_PENALTY_FORCES<TV>(particles, io, (T)s.pen_prm[0], (T)s.pen_prm[1], (T)1);
            pf->coefficient_of_friction = (T)o.friction;
            this->Add_Force(*pf);
        }
    }

    IMPLICIT_OBJECT<TV>* Plane_Object(const VECTOR<T, 3>& n, const VECTOR<T, 3>& x0)
    {return new ANALYTIC_IMPLICIT_OBJECT<PLANE<T> >(PLANE<T>(n, x0));}
    IMPLICIT_OBJECT<TV>* Plane_Object(const VECTOR<T, 2>&, const VECTOR<T, 2>&)
    {throw std::runtime_error("plane objects are only wired for 3D in the runner");}

    void Add_Plane(const VECTOR<T, 3>& n, const VECTOR<T, 3>& x0, COLLISION_TYPE type, T friction,
        std::function<FRAME<TV>(T)> frame, std::function<TWIST<TV>(T)> twist)
    {this->Add_Collision_Object(PLANE<T>(n, x0), type, friction, frame, twist);}
    void Add_Plane(const VECTOR<T, 2>&, const VECTOR<T, 2>&, COLLISION_TYPE, T, std::function<FRAME<TV>(T)>,
        std::function<TWIST<TV>(T)>)
    {throw std::runtime_error("plane objects are only wired for 3D in the runner");}
};
}  // namespace
